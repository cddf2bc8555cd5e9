// synth_device.cu -- the synthetic particle-image generator on the GPU (no counterpart in
// the reference).  It draws the same particles, displacement field and noise as the host
// generator piv_synth_pair (synth.cpp; shared streams in synth_model.h) and renders the
// same pixel-integrated Gaussian spots, one thread per particle accumulating with atomic
// adds.  Only the order of the float accumulation differs from the host, so a pixel can
// differ by one grey level where its value sits on a rounding tie.  It exists to make
// training sets of thousands of pairs in seconds.
#include <cuda_runtime.h>

#include "piv_b200.h"
#include "synth_model.h"

namespace piv {
namespace {

struct SynthDev {
    SynthModel m;
    int Nx, Ny;
    long np;
    double W, H, margin;
    double i_min, i_span, sigma, k, norm, rad;
    double background, noise_sigma;
    uint64_t seed;
};

__device__ void render_spot(float *acc, const SynthDev &d, double xp, double yp, double I0)
{
    int x0 = (int)floor(xp - d.rad), x1 = (int)ceil(xp + d.rad);
    int y0 = (int)floor(yp - d.rad), y1 = (int)ceil(yp + d.rad);
    if (x1 < 0 || y1 < 0 || x0 >= d.Nx || y0 >= d.Ny) return;
    x0 = max(x0, 0);
    y0 = max(y0, 0);
    x1 = min(x1, d.Nx - 1);
    y1 = min(y1, d.Ny - 1);
    const int nx = x1 - x0 + 1, ny = y1 - y0 + 1;
    if (nx > 16 || ny > 16) return;
    double gx[16];
    for (int i = 0; i < nx; ++i) {
        const double px = x0 + i;
        gx[i] = (erf((px + 0.5 - xp) * d.k) - erf((px - 0.5 - xp) * d.k)) * d.norm;
    }
    for (int j = 0; j < ny; ++j) {
        const double py = y0 + j;
        const double gy = (erf((py + 0.5 - yp) * d.k) - erf((py - 0.5 - yp) * d.k)) * d.norm;
        const double a = I0 * gy;
        float *row = acc + (size_t)(y0 + j) * d.Nx + x0;
        for (int i = 0; i < nx; ++i) atomicAdd(row + i, (float)(a * gx[i]));
    }
}

__global__ void particle_kernel(const SynthDev d, float *acc1, float *acc2)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= d.np) return;
    const U4 r = philox((uint32_t)p, (uint32_t)(p >> 32), kStreamParticle, 0, d.seed);
    const double xp = u01(r.v[0]) * d.W - d.margin, yp = u01(r.v[1]) * d.H - d.margin;
    const double I0 = d.i_min + d.i_span * u01(r.v[2]);
    double u, v;
    synth_eval(d.m, xp, yp, u, v);
    render_spot(acc1, d, xp, yp, I0);
    render_spot(acc2, d, xp + u, yp + v, I0);
}

// background + spots + Box-Muller noise (two normals per Philox draw), clipped, rounded
__global__ void finish_kernel(const SynthDev d, const float *acc1, const float *acc2, uint8_t *f1, uint8_t *f2)
{
    const size_t n = (size_t)d.Nx * d.Ny;
    const size_t i = 2 * ((size_t)blockIdx.x * blockDim.x + threadIdx.x);
    const uint32_t frame = blockIdx.y;
    if (i >= n) return;
    const float *acc = frame ? acc2 : acc1;
    uint8_t *out = frame ? f2 : f1;
    const U4 r = philox((uint32_t)i, (uint32_t)(i >> 32), kStreamNoise, frame, d.seed);
    const double rr = sqrt(-2.0 * log(u01(r.v[0]))), th = 2 * kSynthPi * u01(r.v[1]);
    const double z[2] = {rr * cos(th), rr * sin(th)};
    for (int q = 0; q < 2 && i + q < n; ++q) {
        double v = d.background + acc[i + q] + d.noise_sigma * z[q];
        v = v < 0 ? 0 : (v > 255 ? 255 : v);
        out[i + q] = (uint8_t)floor(v + 0.5);
    }
}

}  // namespace
}  // namespace piv

extern "C" int piv_synth_pair_device(const piv_synth_params *s, uint8_t *d_f1, uint8_t *d_f2, float *d_scratch,
                                     void *stream)
{
    using namespace piv;
    if (!s || !d_f1 || !d_f2 || !d_scratch || s->Nx < 1 || s->Ny < 1 || s->ppp < 0 || s->sigma <= 0)
        return PIV_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    SynthDev d;
    d.m = synth_model(s);
    d.Nx = s->Nx;
    d.Ny = s->Ny;
    d.margin = 32;
    d.W = s->Nx + 2.0 * d.margin;
    d.H = s->Ny + 2.0 * d.margin;
    d.np = std::lround(s->ppp * d.W * d.H);
    d.i_min = s->i_min;
    d.i_span = s->i_max - s->i_min;
    d.sigma = s->sigma;
    d.k = 1.0 / (std::sqrt(2.0) * s->sigma);
    d.norm = 1.0 / (2.0 * std::erf(0.5 / (std::sqrt(2.0) * s->sigma)));
    d.rad = 3.0 * s->sigma + 1.0;
    d.background = s->background;
    d.noise_sigma = s->noise_sigma;
    d.seed = s->seed;
    const size_t n = (size_t)s->Nx * s->Ny;
    float *acc1 = d_scratch, *acc2 = d_scratch + n;
    if (cudaMemsetAsync(d_scratch, 0, 2 * n * sizeof(float), st) != cudaSuccess) return PIV_ERR_CUDA;
    if (d.np > 0) {
        const int tb = 128;
        particle_kernel<<<(unsigned)((d.np + tb - 1) / tb), tb, 0, st>>>(d, acc1, acc2);
        if (cudaGetLastError() != cudaSuccess) return PIV_ERR_CUDA;
    }
    const size_t pairs = (n + 1) / 2;
    finish_kernel<<<dim3((unsigned)((pairs + 255) / 256), 2), 256, 0, st>>>(d, acc1, acc2, d_f1, d_f2);
    if (cudaGetLastError() != cudaSuccess) return PIV_ERR_CUDA;
    return PIV_OK;
}
