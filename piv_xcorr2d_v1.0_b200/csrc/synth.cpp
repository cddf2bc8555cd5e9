// synth.cpp -- seeded synthetic PIV image pairs (no counterpart in the reference; it
// stands in for the missing sample TIFFs and for the public benchmark data the
// reference never shipped).
//
// Particles: uniform positions over the image plus a 32 px margin at density ppp,
// peak intensity U(i_min, i_max), pixel-integrated Gaussian spots
//   I(px) = I0 * gx(px) * gy(py),
//   gx(px) = [erf((px+0.5-xp)/(sqrt2 s)) - erf((px-0.5-xp)/(sqrt2 s))] / (2 erf(0.5/(sqrt2 s))),
// so a particle centred on a pixel gives I0 there.  Frame 2 moves every particle by
// the field evaluated at its frame-1 position (x2 = x1 + u(x1)).  Background and
// Gaussian noise are added per pixel, then clipped to [0, 255] and rounded.
// Random numbers and field models: synth_model.h (shared with the device generator,
// synth_device.cu), so every value is reproducible and independent of evaluation order.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "piv_b200.h"
#include "synth_model.h"

namespace {

using piv::kStreamNoise;
using piv::kStreamParticle;
using piv::philox;
using piv::U4;
using piv::u01;

void render(std::vector<float> &acc, int Nx, int Ny, double xp, double yp, double I0, double sigma, double norm)
{
    const double rad = 3.0 * sigma + 1.0, k = 1.0 / (std::sqrt(2.0) * sigma);
    int x0 = (int)std::floor(xp - rad), x1 = (int)std::ceil(xp + rad);
    int y0 = (int)std::floor(yp - rad), y1 = (int)std::ceil(yp + rad);
    if (x1 < 0 || y1 < 0 || x0 >= Nx || y0 >= Ny) return;
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    if (x1 > Nx - 1) x1 = Nx - 1;
    if (y1 > Ny - 1) y1 = Ny - 1;
    double gx[16], gy[16];
    const int nx = x1 - x0 + 1, ny = y1 - y0 + 1;
    if (nx > 16 || ny > 16) return;
    for (int i = 0; i < nx; ++i) {
        double px = x0 + i;
        gx[i] = (std::erf((px + 0.5 - xp) * k) - std::erf((px - 0.5 - xp) * k)) * norm;
    }
    for (int j = 0; j < ny; ++j) {
        double py = y0 + j;
        gy[j] = (std::erf((py + 0.5 - yp) * k) - std::erf((py - 0.5 - yp) * k)) * norm;
    }
    for (int j = 0; j < ny; ++j) {
        float *row = acc.data() + (size_t)(y0 + j) * Nx + x0;
        const double a = I0 * gy[j];
        for (int i = 0; i < nx; ++i) row[i] += (float)(a * gx[i]);
    }
}

void finish(const std::vector<float> &acc, const piv_synth_params *s, uint32_t frame, uint8_t *out)
{
    const size_t n = (size_t)s->Nx * s->Ny;
    for (size_t i = 0; i < n; i += 2) {
        // Box-Muller: two normals per Philox draw
        U4 r = philox((uint32_t)i, (uint32_t)(i >> 32), kStreamNoise, frame, s->seed);
        double rr = std::sqrt(-2.0 * std::log(u01(r.v[0]))), th = 2 * piv::kSynthPi * u01(r.v[1]);
        double z[2] = {rr * std::cos(th), rr * std::sin(th)};
        for (int q = 0; q < 2 && i + q < n; ++q) {
            double v = s->background + acc[i + q] + s->noise_sigma * z[q];
            v = v < 0 ? 0 : (v > 255 ? 255 : v);
            out[i + q] = (uint8_t)std::floor(v + 0.5);
        }
    }
}

}  // namespace

extern "C" {

int piv_synth_field(const piv_synth_params *s, const float *x, const float *y, int n, float *u, float *v)
{
    if (!s || !x || !y || !u || !v || n < 0) return PIV_ERR_ARG;
    const piv::SynthModel f = piv::synth_model(s);
    for (int i = 0; i < n; ++i) {
        double uu, vv;
        piv::synth_eval(f, x[i], y[i], uu, vv);
        u[i] = (float)uu;
        v[i] = (float)vv;
    }
    return PIV_OK;
}

int piv_synth_pair(const piv_synth_params *s, uint8_t *f1, uint8_t *f2)
{
    if (!s || !f1 || !f2 || s->Nx < 1 || s->Ny < 1 || s->ppp < 0 || s->sigma <= 0) return PIV_ERR_ARG;
    const int m = 32;
    const double W = s->Nx + 2.0 * m, H = s->Ny + 2.0 * m;
    const long np = std::lround(s->ppp * W * H);
    const piv::SynthModel fld = piv::synth_model(s);
    const double norm = 1.0 / (2.0 * std::erf(0.5 / (std::sqrt(2.0) * s->sigma)));
    std::vector<float> a1((size_t)s->Nx * s->Ny, 0.f), a2((size_t)s->Nx * s->Ny, 0.f);
    for (long p = 0; p < np; ++p) {
        U4 r = philox((uint32_t)p, (uint32_t)(p >> 32), kStreamParticle, 0, s->seed);
        const double xp = u01(r.v[0]) * W - m, yp = u01(r.v[1]) * H - m;
        const double I0 = s->i_min + (s->i_max - s->i_min) * u01(r.v[2]);
        double u, v;
        piv::synth_eval(fld, xp, yp, u, v);
        render(a1, s->Nx, s->Ny, xp, yp, I0, s->sigma, norm);
        render(a2, s->Nx, s->Ny, xp + u, yp + v, I0, s->sigma, norm);
    }
    finish(a1, s, 0, f1);
    finish(a2, s, 1, f2);
    return PIV_OK;
}

}  // extern "C"
