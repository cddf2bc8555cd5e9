// mhe_kernels.cu -- MHE contrast enhancement (X/MHE7_4_gpu.cu), integer and
// bit-exact with the reference.  Two kernels, one CTA per ws x ws tile:
//   mhe_hist_kernel   MakeHist_kernel (:66) with per-warp shared-memory histograms
//                     instead of global atomics; written into a zero-ringed tile grid.
//   mhe_apply_kernel  CreateTransfer_kernel (:85) + prescan_kernel (:5) +
//                     Calc_Enhanced_value_kernel (:103) + Enhanced_kernel (:121):
//                     9-tile transfer histogram, inclusive prefix sum, threshold
//                     stretch to a 256-entry LUT, LUT applied to the tile's pixels.
// The neighbour count of Calc_cnt_neigh_kernel (:45) is computed inline.
#include <cmath>

#include "piv_common.cuh"

namespace piv {

bool mhe_geometry(int Nx, int Ny, int ws, float thresh, MheGeom &m)
{
    if (Nx < 1 || Ny < 1 || ws < 1) return false;
    m.Nx = Nx;
    m.Ny = Ny;
    m.ws = ws;
    // mhe_gpu::init (X/MHE7_4_gpu.cu:157-178)
    if (Nx % ws == 0 && Ny % ws == 0) {
        m.height = Ny;
        m.width = Nx;
        m.xs = 0;
        m.ys = 0;
    } else {
        m.width = ws * (Nx / ws);
        m.xs = (Nx - m.width) / 2;
        m.height = ws * (Ny / ws);
        m.ys = (Ny - m.height) / 2;
    }
    m.maxI = m.height / ws;
    m.maxJ = m.width / ws;
    m.Ntrash = (int)roundf((float)(ws * ws) * thresh);
    m.Nnontrash = ws * ws - m.Ntrash;
    return m.maxI >= 1 && m.maxJ >= 1 && m.Nnontrash > 0;
}

// A tile's pixels are read as 4-byte words when the tile start, the width and the pitch
// allow it (the usual case), else byte by byte.  Each thread fetches a batch of kBatch
// elements before using any of them, so the loads overlap instead of paying the
// memory latency once per element.
constexpr int kBatch = 8;

__device__ __forceinline__ bool mhe_words(const uint8_t *p, int pitch, int ws)
{
    return ((reinterpret_cast<uintptr_t>(p) & 3) == 0) && (pitch % 4 == 0) && (ws % 4 == 0);
}

__global__ void __launch_bounds__(256) mhe_hist_kernel(const MheGeom m, const uint8_t *in, int in_pitch, int *levels)
{
    // one histogram per warp (fewer same-address collisions), summed at the end
    __shared__ int h[8][256];
    const int tid = threadIdx.x, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < 8; ++q) h[q][tid] = 0;
    __syncthreads();
    const int ty = blockIdx.x / m.maxJ, tx = blockIdx.x - ty * m.maxJ;
    const uint8_t *src = in + (size_t)(m.ys + ty * m.ws) * in_pitch + m.xs + tx * m.ws;
    int *hw = h[warp];
    if (mhe_words(src, in_pitch, m.ws)) {
        const int wpr = m.ws / 4, nw = wpr * m.ws;
        for (int base = 0; base < nw; base += 256 * kBatch) {
            uint32_t v[kBatch];
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int q = base + k * 256 + tid;
                v[k] = 0;
                if (q < nw) {
                    const int r = q / wpr, c = q - r * wpr;
                    v[k] = __ldg(reinterpret_cast<const uint32_t *>(src + (size_t)r * in_pitch) + c);
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                if (base + k * 256 + tid < nw) {
                    atomicAdd(&hw[v[k] & 0xff], 1);
                    atomicAdd(&hw[(v[k] >> 8) & 0xff], 1);
                    atomicAdd(&hw[(v[k] >> 16) & 0xff], 1);
                    atomicAdd(&hw[v[k] >> 24], 1);
                }
            }
        }
    } else {
        const int npx = m.ws * m.ws;
        for (int base = 0; base < npx; base += 256 * kBatch) {
            int v[kBatch];
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int p = base + k * 256 + tid;
                v[k] = -1;
                if (p < npx) {
                    const int r = p / m.ws, c = p - r * m.ws;
                    v[k] = __ldg(src + (size_t)r * in_pitch + c);
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k)
                if (v[k] >= 0) atomicAdd(&hw[v[k]], 1);
        }
    }
    __syncthreads();
    int t = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t += h[q][tid];
    levels[((size_t)(ty + 1) * (m.maxJ + 2) + 1 + tx) * 256 + tid] = t;
}

__global__ void __launch_bounds__(256) mhe_apply_kernel(const MheGeom m, const uint8_t *in, int in_pitch,
                                                        const int *levels, uint8_t *out, int out_pitch, int ox, int oy)
{
    __shared__ int wsum[8];
    __shared__ uint8_t lut[256];
    const int b = threadIdx.x, lane = b & 31, warp = b >> 5;
    const int ty = blockIdx.x / m.maxJ, tx = blockIdx.x - ty * m.maxJ;
    const int W = m.maxJ + 2;
    const int c = (ty + 1) * W + 1 + tx;
    const uint8_t *src = in + (size_t)(m.ys + ty * m.ws) * in_pitch + m.xs + tx * m.ws;
    uint8_t *dst = out + (size_t)(oy + m.ys + ty * m.ws) * out_pitch + ox + m.xs + tx * m.ws;
    const bool words = mhe_words(src, in_pitch, m.ws) && mhe_words(dst, out_pitch, m.ws);
    const int wpr = m.ws / 4, nw = wpr * m.ws;
    // the first batch of the tile's pixels is fetched before the LUT is built
    uint32_t pre[kBatch];
    if (words) {
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const int q = k * 256 + b;
            pre[k] = 0;
            if (q < nw) {
                const int r = q / wpr, cc = q - r * wpr;
                pre[k] = __ldg(reinterpret_cast<const uint32_t *>(src + (size_t)r * in_pitch) + cc);
            }
        }
    }
    // CreateTransfer_kernel: 3x3 tile neighbourhood of the zero-ringed grid
    int tr = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) tr += __ldg(levels + (size_t)(c + dy * W + dx) * 256 + b);
    // inclusive prefix sum over the 256 bins (prescan_kernel + its one-element shift)
    int v = tr;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int n = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += n;
    }
    if (lane == 31) wsum[warp] = v;
    __syncthreads();
    int base = 0;
    for (int q = 0; q < warp; ++q) base += wsum[q];
    int cum = v + base;
    // Calc_cnt_neigh_kernel with (Nx, Ny) = (maxJ, maxI)
    int cnt;
    if (tx >= 1 && tx <= m.maxJ - 2 && ty >= 1 && ty <= m.maxI - 2)
        cnt = 9;
    else if ((tx == 0 && ty == 0) || (tx == 0 && ty == m.maxI - 1) || (tx == m.maxJ - 1 && ty == 0) ||
             (tx == m.maxJ - 1 && ty == m.maxI - 1))
        cnt = 4;
    else
        cnt = 6;
    // Calc_Enhanced_value_kernel
    cum = cum - cnt * m.Ntrash;
    cum = (cum >= 0) ? cum : 0;
    cum = min(255, cum * 255 / (cnt * m.Nnontrash));
    if (b == 0) cum = 0;
    if (b == 255) cum = 255;
    lut[b] = (uint8_t)cum;
    __syncthreads();
    // Enhanced_kernel on this tile
    if (words) {
        for (int base = 0; base < nw; base += 256 * kBatch) {
            uint32_t w[kBatch];
            if (base == 0) {
#pragma unroll
                for (int k = 0; k < kBatch; ++k) w[k] = pre[k];
            } else {
#pragma unroll
                for (int k = 0; k < kBatch; ++k) {
                    const int q = base + k * 256 + b;
                    w[k] = 0;
                    if (q < nw) {
                        const int r = q / wpr, cc = q - r * wpr;
                        w[k] = __ldg(reinterpret_cast<const uint32_t *>(src + (size_t)r * in_pitch) + cc);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int q = base + k * 256 + b;
                if (q < nw) {
                    const int r = q / wpr, cc = q - r * wpr;
                    const uint32_t o = (uint32_t)lut[w[k] & 0xff] | ((uint32_t)lut[(w[k] >> 8) & 0xff] << 8) |
                                       ((uint32_t)lut[(w[k] >> 16) & 0xff] << 16) | ((uint32_t)lut[w[k] >> 24] << 24);
                    reinterpret_cast<uint32_t *>(dst + (size_t)r * out_pitch)[cc] = o;
                }
            }
        }
    } else {
        const int npx = m.ws * m.ws;
        for (int base = 0; base < npx; base += 256 * kBatch) {
            int px[kBatch];
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int p = base + k * 256 + b;
                px[k] = 0;
                if (p < npx) {
                    const int r = p / m.ws, cc = p - r * m.ws;
                    px[k] = __ldg(src + (size_t)r * in_pitch + cc);
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int p = base + k * 256 + b;
                if (p < npx) {
                    const int r = p / m.ws, cc = p - r * m.ws;
                    dst[(size_t)r * out_pitch + cc] = lut[px[k]];
                }
            }
        }
    }
}

cudaError_t launch_mhe(const MheGeom &m, const uint8_t *in, int in_pitch, int *levels, uint8_t *out, int out_pitch,
                       int ox, int oy, cudaStream_t s)
{
    const int tiles = m.maxI * m.maxJ;
    mhe_hist_kernel<<<tiles, 256, 0, s>>>(m, in, in_pitch, levels);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    mhe_apply_kernel<<<tiles, 256, 0, s>>>(m, in, in_pitch, levels, out, out_pitch, ox, oy);
    return cudaGetLastError();
}

}  // namespace piv
