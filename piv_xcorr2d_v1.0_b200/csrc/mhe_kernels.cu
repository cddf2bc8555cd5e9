// mhe_kernels.cu -- MHE contrast enhancement (X/MHE7_4_gpu.cu), integer and
// bit-exact with the reference.  Two kernels, one warp per ws x ws tile:
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

// One warp per ws x ws tile, 8 tiles per CTA, and no CTA-wide barrier: a tile's work is
// short, so a CTA per tile spent most of its life in launch and barrier latency.
// A tile's pixels are read as 4-byte words when the tile start, the width and the pitch
// allow it (the usual case), else byte by byte; each lane fetches a batch of kBatch
// elements before using any of them, so the loads overlap.
constexpr int kTilesPerCta = 8;
constexpr int kBatch = 16;

__device__ __forceinline__ bool mhe_words(const uint8_t *p, int pitch, int ws)
{
    return ((reinterpret_cast<uintptr_t>(p) & 3) == 0) && (pitch % 4 == 0) && (ws % 4 == 0);
}

// q / d by a multiply with ceil(2^32 / d) and a 32-bit shift: exact while q * d < 2^32
// (the reciprocal's rounding error then stays below 1/d), which tile sizes here satisfy.
__device__ __forceinline__ int div_small(int q, uint64_t magic) { return (int)(((uint64_t)q * magic) >> 32); }
__host__ __device__ inline uint64_t div_magic(int d) { return (0x100000000ull + (uint64_t)d - 1) / (uint64_t)d; }

__global__ void __launch_bounds__(256) mhe_hist_kernel(const MheGeom m, const uint8_t *in, int in_pitch, int *levels)
{
    __shared__ int h[kTilesPerCta][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kTilesPerCta + warp;
    int *hw = h[warp];
#pragma unroll
    for (int b = lane; b < 256; b += 32) hw[b] = 0;
    __syncwarp();
    if (tile >= m.maxI * m.maxJ) return;  // warp-uniform
    const int ty = tile / m.maxJ, tx = tile - ty * m.maxJ;
    const uint8_t *src = in + (size_t)(m.ys + ty * m.ws) * in_pitch + m.xs + tx * m.ws;
    if (mhe_words(src, in_pitch, m.ws)) {
        const int wpr = m.ws / 4, nw = wpr * m.ws;
        const uint64_t mg = div_magic(wpr);
        for (int base = 0; base < nw; base += 32 * kBatch) {
            uint32_t v[kBatch];
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int q = base + k * 32 + lane;
                v[k] = 0;
                if (q < nw) {
                    const int r = div_small(q, mg), c = q - r * wpr;
                    v[k] = __ldg(reinterpret_cast<const uint32_t *>(src + (size_t)r * in_pitch) + c);
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                if (base + k * 32 + lane < nw) {
                    atomicAdd(&hw[v[k] & 0xff], 1);
                    atomicAdd(&hw[(v[k] >> 8) & 0xff], 1);
                    atomicAdd(&hw[(v[k] >> 16) & 0xff], 1);
                    atomicAdd(&hw[v[k] >> 24], 1);
                }
            }
        }
    } else {
        const int npx = m.ws * m.ws;
        const uint64_t mg = div_magic(m.ws);
        for (int base = 0; base < npx; base += 32 * kBatch) {
            int v[kBatch];
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int p = base + k * 32 + lane;
                v[k] = -1;
                if (p < npx) {
                    const int r = div_small(p, mg), c = p - r * m.ws;
                    v[k] = __ldg(src + (size_t)r * in_pitch + c);
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k)
                if (v[k] >= 0) atomicAdd(&hw[v[k]], 1);
        }
    }
    __syncwarp();
    int *dst = levels + ((size_t)(ty + 1) * (m.maxJ + 2) + 1 + tx) * 256;
#pragma unroll
    for (int b = lane; b < 256; b += 32) dst[b] = hw[b];
}

__global__ void __launch_bounds__(256) mhe_apply_kernel(const MheGeom m, const uint8_t *in, int in_pitch,
                                                        const int *levels, uint8_t *out, int out_pitch, int ox, int oy)
{
    __shared__ __align__(16) uint8_t lut_all[kTilesPerCta][256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x * kTilesPerCta + warp;
    if (tile >= m.maxI * m.maxJ) return;  // warp-uniform; nothing below syncs the CTA
    uint8_t *lut = lut_all[warp];
    const int ty = tile / m.maxJ, tx = tile - ty * m.maxJ;
    const int W = m.maxJ + 2;
    const int c = (ty + 1) * W + 1 + tx;
    const uint8_t *src = in + (size_t)(m.ys + ty * m.ws) * in_pitch + m.xs + tx * m.ws;
    uint8_t *dst = out + (size_t)(oy + m.ys + ty * m.ws) * out_pitch + ox + m.xs + tx * m.ws;
    const bool words = mhe_words(src, in_pitch, m.ws) && mhe_words(dst, out_pitch, m.ws);
    const int wpr = m.ws / 4, nw = wpr * m.ws;
    const uint64_t mgw = div_magic(wpr > 0 ? wpr : 1);
    // the first batch of the tile's pixels is fetched before the LUT is built
    uint32_t pre[kBatch];
    if (words) {
#pragma unroll
        for (int k = 0; k < kBatch; ++k) {
            const int q = k * 32 + lane;
            pre[k] = 0;
            if (q < nw) {
                const int r = div_small(q, mgw), cc = q - r * wpr;
                pre[k] = __ldg(reinterpret_cast<const uint32_t *>(src + (size_t)r * in_pitch) + cc);
            }
        }
    }
    // CreateTransfer_kernel: 3x3 tile neighbourhood of the zero-ringed grid; this lane
    // owns bins [8 lane, 8 lane + 8)
    int tr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            const int4 *h = reinterpret_cast<const int4 *>(levels + (size_t)(c + dy * W + dx) * 256 + 8 * lane);
            const int4 u = __ldg(h), w = __ldg(h + 1);
            tr[0] += u.x;
            tr[1] += u.y;
            tr[2] += u.z;
            tr[3] += u.w;
            tr[4] += w.x;
            tr[5] += w.y;
            tr[6] += w.z;
            tr[7] += w.w;
        }
    // inclusive prefix sum over the 256 bins (prescan_kernel + its one-element shift):
    // within the lane, then an exclusive warp scan of the lane totals
#pragma unroll
    for (int i = 1; i < 8; ++i) tr[i] += tr[i - 1];
    int incl = tr[7];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int n = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += n;
    }
    const int excl = incl - tr[7];
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
    uint32_t lv[2] = {0u, 0u};
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int b = 8 * lane + i;
        int cum = tr[i] + excl - cnt * m.Ntrash;
        cum = (cum >= 0) ? cum : 0;
        cum = min(255, cum * 255 / (cnt * m.Nnontrash));
        if (b == 0) cum = 0;
        if (b == 255) cum = 255;
        lv[i >> 2] |= (uint32_t)cum << (8 * (i & 3));
    }
    reinterpret_cast<uint2 *>(lut)[lane] = make_uint2(lv[0], lv[1]);
    __syncwarp();
    // Enhanced_kernel on this tile
    if (words) {
        for (int base = 0; base < nw; base += 32 * kBatch) {
            uint32_t w[kBatch];
            if (base == 0) {
#pragma unroll
                for (int k = 0; k < kBatch; ++k) w[k] = pre[k];
            } else {
#pragma unroll
                for (int k = 0; k < kBatch; ++k) {
                    const int q = base + k * 32 + lane;
                    w[k] = 0;
                    if (q < nw) {
                        const int r = div_small(q, mgw), cc = q - r * wpr;
                        w[k] = __ldg(reinterpret_cast<const uint32_t *>(src + (size_t)r * in_pitch) + cc);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int q = base + k * 32 + lane;
                if (q < nw) {
                    const int r = div_small(q, mgw), cc = q - r * wpr;
                    const uint32_t o = (uint32_t)lut[w[k] & 0xff] | ((uint32_t)lut[(w[k] >> 8) & 0xff] << 8) |
                                       ((uint32_t)lut[(w[k] >> 16) & 0xff] << 16) | ((uint32_t)lut[w[k] >> 24] << 24);
                    reinterpret_cast<uint32_t *>(dst + (size_t)r * out_pitch)[cc] = o;
                }
            }
        }
    } else {
        const int npx = m.ws * m.ws;
        const uint64_t mgp = div_magic(m.ws);
        for (int base = 0; base < npx; base += 32 * kBatch) {
            int px[kBatch];
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int p = base + k * 32 + lane;
                px[k] = 0;
                if (p < npx) {
                    const int r = div_small(p, mgp), cc = p - r * m.ws;
                    px[k] = __ldg(src + (size_t)r * in_pitch + cc);
                }
            }
#pragma unroll
            for (int k = 0; k < kBatch; ++k) {
                const int p = base + k * 32 + lane;
                if (p < npx) {
                    const int r = div_small(p, mgp), cc = p - r * m.ws;
                    dst[(size_t)r * out_pitch + cc] = lut[px[k]];
                }
            }
        }
    }
}

cudaError_t launch_mhe(const MheGeom &m, const uint8_t *in, int in_pitch, int *levels, uint8_t *out, int out_pitch,
                       int ox, int oy, cudaStream_t s)
{
    const int ctas = (m.maxI * m.maxJ + kTilesPerCta - 1) / kTilesPerCta;
    mhe_hist_kernel<<<ctas, 32 * kTilesPerCta, 0, s>>>(m, in, in_pitch, levels);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    mhe_apply_kernel<<<ctas, 32 * kTilesPerCta, 0, s>>>(m, in, in_pitch, levels, out, out_pitch, ox, oy);
    return cudaGetLastError();
}

}  // namespace piv
