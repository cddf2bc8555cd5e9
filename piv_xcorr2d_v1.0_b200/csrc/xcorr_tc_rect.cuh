// xcorr_tc_rect.cuh -- the tensor-core correlation kernel for the non-square windows 48x24 and
// 24x48 (WX columns, WY rows).  Same contract and the same four DFT-product passes as the
// square kernel (xcorr_tc.cuh; the reference's organize_data_fft2d_multi(_deformed),
// cufftExecC2C x3, multiply_conjugate, complex2amp, fftshift, find_local_max_2d ..
// kernel_remove_nan, X/xcorr2d_multi_grid.cu:497-654, 1334-1347, 1649-1662), with two
// DFT matrices:
//   Gx = [[Cx, -Sx], [Sx, Cx]] (2WX x 2WX) and Gy (2WY x 2WY), once per CTA in shared memory.
// A tile is 2 windows; its rows per pass:
//   A  (window, y)   x [f1 row | f2 row]      * Gx        K = 2WX, N = 2WX   2*WY rows
//   B  (window, kx)  x [re | im] over y       * Gy        K = 2WY, N = 2WY   2*WX rows
//   C  (window, kx)  x [re | im] over ky      * Gy^T      K = 2WY, N = 2WY   2*WX rows
//   D  (window, y)   x [re | im] over kx      * Gx^T[:, :WX]  K = 2WX, N = WX (x16)  2*WY rows
// of the 128-row MMA (the unused rows are computed and ignored).  The pass-B rows of a window
// are ordered so that every warp's share of its columns is closed under kx -> -kx (the cross
// spectrum's partner column is a shuffle away).  Operand scales for FP16 are powers of two
// (rounded up from WX and WY); the plane is |out| * 2^s (exact) * 1/N as in the SIMT kernel.
// Waits are bounded as in the square kernel.
#pragma once
#include "xcorr_tc.cuh"

namespace piv {

// Pass-B row order of window wl (0 or 1) of a tile: its rows wl*WX + p, p < WX, split at warp
// boundaries into segments; the first segment takes kx = 0 and WX/2 (their own partners) and
// then pairs (k, WX - k) in increasing k, the next segments the following pairs.  Every
// segment has even size, so each is closed under negation.
template <int WX>
struct RectOrder {
    int col[2][WX];  // column at position p
    int pos[2][WX];  // position of column kx
};
template <int WX>
constexpr RectOrder<WX> make_rect_order()
{
    RectOrder<WX> o{};
    for (int wl = 0; wl < 2; ++wl) {
        int p = 0, next_pair = 1;
        bool singles_done = false;
        const int row0 = wl * WX;
        while (p < WX) {
            const int seg_end_row = ((row0 + p) / 32 + 1) * 32;  // end of the warp holding row0 + p
            const int seg = (seg_end_row - row0 < WX ? seg_end_row - row0 : WX) - p;
            int filled = 0;
            if (!singles_done) {
                o.col[wl][p + filled++] = 0;
                o.col[wl][p + filled++] = WX / 2;
                singles_done = true;
            }
            while (filled < seg) {
                o.col[wl][p + filled++] = next_pair;
                o.col[wl][p + filled++] = WX - next_pair;
                ++next_pair;
            }
            p += seg;
        }
        for (int q = 0; q < WX; ++q) o.pos[wl][o.col[wl][q]] = q;
    }
    return o;
}
template <int WX>
__constant__ RectOrder<WX> kRectOrder = make_rect_order<WX>();

// whether rows [r0, r1) of a warpgroup hold no nonzero pixel, from the 4 warps' row ballots
__device__ __forceinline__ bool rows_dead(const uint32_t (&nz)[4], int r0, int r1)
{
    uint32_t any = 0;
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        const int lo = max(r0, 32 * w) - 32 * w, hi = min(r1, 32 * w + 32) - 32 * w;
        if (lo < hi) {
            const uint32_t m = (hi - lo == 32) ? 0xffffffffu : (((1u << (hi - lo)) - 1u) << lo);
            any |= nz[w] & m;
        }
    }
    return any == 0u;
}

// N consecutive TMEM columns of this warp's lanes (N a multiple of 8): loads of 32, then 16,
// then 8 columns
template <int N>
__device__ __forceinline__ void tmem_cols(uint32_t taddr, float *v)
{
    static_assert(N % 8 == 0, "a multiple of 8 columns");
#pragma unroll
    for (int c = 0; c < N / 32; ++c) {
        float t[32];
        tc::tmem_ld32(taddr + 32 * c, t);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[32 * c + i] = t[i];
    }
    constexpr int b16 = 32 * (N / 32);
    if constexpr ((N - b16) >= 16) {
        float t[16];
        tc::tmem_ld16(taddr + b16, t);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[b16 + i] = t[i];
    }
    constexpr int b8 = b16 + ((N - b16) >= 16 ? 16 : 0);
    if constexpr ((N - b8) == 8) {
        float t[8];
        tc::tmem_ld8(taddr + b8, t);
#pragma unroll
        for (int i = 0; i < 8; ++i) v[b8 + i] = t[i];
    }
}

constexpr int pow2_at_least(int n)
{
    int p = 1;
    while (p < n) p *= 2;
    return p;
}

template <int WX, int WY>
struct TcRectShape {
    static constexpr int KX = 2 * WX, KY = 2 * WY;       // complex extents as re | im
    static constexpr int NG = 3;                         // warpgroups per CTA
    static constexpr int THREADS = 128 * NG;
    static constexpr int KMAX = KX > KY ? KX : KY;
    static constexpr uint32_t GX_BYTES = KX * KX * 2;    // one of Gx hi / lo
    static constexpr uint32_t GY_BYTES = KY * KY * 2;
    static constexpr uint32_t A_BYTES = 128 * KMAX * 2;  // one of A hi / lo
    static constexpr int TCOLS = 128;                    // TMEM columns per warpgroup (N <= 96)
    static constexpr size_t SMEM = 2 * (size_t)GX_BYTES + 2 * (size_t)GY_BYTES + (size_t)NG * 2 * A_BYTES;
    static_assert(KMAX <= 128 && 2 * WX <= 128 && 2 * WY <= 128, "two windows per 128-row tile");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

// Gx or Gy = [[C, -S], [S, C]] (K x K, K = 2n), hi / lo, in the shared layout buf(r, c)
template <int n, bool F16>
__device__ __forceinline__ void fill_dft(uint8_t *hi, uint8_t *lo, const float *cs, const float *sn, int tid,
                                         int nthreads)
{
    constexpr int K = 2 * n;
    for (int t = tid; t < K * K; t += nthreads) {
        const int gr = t / K, gc = t - gr * K;
        const int q = ((gr % n) * (gc % n)) % n;
        const float v = ((gr < n) == (gc < n)) ? cs[q] : ((gr < n) ? -sn[q] : sn[q]);
        uint16_t h, l;
        if constexpr (F16) tc::split_f16(v, h, l);
        else tc::split_bf16(v, h, l);
        const uint32_t o = (gc / 8) * (K * 16) + gr * 16 + (gc % 8) * 2;
        *reinterpret_cast<uint16_t *>(hi + o) = h;
        *reinterpret_cast<uint16_t *>(lo + o) = l;
    }
}

template <int WX, int WY, int NPROD, int K, bool DEF, bool F16>
__global__ void __launch_bounds__(TcRectShape<WX, WY>::THREADS, 1) xcorr_tc_rect_kernel(const XcorrArgs a)
{
    using S = TcRectShape<WX, WY>;
    constexpr int KX = S::KX, KY = S::KY, NG = S::NG;
    constexpr int LDF = WX + 1;  // plane row stride (peak stage)
    constexpr uint32_t GX_BYTES = S::GX_BYTES, GY_BYTES = S::GY_BYTES, A_BYTES = S::A_BYTES;
    constexpr uint32_t TCOLS = S::TCOLS, TALLOC = 512;
    // operand scales (powers of two, exact): FP16 operands take pass B's by 1/PX, the cross
    // spectrum's by 1/(2 PY^2) and pass D's by 1/(2 PY); BF16 (FP32's exponent range) keeps only
    // the cross spectrum's, folded into its constant factors
    constexpr int PX = pow2_at_least(WX), PY = pow2_at_least(WY);
    constexpr float sB = F16 ? 1.0f / (float)PX : 1.0f, sC = 1.0f / (float)(2 * PY * PY);
    constexpr float sD = F16 ? 1.0f / (float)(2 * PY) : 1.0f;
    constexpr float unscale = 1.0f / (sB * sB * sC * sD);
    // pass A's lo products start at this K step (frame 1, and frame 2 when undeformed, hold
    // integers exact in the operand type)
    constexpr int LOF = DEF ? WX / 16 : KX / 16;
    constexpr float inv_n = 1.0f / (float)(WX * WY);
    static_assert(2 * WY * LDF * 4 + 2 * sizeof(PeakPart[2]) <= 2 * A_BYTES, "planes and peak scratch fit");

    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar[NG];
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t s_nz1[NG][4], s_nz2[NG][4];

    const GridGeom &g = a.g;
    const int tid = threadIdx.x, wg = tid >> 7, lt = tid & 127;
    const int lane = tid & 31, wq = lt >> 5;
    uint8_t *gx_hi = smem, *gx_lo = smem + GX_BYTES;
    uint8_t *gy_hi = smem + 2 * GX_BYTES, *gy_lo = gy_hi + GY_BYTES;
    uint8_t *a_hi = smem + 2 * GX_BYTES + 2 * GY_BYTES + (size_t)wg * 2 * A_BYTES, *a_lo = a_hi + A_BYTES;
    float *planes = reinterpret_cast<float *>(a_hi);
    const uint32_t mb = tc::smem_u32(&mbar[wg]);
    const uint32_t bar_id = 1 + wg;

    fill_dft<WX, F16>(gx_hi, gx_lo, kTw<WX>.c, kTw<WX>.s, tid, S::THREADS);
    fill_dft<WY, F16>(gy_hi, gy_lo, kTw<WY>.c, kTw<WY>.s, tid, S::THREADS);
    if (lt == 0) {
        tc::mbar_init(mb, 1);
        tc::fence_mbar_init();
    }
    if (tid < 32) tc::tmem_alloc(tc::smem_u32(&tmem_base), TALLOC);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base + wg * TCOLS;
    const uint32_t lane_addr = tmem + ((uint32_t)(wq * 32) << 16);
    const uint32_t sa_hi = tc::smem_u32(a_hi), sa_lo = tc::smem_u32(a_lo);
    const uint32_t sgx_hi = tc::smem_u32(gx_hi), sgx_lo = tc::smem_u32(gx_lo);
    const uint32_t sgy_hi = tc::smem_u32(gy_hi), sgy_lo = tc::smem_u32(gy_lo);

    // pass A / D row (window, y) and pass B / C row (window, position of kx) of this thread
    const bool rowA = lt < 2 * WY, rowB = lt < 2 * WX;
    const int wlA = rowA ? lt / WY : 0, y = rowA ? lt - wlA * WY : 0;
    const int wlB = rowB ? lt / WX : 0, pB = rowB ? lt - wlB * WX : 0;
    const int kx = kRectOrder<WX>.col[wlB][pB];
    // the lane holding column -kx of the same window (same warp by construction)
    const int partner = rowB ? ((wlB * WX + kRectOrder<WX>.pos[wlB][(WX - kx) % WX]) & 31) : lane;

    const int n_win = a.w_end - a.w_first;
    const int n_tiles = (n_win + 1) / 2;
    uint32_t phase = 0;
    bool failed = false;
    auto wait_pass = [&]() -> bool {
        const bool ok = __all_sync(0xffffffffu, tc::mbar_wait(mb, phase & 1));
        ++phase;
        tc::fence_after_sync();
        return ok;
    };
    auto sync_issue = [&](bool ok) -> bool {
        tc::fence_async_smem();
        tc::fence_before_sync();
        const bool bad = tc::named_sync_or(bar_id, 128, !ok);
        tc::fence_after_sync();
        return !bad;
    };

    for (int tile = blockIdx.x * NG + wg; tile < n_tiles; tile += gridDim.x * NG) {
        const int w0 = a.w_first + tile * 2;

        // ---- pass A operand: row (wl, y) = [f1 row | f2 row], K-major; row ballots ----
        {
            float v1[WX], v2[WX];
            const int w = w0 + wlA;
            if (rowA && w < a.w_end) {
                const int iy = w / g.Nx_vec, ix = w - iy * g.Nx_vec;
                const int x0 = ix * g.sp_x - g.Nx_left + a.f1.mx;
                const int y1 = iy * g.sp_y + y - g.Ny_left + a.f1.my;
                load_u8_row<WX>(a.f1.base + (size_t)y1 * a.f1.pitch + x0, v1);
                if constexpr (DEF) {
                    load_f32_row<WX>(a.def + (size_t)(iy * g.sp_y + y) * a.def_pitch + ix * g.sp_x, v2);
                } else {
                    load_u8_row<WX>(a.f2.base + (size_t)y1 * a.f2.pitch + x0, v2);
                }
            } else {
#pragma unroll
                for (int i = 0; i < WX; ++i) v1[i] = v2[i] = 0.f;
            }
            const uint32_t b1 = __ballot_sync(0xffffffffu, any_nonzero<WX>(v1));
            const uint32_t b2 = __ballot_sync(0xffffffffu, any_nonzero<WX>(v2));
            if (lane == 0) {
                s_nz1[wg][wq] = b1;
                s_nz2[wg][wq] = b2;
            }
#pragma unroll
            for (int c = 0; c < WX / 8; ++c) {
                // integer columns below the lo products' first K step: the hi part only
                if (8 * c + 8 <= 16 * LOF) store8_exact<F16>(a_hi, tc::off_kmajor(lt, 8 * c, 128), v1 + 8 * c);
                else store8<NPROD, F16>(a_hi, a_lo, tc::off_kmajor(lt, 8 * c, 128), v1 + 8 * c);
                if (WX + 8 * c + 8 <= 16 * LOF) store8_exact<F16>(a_hi, tc::off_kmajor(lt, WX + 8 * c, 128), v2 + 8 * c);
                else store8<NPROD, F16>(a_hi, a_lo, tc::off_kmajor(lt, WX + 8 * c, 128), v2 + 8 * c);
            }
        }
        if (!sync_issue(true)) break;
        if (lt == 0) {
            // frame 1 is integer-valued (exact in the 16-bit formats); frame 2 only when deformed
            issue_pass<KX, KX, false, true, NPROD, LOF, F16>(tmem, sa_hi, sa_lo, sgx_hi, sgx_lo);
            tc::mma_commit(mb);
        }
        // windows with an all-zero frame: spectrum and plane 0 (the reference's exact zeros)
        const bool deadA = rows_dead(s_nz1[wg], wlA * WY, wlA * WY + WY) || rows_dead(s_nz2[wg], wlA * WY, wlA * WY + WY);
        const bool deadB = rows_dead(s_nz1[wg], wlB * WY, wlB * WY + WY) || rows_dead(s_nz2[wg], wlB * WY, wlB * WY + WY);

        // ---- pass B operand: MN-major, m = (wl, position of kx), k = (re|im, y) ----
        {
            const bool ok = wait_pass();
            if (ok) {
                float zr[WX], zi[WX];
                tmem_cols<WX>(lane_addr, zr);
                tmem_cols<WX>(lane_addr + WX, zi);
                tc::tmem_wait_ld();
                if (rowA) {
#pragma unroll
                    for (int c = 0; c < WX / 8; ++c) {
                        float br[8], bi[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const int col = kRectOrder<WX>.col[wlA][8 * c + i];
                            br[i] = zr[col];
                            bi[i] = zi[col];
                        }
                        store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wlA * WX + 8 * c, y, KY), br, sB);
                        store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wlA * WX + 8 * c, WY + y, KY), bi, sB);
                    }
                }
            }
            if (!sync_issue(ok)) {
                failed = true;
                break;
            }
        }
        if (lt == 0) {
            issue_pass<KY, KY, true, true, NPROD, 0, F16>(tmem, sa_hi, sa_lo, sgy_hi, sgy_lo);
            tc::mma_commit(mb);
        }

        // ---- cross spectrum; pass C operand: K-major row (wl, kx), k = (re|im, ky) ----
        {
            const bool ok = wait_pass();
            if (ok) {
                float zr[WY], zi[WY];
                tmem_cols<WY>(lane_addr, zr);
                tmem_cols<WY>(lane_addr + WY, zi);
                tc::tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < WY / 8; ++c) {
                    float cr[8], ci[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int ky = 8 * c + i, km = (WY - ky) % WY;
                        const float pr = __shfl_sync(0xffffffffu, zr[km], partner);
                        const float pi = __shfl_sync(0xffffffffu, zi[km], partner);
                        // scaled by sC, folded into the exact constant factors
                        cr[i] = deadB ? 0.f : (0.5f * sC) * (zr[ky] * pi + zi[ky] * pr);
                        ci[i] = deadB ? 0.f : (0.25f * sC) * ((pr * pr + pi * pi) - (zr[ky] * zr[ky] + zi[ky] * zi[ky]));
                    }
                    if (rowB) {
                        store8<NPROD, F16>(a_hi, a_lo, tc::off_kmajor(lt, 8 * c, 128), cr);
                        store8<NPROD, F16>(a_hi, a_lo, tc::off_kmajor(lt, WY + 8 * c, 128), ci);
                    }
                }
            }
            if (!sync_issue(ok)) {
                failed = true;
                break;
            }
        }
        if (lt == 0) {
            issue_pass<KY, KY, false, false, NPROD, 0, F16>(tmem, sa_hi, sa_lo, sgy_hi, sgy_lo);
            tc::mma_commit(mb);
        }

        // ---- pass D operand: MN-major, m = (wl, y), k = (re|im, kx) ----
        {
            const bool ok = wait_pass();
            if (ok) {
                float tr[WY], ti[WY];
                tmem_cols<WY>(lane_addr, tr);
                tmem_cols<WY>(lane_addr + WY, ti);
                tc::tmem_wait_ld();
                if (rowB) {
#pragma unroll
                    for (int c = 0; c < WY / 8; ++c) {
                        store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wlB * WY + 8 * c, kx, KX), tr + 8 * c, sD);
                        store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wlB * WY + 8 * c, WX + kx, KX), ti + 8 * c, sD);
                    }
                }
            }
            if (!sync_issue(ok)) {
                failed = true;
                break;
            }
        }
        if (lt == 0) {
            // N: the real output's WX columns rounded up to the MMA's multiple of 16 (the extra
            // columns are the first rows of the imaginary block, computed and ignored)
            issue_pass<KX, (WX + 15) / 16 * 16, true, false, NPROD, 0, F16>(tmem, sa_hi, sa_lo, sgx_hi, sgx_lo);
            tc::mma_commit(mb);
        }

        // ---- correlation row (wl, y) -> |.|/N into the fftshifted plane ----
        {
            const bool ok = wait_pass();
            if (ok) {
                float cv[WX];
                tmem_cols<WX>(lane_addr, cv);
                tc::tmem_wait_ld();
                if (rowA) {
                    float *prow = planes + wlA * (WY * LDF) + ((y + WY / 2) % WY) * LDF;
#pragma unroll
                    for (int x = 0; x < WX; ++x)
                        prow[(x + WX / 2) % WX] = deadA ? 0.f : (fabsf(cv[x]) * unscale) * inv_n;
                }
            }
            tc::fence_before_sync();
            const bool bad = tc::named_sync_or(bar_id, 128, !ok);
            tc::fence_after_sync();
            if (bad) {
                failed = true;
                break;
            }
        }

        // ---- peaks: warp per window (two per window of more than 32 rows) ----
        if constexpr (WY > 32) {
            PeakPart(*parts)[2] = reinterpret_cast<PeakPart(*)[2]>(planes + 2 * WY * LDF);
            const int b = wq >> 1, part = wq & 1;
            const int wb = w0 + b;
            const float *P = planes + b * (WY * LDF);
            if (wb < a.w_end) peak_window_part<WX, WY, K>(a, P, part, lane, parts[b][part]);
            tc::named_sync(bar_id, 128);
            if (wb < a.w_end && part == 0) peak_window_merge<WX, WY>(a, P, wb, lane, parts[b]);
        } else if (wq < 2) {
            const int wb = w0 + wq;
            if (wb < a.w_end) peak_window<WX, WY, K>(a, planes + wq * (WY * LDF), wb, lane);
        }
        tc::named_sync(bar_id, 128);  // planes (aliasing the operand buffers) are consumed
    }

    if (failed) {
        if (lt == 0 && a.status) atomicOr(a.status, kStatusMmaWait);
        tc::mbar_wait(mb, (phase - 1) & 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid < 32) tc::tmem_dealloc(tmem_base, TALLOC);
}

// One CTA per SM (tensor memory), persistent over the tiles of 2 windows.
template <int WX, int WY, int NPROD, bool F16>
cudaError_t launch_tc_rect_shape(const XcorrArgs &a, bool deformed, int K, cudaStream_t s)
{
    using S = TcRectShape<WX, WY>;
    const int n = a.w_end - a.w_first;
    if (n <= 0) return cudaSuccess;
    const int tiles = (n + 1) / 2;
    cudaError_t e = cudaSuccess;
    auto go = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        if (e != cudaSuccess) return;
        int dev = 0, sms = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return;
        const int want = (tiles + S::NG - 1) / S::NG;
        const int grid = want < sms ? want : sms;
        kern<<<grid, S::THREADS, S::SMEM, s>>>(a);
        e = cudaGetLastError();
    };
    if (K <= 4) {
        if (deformed) go(xcorr_tc_rect_kernel<WX, WY, NPROD, 4, true, F16>);
        else go(xcorr_tc_rect_kernel<WX, WY, NPROD, 4, false, F16>);
    } else {
        if (deformed) go(xcorr_tc_rect_kernel<WX, WY, NPROD, 8, true, F16>);
        else go(xcorr_tc_rect_kernel<WX, WY, NPROD, 8, false, F16>);
    }
    return e;
}

}  // namespace piv
