// xcorr_kernel.cu -- the fused correlation + peak kernel (FP32 SIMT path).
//
// One launch replaces, for a section of windows, the reference's
//   organize_data_fft2d_multi(_deformed)  X/xcorr2d_multi_grid.cu:497, 654
//   cufftExecC2C FORWARD x2               :1334-1341, 1649-1656
//   multiply_conjugate                    :519
//   cufftExecC2C INVERSE                  :1347, 1662
//   complex2amp_xcorr2d                   :536
//   fftshift2d_xcorr2d_row/col            :547, 566
//   find_local_max_2d                     :585
//   reduce_max_index_general/final x4     :32, 103
//   replace_local_max_2d                  :298
//   peak_subpixel_4peak_2d                :309
//   kernel_remove_nan                     :457
// The correlation planes never leave shared memory.
//
// Per CTA: a batch of B windows (B even).  Data flow in shared memory:
//   P1  row task (window, row): gather frame-1 and frame-2 rows straight from HBM,
//       pack z = f1 + i*f2, row FFT in registers, store.
//   P2  column task: column FFT in registers -> Z = FFT2(f1) + i*FFT2(f2).
//   P3  column task (window pair, column; a lane pair per task for columns of 32 and
//       more when the CTA has the threads): the cross spectrum conj(F1)*F2 follows
//       from Z(k) and Z(-k) as  C = Im(Z(k)Z(-k))/2 + i(|Z(-k)|^2 - |Z(k)|^2)/4;
//       it is Hermitian, so two windows share one inverse transform:
//       W = C_a + i*C_b, inverse column FFT in registers.
//   P4  row task (pair, row; a lane pair per task likewise): inverse row FFT ->
//       Re = corr_a, Im = corr_b;
//       |.|/N written as fftshifted FP32 planes.
//   P5  warp per window (two warps for windows taller than 32 rows when the CTA has
//       them): 4-neighbour local maxima inside the search region,
//       count, register top-K (value desc, then lower index), 3-point Gaussian fit
//       with an accurate log-ratio denominator, predictor, limits, NaN/Inf removal.
#pragma once
#include <cfloat>
#include <climits>

#include "fft_reg.cuh"
#include "piv_common.cuh"

namespace piv {

// Byte b of w as a float: the byte is placed into the low mantissa bits of 2^23
// (0x4B0000bb), then 2^23 is subtracted -- exact for 0..255, one PRMT + one FADD.
template <int b>
__device__ __forceinline__ float byte_to_float(uint32_t w)
{
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | b)) - 8388608.0f;
}

template <int WSX>
__device__ __forceinline__ void load_u8_row(const uint8_t *p, float (&v)[WSX])
{
    uintptr_t ad = reinterpret_cast<uintptr_t>(p);
    if constexpr (WSX % 8 == 0) {
        if ((ad & 7) == 0) {
#pragma unroll
            for (int q = 0; q < WSX / 8; ++q) {
                uint2 u = __ldg(reinterpret_cast<const uint2 *>(p) + q);
                v[8 * q + 0] = byte_to_float<0>(u.x);
                v[8 * q + 1] = byte_to_float<1>(u.x);
                v[8 * q + 2] = byte_to_float<2>(u.x);
                v[8 * q + 3] = byte_to_float<3>(u.x);
                v[8 * q + 4] = byte_to_float<0>(u.y);
                v[8 * q + 5] = byte_to_float<1>(u.y);
                v[8 * q + 6] = byte_to_float<2>(u.y);
                v[8 * q + 7] = byte_to_float<3>(u.y);
            }
            return;
        }
    }
    if ((ad & 3) == 0) {
#pragma unroll
        for (int q = 0; q < WSX / 4; ++q) {
            uint32_t u = __ldg(reinterpret_cast<const uint32_t *>(p) + q);
            v[4 * q + 0] = byte_to_float<0>(u);
            v[4 * q + 1] = byte_to_float<1>(u);
            v[4 * q + 2] = byte_to_float<2>(u);
            v[4 * q + 3] = byte_to_float<3>(u);
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < WSX; ++i) v[i] = (float)__ldg(p + i);
}

template <int WSX>
__device__ __forceinline__ void load_f32_row(const float *p, float (&v)[WSX])
{
    if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
        for (int q = 0; q < WSX / 4; ++q) {
            float4 u = __ldg(reinterpret_cast<const float4 *>(p) + q);
            v[4 * q] = u.x;
            v[4 * q + 1] = u.y;
            v[4 * q + 2] = u.z;
            v[4 * q + 3] = u.w;
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < WSX; ++i) v[i] = __ldg(p + i);
}

// total order used for the top-K: larger value first, then the lower index
__device__ __forceinline__ bool better(float v1, int i1, float v2, int i2)
{
    return v1 > v2 || (v1 == v2 && i1 < i2);
}

template <int K>
__device__ __forceinline__ void topk_insert(float (&tv)[K], int (&ti)[K], float v, int i)
{
    if (!better(v, i, tv[K - 1], ti[K - 1])) return;
#pragma unroll
    for (int s = K - 1; s >= 1; --s) {
        bool up = better(v, i, tv[s - 1], ti[s - 1]);  // v goes above slot s-1
        bool here = !up && better(v, i, tv[s], ti[s]);
        float nv = up ? tv[s - 1] : (here ? v : tv[s]);
        int ni = up ? ti[s - 1] : (here ? i : ti[s]);
        tv[s] = nv;
        ti[s] = ni;
    }
    if (better(v, i, tv[0], ti[0])) {
        tv[0] = v;
        ti[0] = i;
    }
}

// ------------------------------------------------------------------------------
// Peak stage of one window: 4-neighbour local maxima inside the search region, count,
// top-Npeak_save, 3-point Gaussian fit, predictor, limits, NaN/Inf removal
// (find_local_max_2d, reduce_max_index_*, replace_local_max_2d, peak_subpixel_4peak_2d,
// kernel_remove_nan).  P: the window's fftshifted plane in shared memory with row
// stride WSX + 1.  One warp per window (peak_window), or, for windows of more than 32
// rows, two warps that each scan half of the rows and merge their top-N through shared
// memory (peak_window_part, then peak_window_merge after a barrier).
// ------------------------------------------------------------------------------

// Region rows first, first + step, ... scanned by this lane into its sorted top-K
// (value desc, index asc); returns the lane's count of maxima.
template <int WSX, int WSY, int K>
__device__ __forceinline__ int peak_scan(const GridGeom &g, const float *P, int first, int step, float (&tv)[K],
                                         int (&ti)[K])
{
    constexpr int LDF = WSX + 1;
    const int rows = WSY - 2 * g.by;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        tv[k] = -1.f;
        ti[k] = INT_MAX;
    }
    // columns allowed by the border (and by the 4-neighbour stencil) as a bitmask
    constexpr int NWRD = (WSX + 31) / 32;
    const int lo = g.bx > 1 ? g.bx : 1, hi = (WSX - 1 - g.bx) < (WSX - 2) ? (WSX - 1 - g.bx) : (WSX - 2);
    uint32_t allow[NWRD];
#pragma unroll
    for (int q = 0; q < NWRD; ++q) {
        // bits [lo, hi] of word q
        const int l = lo - 32 * q, h = hi - 32 * q;
        const uint32_t upto = h >= 31 ? 0xffffffffu : (h < 0 ? 0u : ((2u << h) - 1u));
        const uint32_t from = l <= 0 ? 0xffffffffu : (l > 31 ? 0u : ~((1u << l) - 1u));
        allow[q] = upto & from;
    }
    // v > 0 and v >= all four neighbours  <=>  v >= max(neighbours, smallest subnormal)
    const float tiny = __int_as_float(1);
    int cnt = 0;
    for (int jj = first; jj < rows; jj += step) {
        const int j = g.by + jj;
        const float *pm = P + j * LDF;
        float mid[WSX];
#pragma unroll
        for (int i = 0; i < WSX; ++i) mid[i] = pm[i];
        // local-maximum test of every column without branches, as a bitmask
        uint32_t mk[NWRD];
#pragma unroll
        for (int q = 0; q < NWRD; ++q) mk[q] = 0;
#pragma unroll
        for (int i = 1; i < WSX - 1; ++i) {
            const float m = fmaxf(fmaxf(mid[i - 1], mid[i + 1]), fmaxf(fmaxf(pm[i - LDF], pm[i + LDF]), tiny));
            mk[i >> 5] |= (uint32_t)(mid[i] >= m) << (i & 31);
        }
        // the row's maxima in column order into the lane's top-K
#pragma unroll
        for (int q = 0; q < NWRD; ++q) {
            uint32_t m = mk[q] & allow[q];
            cnt += __popc(m);
            while (m) {
                const int i = 32 * q + __ffs(m) - 1;
                m &= m - 1;
                topk_insert<K>(tv, ti, pm[i], j * WSX + i);
            }
        }
    }
    return cnt;
}

// Nps rounds of a warp arg-max over the lanes' list heads; lane k < Nps receives the
// k-th best (value, index), -1 / INT_MAX when there are fewer candidates.  Candidates
// are positive, so their bit patterns order as unsigned integers: the largest value
// is one warp max-reduction, the lowest index holding it one min-reduction (the order
// of better()).  Indices are unique, so exactly one lane owns each winner and pops it.
template <int K>
__device__ __forceinline__ void peak_select(int Nps, int lane, float (&tv)[K], int (&ti)[K], float &v, int &idx)
{
    v = -1.f;
    idx = INT_MAX;
    for (int k = 0; k < Nps; ++k) {
        const uint32_t key = tv[0] > 0.f ? __float_as_uint(tv[0]) : 0u;
        const uint32_t kmax = __reduce_max_sync(0xffffffffu, key);
        const uint32_t imin = __reduce_min_sync(0xffffffffu, key == kmax ? (uint32_t)ti[0] : 0xffffffffu);
        const float bv = kmax ? __uint_as_float(kmax) : -1.f;
        const int bi = kmax ? (int)imin : INT_MAX;
        if (lane == k) {
            v = bv;
            idx = bi;
        }
        if (bi == ti[0] && bv > 0.f) {
#pragma unroll
            for (int s = 0; s < K - 1; ++s) {
                tv[s] = tv[s + 1];
                ti[s] = ti[s + 1];
            }
            tv[K - 1] = -1.f;
            ti[K - 1] = INT_MAX;
        }
    }
}

// ln(fm fp / c^2), the Gaussian fit's denominator, which cancels near flat peaks (the
// reference's ln fm + ln fp - 2 ln c in FP32 loses most of its bits there).  fm fp - c^2 is
// formed exactly, up to one rounding, from the two products and their FMA residuals, divided
// by c^2 and passed to log1pf: about 2 ulp of the true value, as FP64 would give after the
// final rounding to FP32, without FP64 arithmetic.  Products below 2^-100, where they would
// lose bits to underflow, take the FP64 form.
__device__ __forceinline__ float fit_denominator(float fm, float fp, float c)
{
    const float p = fm * fp, q = c * c;
    if (!(p >= 7.8886091e-31f && q >= 7.8886091e-31f))  // 2^-100; also zeros and NaN
        return (float)log(((double)fm * (double)fp) / ((double)c * (double)c));
    const float ep = fmaf(fm, fp, -p), eq = fmaf(c, c, -q);
    return log1pf(((p - q) + (ep - eq)) / q);
}

// Sub-pixel fit of the candidates held by lanes < Nps, limits, NaN/Inf removal and the
// stores of the window's outputs; cnt is the window's count of maxima.  Called by whole
// warps (the fits' x and y halves run on separate lanes and meet by shuffle).
template <int WSX, int WSY>
__device__ __forceinline__ void peak_fit_store(const XcorrArgs &a, const float *P, int w, int lane, float v, int idx,
                                               int cnt, float pred_x, float pred_y)
{
    constexpr int LDF = WSX + 1;
    const GridGeom &g = a.g;
    const int Nps = g.Nps;
    // lanes [0, Nps) fit x and lanes [Nps, 2 Nps) fit y of the same candidates (the fits are
    // independent, so each lane does one instead of two: the warp issues the FP64 path once)
    const int comp = lane < Nps ? 0 : (lane < 2 * Nps ? 1 : 2);
    const int k = comp == 1 ? lane - Nps : lane;
    const float cv = __shfl_sync(0xffffffffu, v, k & 31);
    const int cidx = __shfl_sync(0xffffffffu, idx, k & 31);
    float sh = 0.f;
    bool inner = false;
    if (comp < 2 && cv > 0.f) {
        const int j = cidx / WSX, i = cidx - j * WSX;
        if (i != 0 && i != WSX - 1 && j != 0 && j != WSY - 1) {
            const float *pc = P + j * LDF + i;
            const int step = comp ? LDF : 1;
            const float f0 = pc[-step], f2 = pc[step];
            // numerator ln f- - ln f+ in FP32 as the reference; the cancelling denominator
            // ln(f- f+ / f0^2) accurately (fit_denominator)
            const float nn = logf(f0) - logf(f2);
            sh = nn / fit_denominator(f0, f2, cv) * 0.5f;
            inner = true;
        }
    }
    const float sy = __shfl_sync(0xffffffffu, sh, (lane + Nps) & 31);
    if (lane < Nps) {
        float ox = 0.f, oy = 0.f;
        bool ok = false;
        if (inner) {
            const int j = idx / WSX, i = idx - j * WSX;
            ox = (float)i + sh - (float)WSX / 2 + pred_x;
            oy = (float)j + sy - (float)WSY / 2 + pred_y;
            ok = true;
            if (ox < g.lx1 || ox > g.lx2 || oy < g.ly1 || oy > g.ly2) {
                ok = false;
                ox = 0.f;
                oy = 0.f;
            }
            if (isnan(ox) || isnan(oy) || isinf(ox) || isinf(oy)) {
                ok = false;
                ox = 0.f;
                oy = 0.f;
            }
        }
        const size_t o = (size_t)w * Nps + lane;
        a.cdx[o] = ox;
        a.cdy[o] = oy;
        a.cvalid[o] = ok ? 1 : 0;
        a.pidx[o] = (v > 0.f) ? idx : -1;
        a.pval[o] = (v > 0.f) ? v : 0.f;
    }
    if (lane == 0) a.count[w] = cnt;
}

// diagnostic mode: the plane only, the pass outputs stay untouched
template <int WSX, int WSY>
__device__ __forceinline__ void peak_dump(const XcorrArgs &a, const float *P, int w, int lane)
{
    constexpr int LDF = WSX + 1;
    float *dst = a.cc_dump + (size_t)(w - a.w_first) * (WSX * WSY);
    for (int t = lane; t < WSX * WSY; t += 32) {
        const int j = t / WSX, i = t - j * WSX;
        dst[t] = P[j * LDF + i];
    }
}

__device__ __forceinline__ int warp_sum(int x)
{
    return __reduce_add_sync(0xffffffffu, x);
}

// One warp per window.
template <int WSX, int WSY, int K>
__device__ __forceinline__ void peak_window(const XcorrArgs &a, const float *P, int w, int lane)
{
    if (a.cc_dump) {
        peak_dump<WSX, WSY>(a, P, w, lane);
        return;
    }
    // the predictor of the window, fetched early (used by the Nps fitting lanes)
    float pred_x = 0.f, pred_y = 0.f;
    if (lane < a.g.Nps) {
        pred_x = a.pred_x[w];
        pred_y = a.pred_y[w];
    }
    float tv[K];
    int ti[K];
    const int cnt = warp_sum(peak_scan<WSX, WSY, K>(a.g, P, lane, 32, tv, ti));
    float v;
    int idx;
    peak_select<K>(a.g.Nps, lane, tv, ti, v, idx);
    peak_fit_store<WSX, WSY>(a, P, w, lane, v, idx, cnt, pred_x, pred_y);
}

// Two warps per window: one warp's half of the rows and its top-Nps.
struct PeakPart {
    float v[8];
    int idx[8];
    int cnt;
};

template <int WSX, int WSY, int K>
__device__ __forceinline__ void peak_window_part(const XcorrArgs &a, const float *P, int part, int lane,
                                                 PeakPart &out)
{
    if (a.cc_dump) return;
    float tv[K];
    int ti[K];
    const int cnt = warp_sum(peak_scan<WSX, WSY, K>(a.g, P, 32 * part + lane, 64, tv, ti));
    float v;
    int idx;
    peak_select<K>(a.g.Nps, lane, tv, ti, v, idx);
    if (lane < a.g.Nps) {
        out.v[lane] = v;
        out.idx[lane] = idx;
    }
    if (lane == 0) out.cnt = cnt;
}

// After a barrier, one warp merges the two halves' top-Nps (one entry per lane) and fits.
template <int WSX, int WSY>
__device__ __forceinline__ void peak_window_merge(const XcorrArgs &a, const float *P, int w, int lane,
                                                  const PeakPart (&parts)[2])
{
    if (a.cc_dump) {
        peak_dump<WSX, WSY>(a, P, w, lane);
        return;
    }
    const int Nps = a.g.Nps;
    float pred_x = 0.f, pred_y = 0.f;
    if (lane < Nps) {
        pred_x = a.pred_x[w];
        pred_y = a.pred_y[w];
    }
    float tv[1] = {-1.f};
    int ti[1] = {INT_MAX};
    if (lane < 2 * Nps) {
        const PeakPart &pp = parts[lane >= Nps];
        const int k = lane >= Nps ? lane - Nps : lane;
        tv[0] = pp.v[k];
        ti[0] = pp.idx[k];
    }
    float v;
    int idx;
    peak_select<1>(Nps, lane, tv, ti, v, idx);
    peak_fit_store<WSX, WSY>(a, P, w, lane, v, idx, parts[0].cnt + parts[1].cnt, pred_x, pred_y);
}

// Residency asked of the register allocation (the second __launch_bounds__ argument).
// 32x32 windows, 4 per CTA of 128 threads: 33.8 KB of shared memory lets 6 CTAs share an
// SM, and at 80 registers (checked spill-free) so do the registers, against 5 CTAs at the
// unconstrained 84.  Elsewhere the compiler's own choice (a blanket bound makes the small
// variants spill).
template <int WSX, int WSY, int B, int NT>
constexpr int xcorr_min_ctas()
{
    return (WSX == 32 && WSY == 32 && B == 4 && NT == 128) ? 6 : 1;
}


template <int WSX, int WSY, int B, int NT, int K, bool DEF>
__global__ void __launch_bounds__(NT, (xcorr_min_ctas<WSX, WSY, B, NT>())) xcorr_peak_kernel(const XcorrArgs a)
{
    constexpr int VB = 1;
    const unsigned blk = blockIdx.x;
#include "xcorr_body.inc"
}

// 2x2-block form: a CTA takes two horizontally adjacent window pairs in two consecutive window
// rows, whose overlapping pixel rows are gathered and row-transformed once (at 50 % overlap 3/4
// of the row transforms of the row-major form).  Same arithmetic per window, so the same bits.
template <int WSX, int WSY, int NT, int K, bool DEF>
__global__ void __launch_bounds__(NT, (xcorr_min_ctas<WSX, WSY, 4, NT>())) xcorr_block_kernel(const XcorrArgs a)
{
    constexpr int B = 4, VB = 2;
    const unsigned blk = blockIdx.x;
#include "xcorr_body.inc"
}

// Batch form: the CTA-sized window batches ("items") of many pairs with the same window
// shape in one launch, one CTA per item.  Pair i owns items [first[i], first[i+1]); a
// CTA finds its pair by bisection and reads the pair's arguments from the parameter
// (constant bank; read from global memory instead, the kernel ran 2.8 % slower).
// (A persistent grid whose CTAs loop over items was measured against this: the loop made
// the compiler hold loop-invariant state through every phase, 62 -> 106 registers at
// 16x16 and 152 -> 216 at 64x64, and lose occupancy; the hardware scheduler balances
// one-item CTAs as well.)
template <int WSX, int WSY, int B, int NT, int K, bool DEF>
__global__ void __launch_bounds__(NT, (xcorr_min_ctas<WSX, WSY, B, NT>())) xcorr_batch_kernel(const __grid_constant__ XcorrBatch b)
{
    const int it = blockIdx.x;
    int lo = 0, hi = b.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (b.first[mid] <= it) lo = mid;
        else hi = mid - 1;
    }
    const XcorrArgs &a = b.pairs[lo];
    const unsigned blk = it - b.first[lo];
    constexpr int VB = 1;
#include "xcorr_body.inc"
}

// ------------------------------------------------------------------------------
// Launch of one instantiated shape (explicitly instantiated in xcorr_shape_*.cu).
// ------------------------------------------------------------------------------
template <int WSX, int WSY, int B, int NT>
cudaError_t launch_shape(const XcorrArgs &a, bool deformed, int K, cudaStream_t s)
{
    if (a.w_end <= a.w_first) return cudaSuccess;
    const int n = a.w_end - (a.w_first & ~1);  // CTAs start at an even window (pairing)
    const size_t smem = (size_t)B * WSY * (WSX + 1) * sizeof(float2);
    dim3 grid((n + B - 1) / B);
    cudaError_t e = cudaSuccess;
    auto go = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return;
        kern<<<grid, NT, smem, s>>>(a);
        e = cudaGetLastError();
    };
    if (K <= 4) {
        if (deformed) go(xcorr_peak_kernel<WSX, WSY, B, NT, 4, true>);
        else go(xcorr_peak_kernel<WSX, WSY, B, NT, 4, false>);
    } else {
        if (deformed) go(xcorr_peak_kernel<WSX, WSY, B, NT, 8, true>);
        else go(xcorr_peak_kernel<WSX, WSY, B, NT, 8, false>);
    }
    return e;
}

// Launch of the 2x2-block form (four windows per CTA): the blocks of the launch's window rows
// (rounded out to whole block rows; windows outside [w_first, w_end) are computed, not
// written).  An odd row of windows has no whole pairs of columns: the row-major form then.
template <int WSX, int WSY, int NT>
cudaError_t launch_shape_block(const XcorrArgs &a, bool deformed, int K, cudaStream_t s)
{
    if (a.w_end <= a.w_first) return cudaSuccess;
    const int nx = a.g.Nx_vec;
    if (nx % 2) return launch_shape<WSX, WSY, 4, NT>(a, deformed, K, s);
    const int by0 = (a.w_first / nx) >> 1, by1 = ((a.w_end - 1) / nx) >> 1;
    const size_t smem = (size_t)4 * WSY * (WSX + 1) * sizeof(float2);
    dim3 grid((unsigned)((nx >> 1) * (by1 - by0 + 1)));
    cudaError_t e = cudaSuccess;
    auto go = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return;
        kern<<<grid, NT, smem, s>>>(a);
        e = cudaGetLastError();
    };
    if (K <= 4) {
        if (deformed) go(xcorr_block_kernel<WSX, WSY, NT, 4, true>);
        else go(xcorr_block_kernel<WSX, WSY, NT, 4, false>);
    } else {
        if (deformed) go(xcorr_block_kernel<WSX, WSY, NT, 8, true>);
        else go(xcorr_block_kernel<WSX, WSY, NT, 8, false>);
    }
    return e;
}

// Launch of a batch: items = sum over pairs of ceil(windows / B), first[] their prefix
// sums; one CTA per item.
template <int WSX, int WSY, int B, int NT>
cudaError_t launch_shape_batch(const XcorrBatch &b, bool deformed, int K, cudaStream_t s)
{
    if (b.items <= 0) return cudaSuccess;
    const size_t smem = (size_t)B * WSY * (WSX + 1) * sizeof(float2);
    cudaError_t e = cudaSuccess;
    auto go = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return;
        kern<<<b.items, NT, smem, s>>>(b);
        e = cudaGetLastError();
    };
    if (K <= 4) {
        if (deformed) go(xcorr_batch_kernel<WSX, WSY, B, NT, 4, true>);
        else go(xcorr_batch_kernel<WSX, WSY, B, NT, 4, false>);
    } else {
        if (deformed) go(xcorr_batch_kernel<WSX, WSY, B, NT, 8, true>);
        else go(xcorr_batch_kernel<WSX, WSY, B, NT, 8, false>);
    }
    return e;
}

}  // namespace piv
