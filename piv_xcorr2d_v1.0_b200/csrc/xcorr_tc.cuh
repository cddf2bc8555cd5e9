// xcorr_tc.cuh -- the fused correlation + peak kernel on the tcgen05 tensor cores.
//
// Same contract as xcorr_peak_kernel (the reference's organize_data_fft2d_multi(_deformed),
// cufftExecC2C x3, multiply_conjugate, complex2amp_xcorr2d, fftshift2d_xcorr2d_row/col,
// find_local_max_2d .. kernel_remove_nan; X/xcorr2d_multi_grid.cu:497-654, 1334-1347,
// 1649-1662), with the four 1-D transform passes of the WS x WS windows done as dense
// DFT products on the tensor cores instead of register FFTs.
//
// A tile is 128 rows = 128/WS windows, owned by one warpgroup (thread t of the
// warpgroup <-> TMEM lane t).  A CTA holds NG warpgroups working on independent tiles
// with their own operand buffers, TMEM columns, completion barrier and named barrier, so
// that one warpgroup's transposes overlap another's MMAs (a tcgen05 kernel is resident
// once per SM; the warpgroups supply the overlap co-resident CTAs would).  Every pass is one
// 128 x N x 2WS product with the complex values as (re | im) halves of K and N and the
// real DFT matrix  G = [[C, -S], [S, C]]  (C = cos, S = sin of 2*pi*n*k/WS):
//   A  rows (window, y)    x [f1 row | f2 row]    * G    -> row spectra of z = f1 + i f2
//   B  rows (window, kx)   x [re | im] over y     * G    -> Z = FFT2(f1) + i FFT2(f2), column kx
//      cross spectrum conj(F1) F2 = Im(Z(k)Z(-k))/2 + i(|Z(-k)|^2 - |Z(k)|^2)/4, the
//      partner column -kx by warp shuffle (for 64-wide windows the rows of pass B are
//      permuted so that columns kx and -kx always share a warp)
//   C  rows (window, kx)   x [re | im] over ky    * G^T  -> inverse column transforms
//   D  rows (window, y)    x [re | im] over kx    * G^T[:, :WS] -> real correlation row
// G lives once per CTA in shared memory; its K-major view is G^T, its MN-major view G
// (layouts in tc_common.cuh).  Operands are BF16 (F16 = false) or FP16 (F16 = true);
// NPROD = 3 splits every value into hi + lo and accumulates hi*hi + hi*lo + lo*hi in FP32
// (about 16 significant bits per operand in BF16, 22 in FP16), NPROD = 1 uses the rounded
// values only (precision study).  FP16 has a 5-bit exponent, so the operands of passes B,
// C and D are scaled by exact powers of two that keep every value of any 8-bit window pair
// below 65504: pass B's by 1/WS, the cross spectrum by 1/(2 WS^2), pass D's by 1/(2 WS);
// one multiply by a power of two at the end undoes them (the same scaling runs on the
// BF16 path, whose rounding it leaves unchanged).  |corr|/N goes to fftshifted FP32
// planes in shared memory and the peak stage is the SIMT kernel's.
//
// Waits on the MMA completion barrier are bounded: on a timeout the warpgroup stops,
// sets bit kStatusMmaWait in *a.status, and the CTA releases its tensor memory.
#pragma once
#include <cuda.h>

#include <cstring>

#include "tc_common.cuh"
#include "xcorr_kernel.cuh"

namespace piv {

template <int WS>
struct TwTable {
    float c[WS], s[WS];
};
template <int WS>
constexpr TwTable<WS> make_tw()
{
    TwTable<WS> t{};
    for (int i = 0; i < WS; ++i) {
        const CosSin cs = cossin_2pi(i, WS);
        t.c[i] = (float)cs.c;
        t.s[i] = (float)cs.s;
    }
    return t;
}
template <int WS>
__constant__ TwTable<WS> kTw = make_tw<WS>();

// 8 floats -> bf16 / fp16 hi (and lo) as 16 bytes each
template <bool F16>
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    if constexpr (F16) tc::split_f16x2(a, b, hi, lo);
    else tc::split_bf16x2(a, b, hi, lo);
}

template <bool F16>
__device__ __forceinline__ void split8(const float *v, uint4 &hi, uint4 &lo)
{
    split2<F16>(v[0], v[1], hi.x, lo.x);
    split2<F16>(v[2], v[3], hi.y, lo.y);
    split2<F16>(v[4], v[5], hi.z, lo.z);
    split2<F16>(v[6], v[7], hi.w, lo.w);
}

template <int NPROD, bool F16>
__device__ __forceinline__ void store8(uint8_t *hi, uint8_t *lo, uint32_t off, const float *v)
{
    uint4 h, l;
    split8<F16>(v, h, l);
    *reinterpret_cast<uint4 *>(hi + off) = h;
    if constexpr (NPROD > 1) *reinterpret_cast<uint4 *>(lo + off) = l;
}

// the 8 values scaled by a power of two (SCALE), then stored as above
template <int NPROD, bool F16, bool SCALE>
__device__ __forceinline__ void store8s(uint8_t *hi, uint8_t *lo, uint32_t off, const float *v, float scale)
{
    if constexpr (SCALE) {
        float w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) w[i] = v[i] * scale;
        store8<NPROD, F16>(hi, lo, off, w);
    } else {
        store8<NPROD, F16>(hi, lo, off, v);
    }
}

// 8 values exact in the operand type (integers up to 256): the hi part only, the lo part
// being zero (the MMAs never read it for these K columns)
template <bool F16>
__device__ __forceinline__ void store8_exact(uint8_t *hi, uint32_t off, const float *v)
{
    uint4 h;
    if constexpr (F16) {
        const __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
        const __half2 c = __floats2half2_rn(v[4], v[5]), d = __floats2half2_rn(v[6], v[7]);
        h = make_uint4(*reinterpret_cast<const uint32_t *>(&a), *reinterpret_cast<const uint32_t *>(&b),
                       *reinterpret_cast<const uint32_t *>(&c), *reinterpret_cast<const uint32_t *>(&d));
    } else {
        const __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
        const __nv_bfloat162 c = __floats2bfloat162_rn(v[4], v[5]), d = __floats2bfloat162_rn(v[6], v[7]);
        h = make_uint4(*reinterpret_cast<const uint32_t *>(&a), *reinterpret_cast<const uint32_t *>(&b),
                       *reinterpret_cast<const uint32_t *>(&c), *reinterpret_cast<const uint32_t *>(&d));
    }
    *reinterpret_cast<uint4 *>(hi + off) = h;
}

// whether any of the W values is nonzero (by their bits, sign masked): a 3-input OR tree
template <int W>
__device__ __forceinline__ bool any_nonzero(const float (&v)[W])
{
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) acc |= __float_as_uint(v[i]);
    return (acc & 0x7fffffffu) != 0u;
}

// A staged row of W bytes at any byte offset in shared memory: the aligned words covering
// it, each output word assembled by a funnel shift (reads up to 3 bytes past the row, inside
// the staging region), bytes converted as in load_u8_row.
template <int W>
__device__ __forceinline__ void load_u8_row_shared(const uint8_t *p, float (&v)[W])
{
    static_assert(W % 4 == 0, "rows of whole words");
    const uintptr_t ad = reinterpret_cast<uintptr_t>(p);
    const uint32_t *q = reinterpret_cast<const uint32_t *>(ad & ~(uintptr_t)3);
    const uint32_t sh = (uint32_t)(ad & 3) * 8;
    uint32_t w[W / 4 + 1];
#pragma unroll
    for (int i = 0; i <= W / 4; ++i) w[i] = q[i];
#pragma unroll
    for (int c = 0; c < W / 4; ++c) {
        const uint32_t u = __funnelshift_r(w[c], w[c + 1], sh);
        v[4 * c + 0] = byte_to_float<0>(u);
        v[4 * c + 1] = byte_to_float<1>(u);
        v[4 * c + 2] = byte_to_float<2>(u);
        v[4 * c + 3] = byte_to_float<3>(u);
    }
}

template <int W>
__device__ __forceinline__ void load_f32_row_shared(const float *p, float (&v)[W])
{
    if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
#pragma unroll
        for (int q = 0; q < W / 4; ++q) {
            const float4 u = reinterpret_cast<const float4 *>(p)[q];
            v[4 * q] = u.x;
            v[4 * q + 1] = u.y;
            v[4 * q + 2] = u.z;
            v[4 * q + 3] = u.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < W; ++i) v[i] = p[i];
    }
}

// One pass: D[128 x N] = A[128 x KK] * B^T over KK/16 K steps.  A in the K-major
// (A_MN = false) or MN-major layout; B is the G buffer read MN-major (G) or K-major
// (G^T).  The lo*hi product runs from K step LO_FROM on (A's lo part is zero before).
template <int KK, int N, bool A_MN, bool B_MN, int NPROD, int LO_FROM, bool F16>
__device__ __forceinline__ void issue_pass(uint32_t tmem, uint32_t a_hi, uint32_t a_lo, uint32_t g_hi,
                                           uint32_t g_lo)
{
    constexpr uint32_t idesc = tc::idesc_f16(N, A_MN, B_MN, !F16);
    constexpr uint32_t a_lbo = A_MN ? 128u : 128u * 16u, a_sbo = A_MN ? KK * 16u : 128u;
    constexpr uint32_t a_step = A_MN ? 256u : 2u * a_lbo;
    constexpr uint32_t b_lbo = B_MN ? 128u : KK * 16u, b_sbo = B_MN ? KK * 16u : 128u;
    constexpr uint32_t b_step = B_MN ? 256u : 2u * b_lbo;
#pragma unroll
    for (int s = 0; s < KK / 16; ++s) {
        const uint64_t ah = tc::smem_desc(a_hi + s * a_step, a_lbo, a_sbo);
        const uint64_t gh = tc::smem_desc(g_hi + s * b_step, b_lbo, b_sbo);
        tc::mma_f16(tmem, ah, gh, idesc, s > 0 ? 1u : 0u);
        if constexpr (NPROD > 1) {
            tc::mma_f16(tmem, ah, tc::smem_desc(g_lo + s * b_step, b_lbo, b_sbo), idesc, 1u);
            if (s >= LO_FROM) tc::mma_f16(tmem, tc::smem_desc(a_lo + s * a_step, a_lbo, a_sbo), gh, idesc, 1u);
        }
    }
}

// Loads WS consecutive TMEM columns of this warp's lanes.
template <int WS>
__device__ __forceinline__ void tmem_row(uint32_t taddr, float (&v)[WS])
{
    if constexpr (WS == 16) {
        tc::tmem_ld16(taddr, v);
    } else {
        static_assert(WS % 32 == 0, "16 or a multiple of 32 columns");
#pragma unroll
        for (int c = 0; c < WS / 32; ++c) {
            float t[32];
            tc::tmem_ld32(taddr + 32 * c, t);
#pragma unroll
            for (int i = 0; i < 32; ++i) v[32 * c + i] = t[i];
        }
    }
}

// Row order of pass B within a window: position p holds column kx = col_at<WS>(p).
// Identity up to 32 columns (a window's columns share a warp).  For 64 columns the
// first warp takes {0..15, 32, 49..63} and the second {16..31, 33..48}: both sets are
// closed under kx -> -kx mod 64, so the partner column is a shuffle away.
template <int WS>
__host__ __device__ constexpr int col_at(int p)
{
    if constexpr (WS <= 32) {
        return p;
    } else {
        return p <= 15 ? p : p == 16 ? 32 : p <= 31 ? p + 32 : p <= 47 ? p - 16 : p - 15;
    }
}
template <int WS>
__host__ __device__ constexpr int pos_of(int kx)
{
    if constexpr (WS <= 32) {
        return kx;
    } else {
        return kx <= 15 ? kx : kx == 32 ? 16 : kx >= 49 ? kx - 32 : kx <= 31 ? kx + 16 : kx + 15;
    }
}

// Whether window wl of a tile has an all-zero frame 1 or frame 2, from the pass-A row
// ballots of the warpgroup's 4 warps (window wl owns rows [wl*WS, wl*WS + WS)).
template <int WS>
__device__ __forceinline__ bool window_dead(const uint32_t (&nz1)[4], const uint32_t (&nz2)[4], int wl)
{
    uint32_t a = 0, b = 0;
    if constexpr (WS <= 32) {
        const int warp = (wl * WS) >> 5, sh = (wl * WS) & 31;
        const uint32_t m = WS == 32 ? 0xffffffffu : (((1u << WS) - 1u) << sh);
        a = nz1[warp] & m;
        b = nz2[warp] & m;
    } else {
        const int w0 = (wl * WS) >> 5;
#pragma unroll
        for (int q = 0; q < WS / 32; ++q) {
            a |= nz1[w0 + q];
            b |= nz2[w0 + q];
        }
    }
    return a == 0u || b == 0u;
}

template <int WS>
struct TcShape {
    static constexpr int KK = 2 * WS;                          // K (and N) extent: re | im
    static constexpr int NG = WS == 64 ? 2 : 4;                 // warpgroups per CTA
    static constexpr int THREADS = 128 * NG;
    static constexpr uint32_t G_BYTES = KK * KK * 2;            // one of G hi / lo
    static constexpr uint32_t A_BYTES = 128 * KK * 2;           // one of A hi / lo
    static constexpr int TCOLS = KK < 32 ? 32 : KK;             // TMEM columns per warpgroup
    static constexpr size_t BASE = 2 * (size_t)G_BYTES + (size_t)NG * 2 * A_BYTES;
    // TMA staging of a tile's rows per warpgroup (16 and 32 px windows; 64 px windows have no
    // shared memory left and load their rows directly): frame-1 box of up to kStageBx bytes per
    // row, frame-2 box of up to kStageBx floats per row
    static constexpr int STAGE_BX = WS <= 32 ? 128 : 0;
    static constexpr uint32_t STAGE1 = WS * STAGE_BX, STAGE2 = WS * STAGE_BX * 4;
    static constexpr size_t SMEM = BASE + (size_t)NG * (STAGE1 + STAGE2);
    static_assert(SMEM <= 232448, "shared memory");
};


template <int WS, int NPROD, int K, bool DEF, bool F16>
__global__ void __launch_bounds__(TcShape<WS>::THREADS, 1) xcorr_tc_kernel(const XcorrArgs a,
                                                                           const __grid_constant__ TcStaging st)
{
    using S = TcShape<WS>;
    constexpr int KK = S::KK, NG = S::NG;
    constexpr int NWIN = 128 / WS;  // windows per tile
    constexpr int LDF = WS + 1;     // plane row stride (peak stage)
    constexpr uint32_t G_BYTES = S::G_BYTES, A_BYTES = S::A_BYTES;
    constexpr uint32_t TCOLS = S::TCOLS, TALLOC = S::TCOLS * S::NG;
    // operand scales (powers of two, exact): FP16 operands take pass B's by 1/WS, the cross
    // spectrum's by 1/(2 WS^2) and pass D's by 1/(2 WS), which keep every value of any 8-bit
    // window pair below 65504; BF16 has FP32's exponent range and keeps only the cross
    // spectrum's, folded into its constant factors.  The plane is |out| / (sB^2 sC sD N), one
    // exact multiply (4 WS^3 with FP16 operands, 2 with BF16).
    constexpr float sB = F16 ? 1.0f / (float)WS : 1.0f, sC = 1.0f / (float)(2 * WS * WS);
    constexpr float sD = F16 ? 1.0f / (float)(2 * WS) : 1.0f;
    constexpr float out_scale = 1.0f / (sB * sB * sC * sD * (float)(WS * WS));
    static_assert(TALLOC == 32 || TALLOC == 64 || TALLOC == 128 || TALLOC == 256 || TALLOC == 512, "TMEM alloc");
    static_assert((size_t)NWIN * WS * LDF * 4 <= 2 * A_BYTES, "planes fit in the A buffers");

    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar[NG];
    __shared__ __align__(8) uint64_t mbar_tma[NG];
    __shared__ uint32_t tmem_base;
    // per warp of each warpgroup: ballots of its pass-A rows holding a nonzero frame-1 /
    // frame-2 pixel (a window with either frame all zero correlates to exactly 0 in the
    // reference; its cross spectrum and plane are set to 0 here)
    __shared__ uint32_t s_nz1[NG][4], s_nz2[NG][4];

    const GridGeom &g = a.g;
    const int tid = threadIdx.x, wg = tid >> 7, lt = tid & 127;
    const int lane = tid & 31, wq = lt >> 5;  // warp within the warpgroup = TMEM lane quarter
    const int wl = lt / WS, r = lt % WS;      // window in tile; row (pass A) / row position (B)
    uint8_t *g_hi = smem, *g_lo = smem + G_BYTES;
    uint8_t *a_hi = smem + 2 * G_BYTES + (size_t)wg * 2 * A_BYTES, *a_lo = a_hi + A_BYTES;
    float *planes = reinterpret_cast<float *>(a_hi);
    const uint32_t mb = tc::smem_u32(&mbar[wg]);
    const uint32_t bar_id = 1 + wg;
    uint8_t *stg1 = smem + S::BASE + (size_t)wg * (S::STAGE1 + S::STAGE2), *stg2 = stg1 + S::STAGE1;
    const uint32_t mbt = tc::smem_u32(&mbar_tma[wg]);
    // (TMA writes need 128-byte aligned destinations: the staging region is placed at a
    // multiple of 1024 bytes from a dynamic-shared-memory base the kernel checks here)
    const bool use_tma = S::STAGE_BX > 0 && st.use != 0 && (tc::smem_u32(smem + S::BASE) & 1023u) == 0;

    // DFT matrix G = [[C, -S], [S, C]], hi/lo, in the shared layout buf(r, c)
    for (int t = tid; t < KK * KK; t += S::THREADS) {
        const int gr = t / KK, gc = t - gr * KK;
        const int n = gr % WS, k = gc % WS, q = (n * k) % WS;
        const float cv = kTw<WS>.c[q], sv = kTw<WS>.s[q];
        const float v = ((gr < WS) == (gc < WS)) ? cv : ((gr < WS) ? -sv : sv);
        uint16_t h, l;
        if constexpr (F16) tc::split_f16(v, h, l);
        else tc::split_bf16(v, h, l);
        const uint32_t o = (gc / 8) * (KK * 16) + gr * 16 + (gc % 8) * 2;
        *reinterpret_cast<uint16_t *>(g_hi + o) = h;
        *reinterpret_cast<uint16_t *>(g_lo + o) = l;
    }
    if (lt == 0) {
        tc::mbar_init(mb, 1);
        tc::mbar_init(mbt, 1);
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
    const uint32_t sg_hi = tc::smem_u32(g_hi), sg_lo = tc::smem_u32(g_lo);
    // pass-B row r of the window holds column kx; its partner -kx sits in lane
    const int kx = col_at<WS>(r);
    const int partner = (lane & ~(WS <= 32 ? WS - 1 : 31)) | (pos_of<WS>((WS - kx) % WS) & (WS <= 32 ? WS - 1 : 31));

    const int n_win = a.w_end - a.w_first;
    const int n_tiles = (n_win + NWIN - 1) / NWIN;
    uint32_t phase = 0;
    bool failed = false;

    // completion of the pass in flight: bounded wait, warp-uniform outcome
    auto wait_pass = [&]() -> bool {
        const bool ok = __all_sync(0xffffffffu, tc::mbar_wait(mb, phase & 1));
        ++phase;
        tc::fence_after_sync();
        return ok;
    };
    // operand writes -> visible to the MMA unit; false if any warp of the warpgroup failed
    auto sync_issue = [&](bool ok) -> bool {
        tc::fence_async_smem();
        tc::fence_before_sync();
        const bool bad = tc::named_sync_or(bar_id, 128, !ok);
        tc::fence_after_sync();
        return !bad;
    };

    // TMA staging: a tile is staged when its NWIN windows lie in one row of the window grid;
    // the box starts at the tile's first window, x rounded down to a 16-byte boundary
    uint32_t tphase = 0;
    int tma_pending = 0;
    auto in_row = [&](int tile) -> bool {
        const int w0 = a.w_first + tile * NWIN;
        return use_tma && (w0 % g.Nx_vec) + NWIN <= g.Nx_vec;
    };
    auto tile_x = [&](int tile, int &iy, int &ix0, int &x1, int &y1, int &x2) {
        const int w0 = a.w_first + tile * NWIN;
        iy = w0 / g.Nx_vec;
        ix0 = w0 - iy * g.Nx_vec;
        x1 = ix0 * g.sp_x - g.Nx_left + a.f1.mx;  // frame column of window 0 (padded frame)
        y1 = iy * g.sp_y - g.Ny_left + a.f1.my;
        x2 = ix0 * g.sp_x;                         // deformed-frame column of window 0
    };
    auto issue_stage = [&](int tile) {  // one thread
        int iy, ix0, x1, y1, x2;
        tile_x(tile, iy, ix0, x1, y1, x2);
        const int xa1 = x1 & ~15;
        const uint32_t bytes = (uint32_t)st.bx1 * WS + (DEF ? (uint32_t)st.bx2 * 4 * WS : (uint32_t)st.bx1 * WS);
        tc::mbar_expect_tx(mbt, bytes);
        tc::tma_load_2d(tc::smem_u32(stg1), &st.f1, xa1, y1, mbt);
        if constexpr (DEF) tc::tma_load_2d(tc::smem_u32(stg2), &st.f2, x2 & ~3, iy * g.sp_y, mbt);
        else tc::tma_load_2d(tc::smem_u32(stg2), &st.f2, xa1, y1, mbt);
    };
    {
        const int first = blockIdx.x * NG + wg;
        if (first < n_tiles && in_row(first)) {
            if (lt == 0) issue_stage(first);
            ++tma_pending;
        }
    }

    for (int tile = blockIdx.x * NG + wg; tile < n_tiles; tile += gridDim.x * NG) {
        const int w = a.w_first + tile * NWIN + wl;
        const bool staged = in_row(tile);
        bool ok_rows = true;

        // ---- pass A operand: row (wl, y = r) = [f1 row | f2 row], K-major ----
        {
            float v1[WS], v2[WS];
            if (staged) {
                // a copy that did not land in time stays pending (same phase) for the exit path
                ok_rows = __all_sync(0xffffffffu, tc::mbar_wait(mbt, tphase & 1));
                if (ok_rows) {
                    ++tphase;
                    --tma_pending;
                }
            }
            if (staged && ok_rows) {
                int iy, ix0, x1, y1, x2;
                tile_x(tile, iy, ix0, x1, y1, x2);
                const uint8_t *row1 = stg1 + r * st.bx1 + (x1 - (x1 & ~15)) + wl * g.sp_x;
                load_u8_row_shared<WS>(row1, v1);
                if constexpr (DEF) {
                    const float *row2 = reinterpret_cast<const float *>(stg2) + r * st.bx2 + (x2 - (x2 & ~3)) + wl * g.sp_x;
                    load_f32_row_shared<WS>(row2, v2);
                } else {
                    load_u8_row_shared<WS>(stg2 + r * st.bx1 + (x1 - (x1 & ~15)) + wl * g.sp_x, v2);
                }
                if (w >= a.w_end) {  // a partial last tile: windows past the launch read nothing
#pragma unroll
                    for (int i = 0; i < WS; ++i) v1[i] = v2[i] = 0.f;
                }
            } else if (!staged && w < a.w_end) {
                const int iy = w / g.Nx_vec, ix = w - iy * g.Nx_vec;
                const int x0 = ix * g.sp_x - g.Nx_left + a.f1.mx;
                const int y1 = iy * g.sp_y + r - g.Ny_left + a.f1.my;
                load_u8_row<WS>(a.f1.base + (size_t)y1 * a.f1.pitch + x0, v1);
                if constexpr (DEF) {
                    load_f32_row<WS>(a.def + (size_t)(iy * g.sp_y + r) * a.def_pitch + ix * g.sp_x, v2);
                } else {
                    load_u8_row<WS>(a.f2.base + (size_t)y1 * a.f2.pitch + x0, v2);
                }
            } else {
#pragma unroll
                for (int i = 0; i < WS; ++i) v1[i] = v2[i] = 0.f;
            }
            const uint32_t b1 = __ballot_sync(0xffffffffu, any_nonzero<WS>(v1));
            const uint32_t b2 = __ballot_sync(0xffffffffu, any_nonzero<WS>(v2));
            if (lane == 0) {
                s_nz1[wg][wq] = b1;
                s_nz2[wg][wq] = b2;
            }
#pragma unroll
            for (int c = 0; c < WS / 8; ++c) {
                // frame 1 (and frame 2 when undeformed) holds integers, exact in the operand
                // type: their lo part is zero and the MMAs skip it (LO_FROM)
                store8_exact<F16>(a_hi, tc::off_kmajor(lt, 8 * c, 128), v1 + 8 * c);
                if constexpr (DEF) store8<NPROD, F16>(a_hi, a_lo, tc::off_kmajor(lt, WS + 8 * c, 128), v2 + 8 * c);
                else store8_exact<F16>(a_hi, tc::off_kmajor(lt, WS + 8 * c, 128), v2 + 8 * c);
            }
        }
        if (!sync_issue(ok_rows)) {
            failed = true;
            break;
        }
        {
            // the staging buffer is consumed: stage the warpgroup's next tile behind this one
            const int next = tile + gridDim.x * NG;
            const bool stage_next = next < n_tiles && in_row(next);
            if (stage_next) ++tma_pending;
            if (lt == 0) {
                // frame 1 is integer-valued (exact in bf16); frame 2 only when deformed
                issue_pass<KK, KK, false, true, NPROD, DEF ? WS / 16 : KK / 16, F16>(tmem, sa_hi, sa_lo, sg_hi, sg_lo);
                tc::mma_commit(mb);
                if (stage_next) issue_stage(next);
            }
        }

        // ---- pass B operand: MN-major, m = (wl, position of kx), k = (re|im, y = r) ----
        {
            const bool ok = wait_pass();
            if (ok) {
                float zr[WS], zi[WS];
                tmem_row<WS>(lane_addr, zr);
                tmem_row<WS>(lane_addr + WS, zi);
                tc::tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < WS / 8; ++c) {
                    float br[8], bi[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        br[i] = zr[col_at<WS>(8 * c + i)];
                        bi[i] = zi[col_at<WS>(8 * c + i)];
                    }
                    store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wl * WS + 8 * c, r, KK), br, sB);
                    store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wl * WS + 8 * c, WS + r, KK), bi, sB);
                }
            }
            if (!sync_issue(ok)) {
                failed = true;
                break;
            }
        }
        if (lt == 0) {
            issue_pass<KK, KK, true, true, NPROD, 0, F16>(tmem, sa_hi, sa_lo, sg_hi, sg_lo);
            tc::mma_commit(mb);
        }

        // ---- cross spectrum; pass C operand: K-major row (wl, kx), k = (re|im, ky) ----
        const bool dead = window_dead<WS>(s_nz1[wg], s_nz2[wg], wl);
        {
            const bool ok = wait_pass();
            if (ok) {
                float zr[WS], zi[WS];
                tmem_row<WS>(lane_addr, zr);
                tmem_row<WS>(lane_addr + WS, zi);
                tc::tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < WS / 8; ++c) {
                    float cr[8], ci[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int ky = 8 * c + i, km = (WS - ky) % WS;
                        const float pr = __shfl_sync(0xffffffffu, zr[km], partner);
                        const float pi = __shfl_sync(0xffffffffu, zi[km], partner);
                        // scaled by sC, folded into the exact constant factors
                        cr[i] = dead ? 0.f : (0.5f * sC) * (zr[ky] * pi + zi[ky] * pr);
                        ci[i] = dead ? 0.f : (0.25f * sC) * ((pr * pr + pi * pi) - (zr[ky] * zr[ky] + zi[ky] * zi[ky]));
                    }
                    store8<NPROD, F16>(a_hi, a_lo, tc::off_kmajor(lt, 8 * c, 128), cr);
                    store8<NPROD, F16>(a_hi, a_lo, tc::off_kmajor(lt, WS + 8 * c, 128), ci);
                }
            }
            if (!sync_issue(ok)) {
                failed = true;
                break;
            }
        }
        if (lt == 0) {
            issue_pass<KK, KK, false, false, NPROD, 0, F16>(tmem, sa_hi, sa_lo, sg_hi, sg_lo);
            tc::mma_commit(mb);
        }

        // ---- pass D operand: MN-major, m = (wl, y), k = (re|im, kx) ----
        {
            const bool ok = wait_pass();
            if (ok) {
                float tr[WS], ti[WS];
                tmem_row<WS>(lane_addr, tr);
                tmem_row<WS>(lane_addr + WS, ti);
                tc::tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < WS / 8; ++c) {
                    store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wl * WS + 8 * c, kx, KK), tr + 8 * c, sD);
                    store8s<NPROD, F16, F16>(a_hi, a_lo, tc::off_mnmajor(wl * WS + 8 * c, WS + kx, KK), ti + 8 * c, sD);
                }
            }
            if (!sync_issue(ok)) {
                failed = true;
                break;
            }
        }
        if (lt == 0) {
            issue_pass<KK, WS, true, false, NPROD, 0, F16>(tmem, sa_hi, sa_lo, sg_hi, sg_lo);
            tc::mma_commit(mb);
        }

        // ---- correlation row (wl, y = r) -> |.|/N into the fftshifted plane ----
        {
            const bool ok = wait_pass();
            if (ok) {
                float cv[WS];
                tmem_row<WS>(lane_addr, cv);
                tc::tmem_wait_ld();
                float *prow = planes + wl * (WS * LDF) + ((r + WS / 2) % WS) * LDF;
                const float k = dead ? 0.f : out_scale;
#pragma unroll
                for (int x = 0; x < WS; ++x) prow[(x + WS / 2) % WS] = fabsf(cv[x]) * k;
            }
            tc::fence_before_sync();
            const bool bad = tc::named_sync_or(bar_id, 128, !ok);
            tc::fence_after_sync();
            if (bad) {
                failed = true;
                break;
            }
        }

        // ---- peaks: warp per window; two warps per 64-row window ----
        if constexpr (WS > 32) {
            static_assert(NWIN * 2 == 4, "two warps per window");
            static_assert((size_t)NWIN * WS * LDF * 4 + NWIN * sizeof(PeakPart[2]) <= 2 * A_BYTES, "peak scratch");
            PeakPart(*parts)[2] = reinterpret_cast<PeakPart(*)[2]>(planes + NWIN * WS * LDF);
            const int b = wq >> 1, part = wq & 1;
            const int wb = a.w_first + tile * NWIN + b;
            const float *P = planes + b * (WS * LDF);
            if (wb < a.w_end) peak_window_part<WS, WS, K>(a, P, part, lane, parts[b][part]);
            tc::named_sync(bar_id, 128);
            if (wb < a.w_end && part == 0) peak_window_merge<WS, WS>(a, P, wb, lane, parts[b]);
        } else {
            for (int b = wq; b < NWIN; b += 4) {
                const int wb = a.w_first + tile * NWIN + b;
                if (wb < a.w_end) peak_window<WS, WS, K>(a, planes + b * (WS * LDF), wb, lane);
            }
        }
        tc::named_sync(bar_id, 128);  // planes (aliasing the operand buffers) are consumed
    }

    if (failed) {
        if (lt == 0 && a.status) atomicOr(a.status, kStatusMmaWait);
        // the pass that did not complete in time gets one more bounded wait before the
        // tensor memory is released, and a staging copy still in flight one before the
        // shared memory is
        tc::mbar_wait(mb, (phase - 1) & 1);
        if (tma_pending > 0) tc::mbar_wait(mbt, tphase & 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid < 32) tc::tmem_dealloc(tmem_base, TALLOC);
}

// Launch of one tensor-core shape: one CTA per SM (a kernel using tensor memory is
// resident once per SM), persistent over the tiles.
template <int WS, int NPROD, bool F16>
cudaError_t launch_tc_shape(const XcorrArgs &a, bool deformed, int K, cudaStream_t s, const TcStaging *stage)
{
    using S = TcShape<WS>;
    const int n = a.w_end - a.w_first;
    if (n <= 0) return cudaSuccess;
    const int tiles = (n + (128 / WS) - 1) / (128 / WS);
    cudaError_t e = cudaSuccess;
    auto go = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        if (e != cudaSuccess) return;
        int dev = 0, sms = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return;
        const int want = (tiles + S::NG - 1) / S::NG;
        const int grid = want < sms ? want : sms;
        TcStaging none;
        memset(&none, 0, sizeof(none));
        kern<<<grid, S::THREADS, S::SMEM, s>>>(a, stage ? *stage : none);
        e = cudaGetLastError();
    };
    if (K <= 4) {
        if (deformed) go(xcorr_tc_kernel<WS, NPROD, 4, true, F16>);
        else go(xcorr_tc_kernel<WS, NPROD, 4, false, F16>);
    } else {
        if (deformed) go(xcorr_tc_kernel<WS, NPROD, 8, true, F16>);
        else go(xcorr_tc_kernel<WS, NPROD, 8, false, F16>);
    }
    return e;
}

}  // namespace piv
