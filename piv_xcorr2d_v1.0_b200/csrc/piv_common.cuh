// piv_common.cuh -- shared definitions of the B200 PIV engine: geometry, kernel
// argument blocks, compile-time twiddle generation.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "piv_b200.h"

namespace piv {

// ---------------------------------------------------------------------------------
// Compile-time twiddle factors.  exp(-2*pi*i*a/n) is generated in FP64 at compile
// time: exact octant reduction of the rational angle a/n, then a Taylor series on
// [0, pi/4] (16 terms, error far below one FP64 ulp), rounded once to FP32.  The
// factors become instruction immediates; nothing is read from memory.
// ---------------------------------------------------------------------------------
constexpr double kPi = 3.141592653589793238462643383279502884;

constexpr double taylor_sin(double x)
{
    double x2 = x * x, term = x, sum = x;
    for (int k = 1; k < 16; ++k) {
        term *= -x2 / (double)((2 * k) * (2 * k + 1));
        sum += term;
    }
    return sum;
}

constexpr double taylor_cos(double x)
{
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int k = 1; k < 16; ++k) {
        term *= -x2 / (double)((2 * k - 1) * (2 * k));
        sum += term;
    }
    return sum;
}

struct CosSin {
    double c, s;
};

// cos and sin of pi*num/den with num in [0, 2*den).
constexpr CosSin cossin_pi_frac(long num, long den)
{
    bool neg_s = false;
    if (num > den) {  // theta in (pi, 2pi): reflect about 2pi
        num = 2 * den - num;
        neg_s = true;
    }
    bool neg_c = false;
    if (2 * num > den) {  // theta in (pi/2, pi]: reflect about pi
        num = den - num;
        neg_c = true;
    }
    double c = 0, s = 0;
    if (4 * num > den) {  // theta in (pi/4, pi/2]: swap via pi/2 - theta
        double t = kPi * (double)(den - 2 * num) / (double)(2 * den);
        c = taylor_sin(t);
        s = taylor_cos(t);
    } else {
        double t = kPi * (double)num / (double)den;
        c = taylor_cos(t);
        s = taylor_sin(t);
    }
    return CosSin{neg_c ? -c : c, neg_s ? -s : s};
}

// cos(2*pi*a/n), sin(2*pi*a/n)
constexpr CosSin cossin_2pi(long a, long n)
{
    long r = a % n;
    if (r < 0) r += n;
    return cossin_pi_frac(2 * r, n);
}

template <int Begin, int End, typename F>
__host__ __device__ __forceinline__ void static_for(F &&f)
{
    if constexpr (Begin < End) {
        f(std::integral_constant<int, Begin>{});
        static_for<Begin + 1, End>(static_cast<F &&>(f));
    }
}

// ---------------------------------------------------------------------------------
// Geometry (xcorr2d_multi::init, X/xcorr2d_multi_grid.cu:751-894), host side.
// ---------------------------------------------------------------------------------
int compute_geometry(const piv_params &p, piv_geometry &g, const char **why);

// Per-grid constants the kernels need.
struct GridGeom {
    int ws_x, ws_y, sp_x, sp_y;
    int Nx_vec, Ny_vec, Nt_vec;
    int bx, by;          // peak-search borders
    int Nx_left, Ny_left;
    int Nx_aug, Ny_aug;
    int hfws_x, hfws_y;
    int Nps;             // Npeak_save
    float lx1, lx2, ly1, ly2;
};

// A zero-padded uint8 frame: image pixel (x, y) lives at base[(y + my) * pitch + x + mx];
// everything outside the image inside the buffer is zero.
struct Frame8 {
    const uint8_t *base;
    int pitch, mx, my, cols, rows;  // cols = pitch, rows = Ny + 2*my
};

// Correlation + peak kernel arguments.
struct XcorrArgs {
    GridGeom g;
    Frame8 f1, f2;             // frame 1; frame 2 for the undeformed pass
    const float *def;          // deformed frame 2 [Ny_aug][def_pitch] (deformed passes)
    int def_pitch;
    const float *pred_x, *pred_y;  // predictor (filtered field) [Nt_vec]
    int w_first, w_end;        // window range of this launch
    float *cdx, *cdy;          // [Nt_vec][Nps]
    uint8_t *cvalid;
    int32_t *count;            // [Nt_vec]
    int32_t *pidx;             // [Nt_vec][Nps]
    float *pval;               // [Nt_vec][Nps]
    float *cc_dump;            // optional [n][ws_y][ws_x], window w -> cc_dump + (w - w_first)*ws_x*ws_y
    int *status;               // device status word (tensor-core path: kStatusMmaWait), may be null
};

// Batch of pairs sharing a window shape (one launch for all of them), passed whole as the
// kernel's parameter (about 24 KB, under the 32 KB parameter limit) so that the pairs'
// arguments are read from the constant bank: pairs[n], first[n + 1] the prefix sums of
// each pair's CTA-sized window batches.  Larger groups take several launches.
constexpr int kBatchMaxPairs = 96;
struct XcorrBatch {
    XcorrArgs pairs[kBatchMaxPairs];
    int first[kBatchMaxPairs + 1];
    int n, items;
};

// Launches the fused correlation + peak kernel for the window range of a.
// deformed: frame 2 comes from a.def (float) instead of a.f2 (uint8).  variant selects
// one of the shape's instantiations (windows per CTA, threads per CTA); 0 = default.
cudaError_t launch_xcorr(const XcorrArgs &a, bool deformed, cudaStream_t s, const char **why, int variant);
// Persistent batch launch over pairs sharing the window shape (wsx, wsy): variants
// 0 .. xcorr_batch_variants() - 1, each with its windows per CTA (items are batches of
// that many windows).  K: top-K width (4 or 8).
int xcorr_batch_variants(int wsx, int wsy);
int xcorr_batch_windows_per_cta(int wsx, int wsy, int variant);
cudaError_t launch_xcorr_batch(int wsx, int wsy, int variant, const XcorrBatch &b, bool deformed, int K,
                               cudaStream_t s, const char **why);
bool xcorr_supported(int ws_x, int ws_y);
int xcorr_variants(int ws_x, int ws_y);
bool xcorr_variant_shape(int ws_x, int ws_y, int variant, int *windows_per_cta, int *threads_per_cta);
// Tensor-core path (xcorr_tc.cuh): nprod 3 = split-BF16 (hi*hi + hi*lo + lo*hi), 1 = BF16.
bool xcorr_tc_supported(int ws_x, int ws_y);
// TMA staging of the tiles' rows (tensor-core kernels of 16 and 32 px windows): 2D tensor
// maps of frame 1 (u8) and of frame 2 (the u8 frame for an undeformed pass, the FP32 deformed
// frame otherwise), their boxes' widths in elements (frame 1, frame 2), and whether to use
// them (tc_staging_build sets use = 0 where the boxes do not fit the kernel's buffers).
struct TcStaging {
    CUtensorMap f1, f2;
    int bx1, bx2;
    int use;
};
// Encodes the maps for square WS x WS windows at spacing sp_x (box: a tile's 128/WS windows
// of one grid row, x rounded down to 16 bytes): frames f1, f2 of `pitch` x `rows` bytes,
// deformed frame `def` of def_pitch x def_rows floats (NULL: the undeformed form).
cudaError_t tc_staging_build(TcStaging &st, int ws, int sp_x, const uint8_t *f1, const uint8_t *f2, int pitch,
                             int rows, const float *def, int def_pitch, int def_rows);
cudaError_t launch_xcorr_tc(const XcorrArgs &a, bool deformed, cudaStream_t s, const char **why, int nprod,
                            bool f16, const TcStaging *stage);

// Field kernels (field_kernels.cu).
struct DeformArgs {
    Frame8 f2;
    float *out;
    int out_pitch;
    int Nx_aug, Ny_aug;
    const float *fx, *fy;   // filtered field of the grid
    int Nx_vec, Ny_vec;
    int sp_x, sp_y, hfws_x, hfws_y, Nx_left, Ny_left;
};
cudaError_t launch_deform(const DeformArgs &a, cudaStream_t s);

// Fills a uint8 and/or float buffer ([rows][pitch], first `cols` columns) with a
// particle-like pattern (autotuning input).
cudaError_t launch_pattern(uint8_t *u8, float *f32, int pitch, int cols, int rows, uint32_t seed, cudaStream_t s);

struct UpsampleArgs {
    const float *fx1, *fy1;
    int Nx1, Ny1, sp_x1, sp_y1;
    float *fx2, *fy2;
    int Nx2, Ny2, sp_x2, sp_y2;
};
cudaError_t launch_upsample(const UpsampleArgs &a, cudaStream_t s);

struct ValidateArgs {
    const float *cdx, *cdy;
    const uint8_t *cvalid;
    int Nps;
    int Nx_vec, Ny_vec;
    float *fx, *fy;      // canonical filtered field (result)
    uint8_t *fv;
    float *tx, *ty;      // scratch field
    uint8_t *tv;
    int wx_med, wy_med, Npass_median, minNneigh;
    float insert_threshold;
    int wx_sm, wy_sm, Npass_smooth, iffill;
    int *list, *list_n;  // fill work list [Nt_vec] and its length (device)
    int *status;         // device status word (bit 0: fill iteration cap)
    int fill_cap;        // hole-fill iteration cap; <= 0: Nx_vec + Ny_vec + 2
};
cudaError_t launch_validate(const ValidateArgs &a, cudaStream_t s);

// Generic-size correlation kernel (xcorr_generic.cu): any ws_x, ws_y multiple of 4 in
// [4, 1024] and up to kGenericMaxPeaks saved peaks.  Planes above 20,480 points need a
// workspace of workspace_ctas * ws_x * ws_y complex values.
constexpr int kGenericMaxPeaks = 1024;
constexpr int kGenericThreads = 256;
cudaError_t launch_xcorr_generic(const XcorrArgs &a, bool deformed, float2 *workspace, int workspace_ctas,
                                 cudaStream_t s);
bool xcorr_generic_needs_workspace(int wsx, int wsy);
int xcorr_generic_ctas(int wsx, int wsy, int nps);

// MHE (mhe_kernels.cu).
struct MheGeom {
    int Nx, Ny, ws, width, height, xs, ys, maxI, maxJ, Ntrash, Nnontrash;
};
bool mhe_geometry(int Nx, int Ny, int ws, float thresh, MheGeom &m);
// levels: (maxI+2)*(maxJ+2)*256 ints, ring pre-zeroed.  Output pixel (x, y) of the
// crop is written to out[(y + oy) * out_pitch + x + ox].
cudaError_t launch_mhe(const MheGeom &m, const uint8_t *in, int in_pitch, int *levels, uint8_t *out, int out_pitch,
                       int ox, int oy, cudaStream_t s);

// Status bits written by kernels.
enum : int { kStatusFillCap = 1, kStatusMmaWait = 2 };

}  // namespace piv
