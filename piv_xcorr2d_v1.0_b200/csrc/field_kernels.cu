// field_kernels.cu -- window deformation, grid upsampling and vector validation.
//
// The vector-field "extension" of the reference (extend_filtered_vecfield_p1/p2,
// X/xcorr2d_multi_grid.cu:1547-1618: thousands of 1-float device copies that pad the
// field with a 3-cell edge-replicated border) is not materialised: every read of the
// extended field at (m, n) reads the field at (clamp(m-3), clamp(n-3)), which is the
// same value.
#include "piv_common.cuh"

namespace piv {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Extended-field value at ext index (m, n) of a field with Nx x Ny vectors.
__device__ __forceinline__ float ext_field(const float *f, int Nx, int Ny, int m, int n)
{
    return __ldg(f + clampi(n - 3, 0, Ny - 1) * Nx + clampi(m - 3, 0, Nx - 1));
}

// ------------------------------------------------------------------------------
// Kernel_Window_Deformation_2d (X/xcorr2d_multi_grid.cu:608-652, launched at :1300
// and :1624).  Each thread produces 4 consecutive pixels of one row of the
// [Ny_aug][Nx_aug] deformed image and stores them as one float4.  The arithmetic is
// written exactly as the reference writes it.  Frame-2 taps outside the padded
// frame read 0 (the reference reads its zero padding there, or out of bounds).
// ------------------------------------------------------------------------------
// One output pixel of Kernel_Window_Deformation_2d given the 8 field values of its cell.
__device__ __forceinline__ float deform_pixel(const DeformArgs &a, int idx, int Y, float a_x, float a_y, float u1,
                                              float u2, float u3, float u4, float v1, float v2, float v3, float v4,
                                              int col_off, int row_off)
{
    float ce1 = (1 - a_x) * (1 - a_y);
    float ce2 = a_x * (1 - a_y);
    float ce3 = (1 - a_x) * a_y;
    float ce4 = a_x * a_y;
    a_x = (float)idx + ce1 * u1 + ce2 * u2 + ce3 * u3 + ce4 * u4;
    a_y = (float)Y + ce1 * v1 + ce2 * v2 + ce3 * v3 + ce4 * v4;
    int i_x = (int)floorf(a_x);
    int i_y = (int)floorf(a_y);
    a_x = a_x - (float)i_x;
    a_y = a_y - (float)i_y;
    // aug_ex column i_x + hfws_x holds image column i_x - Nx_left -> padded-frame column
    const int c0 = i_x + col_off, r0 = i_y + row_off;
    float p[4];
    if (c0 >= 0 && c0 + 1 < a.f2.cols && r0 >= 0 && r0 + 1 < a.f2.rows) {
        // all four taps inside the padded frame (the common case): no per-tap checks
        const uint8_t *q = a.f2.base + (size_t)r0 * a.f2.pitch + c0;
        p[0] = (float)__ldg(q);
        p[1] = (float)__ldg(q + 1);
        p[2] = (float)__ldg(q + a.f2.pitch);
        p[3] = (float)__ldg(q + a.f2.pitch + 1);
    } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int c = c0 + (t & 1), r = r0 + (t >> 1);
            p[t] = (c >= 0 && c < a.f2.cols && r >= 0 && r < a.f2.rows)
                       ? (float)__ldg(a.f2.base + (size_t)r * a.f2.pitch + c)
                       : 0.f;
        }
    }
    ce1 = (1 - a_x) * (1 - a_y);
    ce2 = a_x * (1 - a_y);
    ce3 = (1 - a_x) * a_y;
    ce4 = a_x * a_y;
    return ce1 * p[0] + ce2 * p[1] + ce3 * p[2] + ce4 * p[3];
}

// (v - st) / sp as the reference writes it; for a power-of-two spacing the reciprocal
// is exact, and multiplying by it gives the identical correctly rounded quotient.
template <bool POW2>
__device__ __forceinline__ float cell_coord(float v, float st, float sp, float inv_sp)
{
    if constexpr (POW2) return (v - st) * inv_sp;
    else return (v - st) / sp;
}

// Each thread writes 8 consecutive pixels of one row (two float4 stores).  When the
// vector spacing and the field origin are multiples of 8 (the `cell8` launches), the 8
// pixels lie in one cell of the field, so its 8 values are loaded once.  Bounded to 6
// blocks per SM (40 registers; the byte gathers want the warps: 88 -> 82 us at the
// 6600x4400 workload, against no change at 5 blocks and the unbounded 54 registers' 4).
template <bool CELL8, bool POW2>
__global__ void __launch_bounds__(256, 6) deform_kernel(const DeformArgs a)
{
    const int X0 = (blockIdx.x * blockDim.x + threadIdx.x) * 8;
    const int Y = blockIdx.y;
    if (X0 >= a.Nx_aug || Y >= a.Ny_aug) return;
    const float x_st_vec = (float)(a.hfws_x - a.sp_x * 3), y_st_vec = (float)(a.hfws_y - a.sp_y * 3);
    const float vsx = (float)a.sp_x, vsy = (float)a.sp_y;
    const float ivx = 1.0f / vsx, ivy = 1.0f / vsy;
    const int col_off = a.f2.mx - a.Nx_left, row_off = a.f2.my - a.Ny_left;

    float a_y = cell_coord<POW2>((float)Y, y_st_vec, vsy, ivy);
    const int i_y = (int)floorf(a_y);
    a_y = a_y - (float)i_y;

    float res[8];
    if (CELL8) {
        const int i_x = (int)floorf(cell_coord<POW2>((float)X0, x_st_vec, vsx, ivx));
        const float u1 = ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x, i_y);
        const float u2 = ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x + 1, i_y);
        const float u3 = ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x, i_y + 1);
        const float u4 = ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x + 1, i_y + 1);
        const float v1 = ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x, i_y);
        const float v2 = ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x + 1, i_y);
        const float v3 = ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x, i_y + 1);
        const float v4 = ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x + 1, i_y + 1);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = X0 + q;
            float a_x = cell_coord<POW2>((float)idx, x_st_vec, vsx, ivx);
            a_x = a_x - (float)i_x;
            res[q] = deform_pixel(a, idx, Y, a_x, a_y, u1, u2, u3, u4, v1, v2, v3, v4, col_off, row_off);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = X0 + q;
            float a_x = cell_coord<POW2>((float)idx, x_st_vec, vsx, ivx);
            const int i_x = (int)floorf(a_x);
            a_x = a_x - (float)i_x;
            res[q] = deform_pixel(a, idx, Y, a_x, a_y, ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x, i_y),
                                  ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x + 1, i_y),
                                  ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x, i_y + 1),
                                  ext_field(a.fx, a.Nx_vec, a.Ny_vec, i_x + 1, i_y + 1),
                                  ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x, i_y),
                                  ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x + 1, i_y),
                                  ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x, i_y + 1),
                                  ext_field(a.fy, a.Nx_vec, a.Ny_vec, i_x + 1, i_y + 1), col_off, row_off);
        }
    }
    float *dst = a.out + (size_t)Y * a.out_pitch + X0;
    if (X0 + 7 < a.Nx_aug) {
        reinterpret_cast<float4 *>(dst)[0] = make_float4(res[0], res[1], res[2], res[3]);
        reinterpret_cast<float4 *>(dst)[1] = make_float4(res[4], res[5], res[6], res[7]);
    } else {
        for (int q = 0; q < 8 && X0 + q < a.Nx_aug; ++q) dst[q] = res[q];
    }
}

cudaError_t launch_deform(const DeformArgs &a, cudaStream_t s)
{
    dim3 block(256);
    dim3 grid(((a.Nx_aug + 7) / 8 + 255) / 256, a.Ny_aug);
    // the 8-pixel runs X0..X0+7 (X0 % 8 == 0) share a field cell when the cell edges
    // x_st + m*sp are multiples of 8; the cell index is then exact for every pixel of
    // the run (its float quotient is exact for these small integers)
    const int x_st = a.hfws_x - a.sp_x * 3;
    const bool cell8 = (a.sp_x % 8 == 0) && (((x_st % 8) + 8) % 8 == 0);
    const bool pow2 = a.sp_x > 0 && a.sp_y > 0 && (a.sp_x & (a.sp_x - 1)) == 0 && (a.sp_y & (a.sp_y - 1)) == 0;
    if (cell8) {
        if (pow2) deform_kernel<true, true><<<grid, block, 0, s>>>(a);
        else deform_kernel<true, false><<<grid, block, 0, s>>>(a);
    } else {
        if (pow2) deform_kernel<false, true><<<grid, block, 0, s>>>(a);
        else deform_kernel<false, false><<<grid, block, 0, s>>>(a);
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------
// Autotuning input: a particle-like pattern (sparse bright pixels on a dark
// background) so that the timed correlation does its full candidate work.
// ------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hash2(uint32_t x, uint32_t y)
{
    uint32_t h = x * 0x9E3779B1u ^ (y + 0x7F4A7C15u) * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return h;
}

__global__ void pattern_kernel(uint8_t *u8, float *f32, int pitch, int cols, int rows, uint32_t seed)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= cols || y >= rows) return;
    const uint32_t h = hash2((uint32_t)x + seed, (uint32_t)y);
    const float v = (h % 23u == 0u) ? (float)(120u + (h >> 24) % 136u) : (float)(8u + (h >> 28));
    if (u8) u8[(size_t)y * pitch + x] = (uint8_t)v;
    if (f32) f32[(size_t)y * pitch + x] = v;
}

cudaError_t launch_pattern(uint8_t *u8, float *f32, int pitch, int cols, int rows, uint32_t seed, cudaStream_t s)
{
    dim3 grid((cols + 255) / 256, rows);
    pattern_kernel<<<grid, 256, 0, s>>>(u8, f32, pitch, cols, rows, seed);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------
// Upsampling_vecfield_kernel_2d (X/xcorr2d_multi_grid.cu:675-704) with the launch
// arguments of Upsampling_vector_field (:1580-1581).
// ------------------------------------------------------------------------------
__global__ void upsample_kernel(const UpsampleArgs a)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= a.Nx2 * a.Ny2) return;
    const float x_st_vec1 = (float)(a.sp_x1 / 2 - 3 * a.sp_x1), y_st_vec1 = (float)(a.sp_y1 / 2 - 3 * a.sp_y1);
    const float vs1x = (float)a.sp_x1, vs1y = (float)a.sp_y1;
    int idy = tid / a.Nx2;
    int idx = tid - idy * a.Nx2;
    idx = idx * a.sp_x2 + a.sp_x2 / 2;
    idy = idy * a.sp_y2 + a.sp_y2 / 2;
    float a_x = (float)(idx - x_st_vec1) / vs1x;
    float a_y = (float)(idy - y_st_vec1) / vs1y;
    const int i_x = (int)floorf(a_x);
    const int i_y = (int)floorf(a_y);
    a_x = a_x - (float)i_x;
    a_y = a_y - (float)i_y;
    const float ce1 = (1 - a_x) * (1 - a_y);
    const float ce2 = a_x * (1 - a_y);
    const float ce3 = (1 - a_x) * a_y;
    const float ce4 = a_x * a_y;
    a.fx2[tid] = ce1 * ext_field(a.fx1, a.Nx1, a.Ny1, i_x, i_y) + ce2 * ext_field(a.fx1, a.Nx1, a.Ny1, i_x + 1, i_y) +
                 ce3 * ext_field(a.fx1, a.Nx1, a.Ny1, i_x, i_y + 1) +
                 ce4 * ext_field(a.fx1, a.Nx1, a.Ny1, i_x + 1, i_y + 1);
    a.fy2[tid] = ce1 * ext_field(a.fy1, a.Nx1, a.Ny1, i_x, i_y) + ce2 * ext_field(a.fy1, a.Nx1, a.Ny1, i_x + 1, i_y) +
                 ce3 * ext_field(a.fy1, a.Nx1, a.Ny1, i_x, i_y + 1) +
                 ce4 * ext_field(a.fy1, a.Nx1, a.Ny1, i_x + 1, i_y + 1);
}

cudaError_t launch_upsample(const UpsampleArgs &a, cudaStream_t s)
{
    const int n = a.Nx2 * a.Ny2;
    upsample_kernel<<<(n + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------
// Validation.
// ------------------------------------------------------------------------------

// Calc_median (X/xcorr2d_multi_grid.cu:174-207) on a thread-private slice: (N+2)/2
// bubble passes move the largest values to the end, leaving the middle in place.
__device__ float median_bubble(float *d, int n, int stride)
{
    int cnt = n;
    for (int i = 0; i < (n + 2) / 2; i++) {
        cnt -= 1;
        float t1 = d[0];
        for (int j = 0; j < cnt; j++) {
            const float t2 = d[(1 + j) * stride];
            if (t1 > t2) {
                d[(1 + j) * stride] = t1;
                d[j * stride] = t2;
            } else {
                t1 = t2;
            }
        }
    }
    if (n % 2 == 0) return (d[(n / 2) * stride] + d[(n / 2 - 1) * stride]) / 2;
    return d[((n - 1) / 2) * stride];
}

// Ascending bitonic sort of a register array (N a power of two, all indices compile-time).
template <int N, int K, int J>
__device__ __forceinline__ void bitonic_step(float (&a)[N])
{
    static_for<0, N>([&](auto ic) {
        constexpr int i = decltype(ic)::value, l = i ^ J;
        if constexpr (l > i) {
            const float x = a[i], y = a[l];
            if constexpr ((i & K) == 0) {
                a[i] = fminf(x, y);
                a[l] = fmaxf(x, y);
            } else {
                a[i] = fmaxf(x, y);
                a[l] = fminf(x, y);
            }
        }
    });
    if constexpr (J > 1) bitonic_step<N, K, J / 2>(a);
}

template <int N, int K = 2>
__device__ __forceinline__ void bitonic_sort(float (&a)[N])
{
    bitonic_step<N, K, K / 2>(a);
    if constexpr (K < N) bitonic_sort<N, K * 2>(a);
}

// Median of the first n (<= N) entries of a sorted array, as Calc_median defines it
// (mean of the two middle values for even n, FP32).
// a[idx] for a runtime idx by a binary select tree over compile-time indices (keeps the
// array in registers; a compare-and-select loop is turned back into a local-memory load).
template <int N>
__device__ __forceinline__ float select_dyn(const float (&a)[N], int idx)
{
    if constexpr (N == 1) {
        return a[0];
    } else {
        float t[N / 2];
        const bool up = (idx & (N / 2)) != 0;
#pragma unroll
        for (int i = 0; i < N / 2; ++i) t[i] = up ? a[i + N / 2] : a[i];
        return select_dyn<N / 2>(t, idx);
    }
}

template <int N>
__device__ __forceinline__ float median_sorted(const float (&a)[N], int n)
{
    const float hi = select_dyn<N>(a, n / 2);  // n odd: (n-1)/2 == n/2
    if (n % 2 != 0) return hi;
    const float lo = select_dyn<N>(a, n / 2 - 1);
    return (hi + lo) / 2;
}

struct MedianPass {
    const float *cdx, *cdy;
    const uint8_t *cvalid;
    int Nps;
    const float *ix, *iy;  // input field; NULL -> candidate 0 (median_filter_data_prep)
    const uint8_t *iv;
    float *ox, *oy;
    uint8_t *ov;
    int Nx, Ny, wx, wy, minN;
    float thr;
    int median;        // 0: only copy candidate 0 (Npass_median == 0)
    int *list, *list_n;  // append invalid outputs here when non-NULL (fill work list)
};

// One pass of organize_median_filter_data + median_validity + Calc_median x4 +
// Calc_devi x2 + median_filtering (X/xcorr2d_multi_grid.cu:209-296, 1464-1513), one
// thread per vector.  Neighbours are gathered in raster stencil order with the centre
// slot (wx*wy-1)/2 skipped; the medians are order statistics, so the gather order
// does not change them.
__device__ __forceinline__ void median_neighbour(const MedianPass &a, int id, bool &ok, float &fxv, float &fyv)
{
    if (a.ix) {
        ok = a.iv[id] != 0;
        fxv = a.ix[id];
        fyv = a.iy[id];
    } else {
        ok = a.cvalid[(size_t)id * a.Nps] != 0;
        fxv = a.cdx[(size_t)id * a.Nps];
        fyv = a.cdy[(size_t)id * a.Nps];
    }
}

// median_filtering's decision: the first valid candidate whose normalised residuals are
// both below the insert threshold replaces the vector, else (0, 0, invalid).
__device__ __forceinline__ void median_decide(const MedianPass &a, int v, float mx, float my, float dmx, float dmy,
                                              float &rx, float &ry, uint8_t &rv)
{
    const float epsilon = 0.1f;  // X/xcorr2d_multi_grid.cuh:192
    for (int i = 0; i < a.Nps; ++i) {
        const size_t c = (size_t)v * a.Nps + i;
        if (!a.cvalid[c]) continue;
        const float cx = a.cdx[c], cy = a.cdy[c];
        const float devix = __fdiv_rn(fabsf(cx - mx), dmx + epsilon);
        const float deviy = __fdiv_rn(fabsf(cy - my), dmy + epsilon);
        if (devix < a.thr && deviy < a.thr) {
            rv = 1;
            rx = cx;
            ry = cy;
            return;
        }
    }
}

// One pass of organize_median_filter_data + median_validity + Calc_median x4 +
// Calc_devi x2 + median_filtering (X/xcorr2d_multi_grid.cu:209-296, 1464-1513), one
// thread per vector.  The medians are order statistics, so how they are found does not
// change them: REG (stencils of at most 32 cells) keeps one register slot per stencil
// cell (+inf when the neighbour is absent) and sorts with a bitonic network; larger
// stencils use the reference's partial bubble sort on a thread-private shared slice.
template <bool REG>
__global__ void __launch_bounds__(128) median_pass_kernel(const MedianPass a)
{
    extern __shared__ float sl[];
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int Nt = a.Nx * a.Ny;
    if (v >= Nt) return;
    const int Ntm = a.wx * a.wy;
    float rx = 0.f, ry = 0.f;
    uint8_t rv = 0;
    if (!a.median) {
        rx = a.cdx[(size_t)v * a.Nps];
        ry = a.cdy[(size_t)v * a.Nps];
        rv = a.cvalid[(size_t)v * a.Nps];
    } else {
        const int vy = v / a.Nx, vx = v - vy * a.Nx;
        const int hfwx = (a.wx - 1) / 2, hfwy = (a.wy - 1) / 2;
        const int centre = (Ntm - 1) / 2;
        if constexpr (REG) {
            const float inf = __int_as_float(0x7f800000);
            float xs[32], ys[32];
            int n = 0;
            int tx = 0, ty = 0;  // stencil column and row of slot t (no division per slot)
#pragma unroll
            for (int t = 0; t < 32; ++t) {
                const int x = vx - hfwx + tx, y = vy - hfwy + ty;
                const bool inb = (t < Ntm) & (t != centre) & (x >= 0) & (x <= a.Nx - 1) & (y >= 0) & (y <= a.Ny - 1);
                bool ok;
                float px, py;
                median_neighbour(a, inb ? y * a.Nx + x : v, ok, px, py);  // always a valid address
                ok = ok & inb;
                xs[t] = ok ? px : inf;
                ys[t] = ok ? py : inf;
                n += ok;
                const bool wrap = ++tx == a.wx;
                tx = wrap ? 0 : tx;
                ty += wrap;
            }
            if (n >= a.minN && n >= 1) {
                bitonic_sort<32>(xs);
                bitonic_sort<32>(ys);
                const float mx = median_sorted<32>(xs, n), my = median_sorted<32>(ys, n);
                // |x - median| over a sorted x falls, then rises (then +inf): a bitonic
                // sequence, which the final merge stage of the network sorts on its own
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    xs[q] = (q < n) ? fabsf(xs[q] - mx) : inf;
                    ys[q] = (q < n) ? fabsf(ys[q] - my) : inf;
                }
                bitonic_step<32, 32, 16>(xs);
                bitonic_step<32, 32, 16>(ys);
                const float dmx = median_sorted<32>(xs, n), dmy = median_sorted<32>(ys, n);
                median_decide(a, v, mx, my, dmx, dmy, rx, ry, rv);
            }
        } else {
            // thread-private slices interleaved across threads: element k of thread t at k*blockDim + t
            const int stride = blockDim.x;
            float *xs = sl + threadIdx.x, *ys = sl + (size_t)Ntm * blockDim.x + threadIdx.x;
            int n = 0;
            for (int t = 0; t < Ntm; ++t) {
                if (t == centre) continue;
                const int ty = t / a.wx, tx = t - ty * a.wx;
                const int x = vx - hfwx + tx, y = vy - hfwy + ty;
                if (x >= 0 && x <= a.Nx - 1 && y >= 0 && y <= a.Ny - 1) {
                    bool ok;
                    float fxv, fyv;
                    median_neighbour(a, y * a.Nx + x, ok, fxv, fyv);
                    if (ok) {
                        xs[n * stride] = fxv;
                        ys[n * stride] = fyv;
                        n++;
                    }
                }
            }
            if (n >= a.minN && n >= 1) {
                const float mx = median_bubble(xs, n, stride), my = median_bubble(ys, n, stride);
                for (int q = 0; q < n; ++q) {
                    xs[q * stride] = fabsf(xs[q * stride] - mx);
                    ys[q * stride] = fabsf(ys[q * stride] - my);
                }
                const float dmx = median_bubble(xs, n, stride), dmy = median_bubble(ys, n, stride);
                median_decide(a, v, mx, my, dmx, dmy, rx, ry, rv);
            }
        }
    }
    a.ox[v] = rx;
    a.oy[v] = ry;
    a.ov[v] = rv;
    if (a.list && !rv) a.list[atomicAdd(a.list_n, 1)] = v;
}

// fill_blank_vecfield + fill_blank_vecfield_update repeated until nothing changes
// (X/xcorr2d_multi_grid.cu:352-397, host loop :1514-1528), on the device without host
// polling: one CTA iterates over the list of invalid vectors.  valid codes: 0
// invalid, 1 valid, 2 filled in this iteration (not yet a source, as in the
// reference's two-kernel update).  The iteration count is capped at Nx+Ny+2 (the
// fill front advances at least one cell per iteration while anything changes); the
// cap sets a status bit instead of spinning.  cap_override > 0 lowers the cap (fault
// injection: a wide hole then hits it).
__global__ void __launch_bounds__(1024) fill_kernel(float *fx, float *fy, uint8_t *fv, int Nx, int Ny,
                                                    const int *list, const int *list_n, int *status,
                                                    int cap_override)
{
    __shared__ int s_cnt[2];
    const int n = *list_n;
    const int cap = cap_override > 0 ? cap_override : Nx + Ny + 2;
    if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int it = 0; it < cap; ++it) {
        int local = 0;
        for (int q = threadIdx.x; q < n; q += blockDim.x) {
            const int v = list[q];
            if (fv[v] != 0) continue;
            const int vy = v / Nx, vx = v - vy * Nx;
            int cnt = 0;
            float sumx = 0.f, sumy = 0.f;
            for (int j = max(0, vy - 1); j <= min(Ny - 1, vy + 1); j++)
                for (int k = max(0, vx - 1); k <= min(Nx - 1, vx + 1); k++) {
                    const int id = j * Nx + k;
                    if (fv[id] == 1) {
                        cnt += 1;
                        sumx += fx[id];
                        sumy += fy[id];
                    }
                }
            if (cnt > 0) {
                local++;
                fx[v] = __fdiv_rn(sumx, (float)cnt);
                fy[v] = __fdiv_rn(sumy, (float)cnt);
                fv[v] = 2;
            }
        }
        if (local) atomicAdd(&s_cnt[it & 1], local);
        __syncthreads();
        for (int q = threadIdx.x; q < n; q += blockDim.x) {
            const int v = list[q];
            if (fv[v] == 2) fv[v] = 1;
        }
        const int total = s_cnt[it & 1];
        if (threadIdx.x == 0) s_cnt[(it + 1) & 1] = 0;
        __syncthreads();
        if (total == 0) return;
    }
    if (threadIdx.x == 0) atomicOr(status, kStatusFillCap);
}

// organize_smooth_filter_data + smoothing_tophat (X/xcorr2d_multi_grid.cu:399-443):
// mean over the in-bounds wx x wy stencil, centre included, summed in raster order
// (the reference sums in atomic-arrival order).
__global__ void smooth_kernel(const float *ix, const float *iy, float *ox, float *oy, int Nx, int Ny, int wx, int wy)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= Nx * Ny) return;
    const int vy = v / Nx, vx = v - vy * Nx;
    const int hfwx = (wx - 1) / 2, hfwy = (wy - 1) / 2;
    float sx = 0.f, sy = 0.f;
    int n = 0;
    for (int ty = 0; ty < wy; ++ty)
        for (int tx = 0; tx < wx; ++tx) {
            const int x = vx - hfwx + tx, y = vy - hfwy + ty;
            if (x >= 0 && x <= Nx - 1 && y >= 0 && y <= Ny - 1) {
                sx += ix[y * Nx + x];
                sy += iy[y * Nx + x];
                n++;
            }
        }
    ox[v] = __fdiv_rn(sx, (float)n);
    oy[v] = __fdiv_rn(sy, (float)n);
}

// MedianFilter_Smoothing_p1/p2: median passes (ping-pong), fill in place, smoothing
// passes (ping-pong); the buffer order is chosen so the result lands in (fx, fy, fv).
cudaError_t launch_validate(const ValidateArgs &a, cudaStream_t s)
{
    const int Nt = a.Nx_vec * a.Ny_vec;
    const int steps_med = a.Npass_median > 0 ? a.Npass_median : 1;
    const int n_steps = steps_med + a.Npass_smooth;
    auto dst_is_canon = [&](int step) { return ((n_steps - step) % 2) == 0; };  // step is 1-based
    const float *cx = nullptr, *cy = nullptr;
    const uint8_t *cv = nullptr;
    cudaError_t e = cudaSuccess;
    int *list = a.iffill ? a.list : nullptr;
    if (list) {
        e = cudaMemsetAsync(a.list_n, 0, sizeof(int), s);
        if (e != cudaSuccess) return e;
    }
    const int tb = 128;
    for (int st = 1; st <= steps_med; ++st) {
        MedianPass m;
        m.cdx = a.cdx;
        m.cdy = a.cdy;
        m.cvalid = a.cvalid;
        m.Nps = a.Nps;
        m.ix = cx;
        m.iy = cy;
        m.iv = cv;
        const bool canon = dst_is_canon(st);
        m.ox = canon ? a.fx : a.tx;
        m.oy = canon ? a.fy : a.ty;
        m.ov = canon ? a.fv : a.tv;
        m.Nx = a.Nx_vec;
        m.Ny = a.Ny_vec;
        m.wx = a.wx_med;
        m.wy = a.wy_med;
        m.minN = a.minNneigh;
        m.thr = a.insert_threshold;
        m.median = a.Npass_median > 0;
        m.list = (st == steps_med) ? list : nullptr;
        m.list_n = a.list_n;
        if (a.wx_med * a.wy_med <= 32) {
            median_pass_kernel<true><<<(Nt + tb - 1) / tb, tb, 0, s>>>(m);
        } else {
            const size_t smem = m.median ? (size_t)2 * a.wx_med * a.wy_med * tb * sizeof(float) : 0;
            if (smem > 48 * 1024) {
                e = cudaFuncSetAttribute(median_pass_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
                if (e != cudaSuccess) return e;
            }
            median_pass_kernel<false><<<(Nt + tb - 1) / tb, tb, smem, s>>>(m);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        cx = m.ox;
        cy = m.oy;
        cv = m.ov;
    }
    if (a.iffill) {
        fill_kernel<<<1, 1024, 0, s>>>(const_cast<float *>(cx), const_cast<float *>(cy), const_cast<uint8_t *>(cv),
                                       a.Nx_vec, a.Ny_vec, a.list, a.list_n, a.status, a.fill_cap);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    for (int k = 0; k < a.Npass_smooth; ++k) {
        const int st = steps_med + 1 + k;
        const bool canon = dst_is_canon(st);
        float *ox = canon ? a.fx : a.tx, *oy = canon ? a.fy : a.ty;
        uint8_t *ov = canon ? a.fv : a.tv;
        smooth_kernel<<<(Nt + 255) / 256, 256, 0, s>>>(cx, cy, ox, oy, a.Nx_vec, a.Ny_vec, a.wx_sm, a.wy_sm);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        // validity is not changed by smoothing: carry it to the destination buffer
        if (ov != cv) {
            e = cudaMemcpyAsync(ov, cv, (size_t)Nt, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
        cx = ox;
        cy = oy;
        cv = ov;
    }
    return cudaSuccess;
}

}  // namespace piv
