// xcorr_generic.cu -- the correlation + peak kernel for every window shape the reference
// accepts (ws_x, ws_y multiples of 4 from 4 to 1024, X/xcorr2d_multi_grid.cu:896-920) and
// any Npeak_save, where the fused register-FFT kernels (xcorr_kernel.cuh, 8..64 px, top-8)
// have no instance.  It replaces the same reference steps as those kernels:
//   organize_data_fft2d_multi(_deformed)  X/xcorr2d_multi_grid.cu:497, 654
//   cufftExecC2C FORWARD x2 / INVERSE     :1334-1347, 1649-1662
//   multiply_conjugate, complex2amp       :519, 536
//   fftshift2d_xcorr2d_row/col            :547, 566
//   find_local_max_2d                     :585
//   reduce_max_index_*, replace_local_max :32, 103, 298 (Npeak_save rounds)
//   peak_subpixel_4peak_2d, remove_nan    :309, 457
//
// One CTA per window, persistent over the launch's windows.  The window's complex plane
// lives in shared memory when it fits (up to 20,480 points, e.g. 128x128 or 160x128), else
// in the CTA's slab of an engine-owned global workspace.
//   load     z = f1 + i*f2 written at the digit-reversed position of the forward
//            transform (mixed radix 4, 2, 3, 5, 7 and any other prime, outermost first);
//   forward  in-place decimation-in-time stages along x, then along y (natural output);
//   spectrum C(k) = conj(F1)F2 from Z(k), Z(-k) as in the fused kernels, C(-k) = conj C(k);
//   inverse  in-place decimation-in-frequency stages (natural input, digit-reversed output,
//            the same permutation), then |.|/N in place;
//   peaks    the fftshifted plane is read through index maps: 4-neighbour local maxima
//            inside the search region, their count, Npeak_save rounds of a block arg-max
//            (value desc, then lower index), the 3-point Gaussian fit with the FP64
//            log-ratio denominator, predictor, limits, NaN/Inf removal.
// Twiddles are exp(-2 pi i t/N) tables computed per CTA in FP64 and rounded once to FP32.
#include <cfloat>
#include <climits>

#include "piv_common.cuh"

namespace piv {

// Radices of the two dimensions (outermost first) and where the plane lives.
struct GenericPlan {
    int nfx, nfy;
    int fx[12], fy[12];
    int in_smem;  // 1: the plane in shared memory, 0: in the CTA's workspace slab
    int any;      // a radix above 7 (prime up to 251): the local-array stage
};

namespace {

constexpr int kGenThreads = kGenericThreads;
constexpr int kGenSmemPlane = 20480;  // complex points of a plane kept in shared memory

__device__ __forceinline__ float2 gmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// W_N^t (forward) or its conjugate (inverse) from the forward table
__device__ __forceinline__ float2 gtw(const float2 *W, int t, bool inv)
{
    const float2 w = W[t];
    return inv ? make_float2(w.x, -w.y) : w;
}

// R-point DFT of x in place: y[k] = sum_q x[q] W_R^(q k), W_R^e = W_N^(e N/R)
template <int R>
__device__ __forceinline__ void gdft(float2 (&x)[R], const float2 *W, int N, bool inv)
{
    if constexpr (R == 2) {
        const float2 a = x[0], b = x[1];
        x[0] = make_float2(a.x + b.x, a.y + b.y);
        x[1] = make_float2(a.x - b.x, a.y - b.y);
    } else if constexpr (R == 4) {
        const float2 a = x[0], b = x[1], c = x[2], d = x[3];
        const float2 t0 = make_float2(a.x + c.x, a.y + c.y), t1 = make_float2(a.x - c.x, a.y - c.y);
        const float2 t2 = make_float2(b.x + d.x, b.y + d.y), u = make_float2(b.x - d.x, b.y - d.y);
        // (b - d) times -i (forward) or +i (inverse)
        const float2 t3 = inv ? make_float2(-u.y, u.x) : make_float2(u.y, -u.x);
        x[0] = make_float2(t0.x + t2.x, t0.y + t2.y);
        x[1] = make_float2(t1.x + t3.x, t1.y + t3.y);
        x[2] = make_float2(t0.x - t2.x, t0.y - t2.y);
        x[3] = make_float2(t1.x - t3.x, t1.y - t3.y);
    } else {
        const int st = N / R;
        float2 y[R];
#pragma unroll
        for (int k = 0; k < R; ++k) {
            float2 acc = x[0];
#pragma unroll
            for (int q = 1; q < R; ++q) {
                const float2 p = gmul(x[q], gtw(W, ((q * k) % R) * st, inv));
                acc.x += p.x;
                acc.y += p.y;
            }
            y[k] = acc;
        }
#pragma unroll
        for (int k = 0; k < R; ++k) x[k] = y[k];
    }
}

// One stage along one dimension of the plane, for all lines.  Elements of a line are
// estride apart, lines lstride apart.  DIT (forward): blocks of L points combine R
// sub-transforms of M = L/R points: inputs at q*M + k1 are twiddled by W_L^(q k1) and
// transformed, outputs to k1 + M*k2.  DIF (inverse): inputs at m + M*q are transformed
// and the outputs twiddled by W_L^(m k2), to m + M*k2.  line_fast: consecutive threads
// take consecutive lines (columns: contiguous addresses) rather than consecutive points.
template <int R>
__device__ __forceinline__ void gstage(float2 *buf, int N, int L, int estride, int lines, int lstride,
                                       const float2 *W, bool inv, bool line_fast)
{
    const int M = L / R, tws = N / L, per_line = N / R, total = lines * per_line;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int line, t;
        if (line_fast) {
            t = b / lines;
            line = b - t * lines;
        } else {
            line = b / per_line;
            t = b - line * per_line;
        }
        const int blk = t / M, k1 = t - blk * M;
        float2 *base = buf + (size_t)line * lstride + (size_t)(blk * L + k1) * estride;
        const size_t step = (size_t)M * estride;
        float2 x[R];
#pragma unroll
        for (int q = 0; q < R; ++q) x[q] = base[q * step];
        if (!inv) {
#pragma unroll
            for (int q = 1; q < R; ++q) x[q] = gmul(x[q], gtw(W, (q * k1 * tws) % N, false));
            gdft<R>(x, W, N, false);
        } else {
            gdft<R>(x, W, N, true);
#pragma unroll
            for (int q = 1; q < R; ++q) x[q] = gmul(x[q], gtw(W, (q * k1 * tws) % N, true));
        }
#pragma unroll
        for (int q = 0; q < R; ++q) base[q * step] = x[q];
    }
}

// A stage of a prime radix above 7 (up to 251): the R-point DFT runs from a local array.
__device__ __noinline__ void gstage_any(float2 *buf, int R, int N, int L, int estride, int lines, int lstride,
                                        const float2 *W, bool inv, bool line_fast)
{
    const int M = L / R, tws = N / L, per_line = N / R, total = lines * per_line, st = N / R;
    float2 x[256];
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int line, t;
        if (line_fast) {
            t = b / lines;
            line = b - t * lines;
        } else {
            line = b / per_line;
            t = b - line * per_line;
        }
        const int blk = t / M, k1 = t - blk * M;
        float2 *base = buf + (size_t)line * lstride + (size_t)(blk * L + k1) * estride;
        const size_t step = (size_t)M * estride;
        for (int q = 0; q < R; ++q) {
            x[q] = base[q * step];
            if (!inv && q > 0) x[q] = gmul(x[q], gtw(W, (q * k1 * tws) % N, false));
        }
        for (int k = 0; k < R; ++k) {
            float2 acc = x[0];
            for (int q = 1; q < R; ++q) {
                const float2 p = gmul(x[q], gtw(W, ((q * k) % R) * st, inv));
                acc.x += p.x;
                acc.y += p.y;
            }
            if (inv && k > 0) acc = gmul(acc, gtw(W, (k * k1 * tws) % N, true));
            base[k * step] = acc;  // inputs are all in x already
        }
    }
}

// ANY: the instance that also carries the local-array stage for primes above 7 (its
// 2 KB per-thread stack is reserved only when such a window shape is launched)
template <bool ANY>
__device__ __forceinline__ void gstage_r(float2 *buf, int R, int N, int L, int estride, int lines, int lstride,
                                         const float2 *W, bool inv, bool line_fast)
{
    switch (R) {
    case 2: gstage<2>(buf, N, L, estride, lines, lstride, W, inv, line_fast); break;
    case 3: gstage<3>(buf, N, L, estride, lines, lstride, W, inv, line_fast); break;
    case 4: gstage<4>(buf, N, L, estride, lines, lstride, W, inv, line_fast); break;
    case 5: gstage<5>(buf, N, L, estride, lines, lstride, W, inv, line_fast); break;
    case 7: gstage<7>(buf, N, L, estride, lines, lstride, W, inv, line_fast); break;
    default:
        if constexpr (ANY) gstage_any(buf, R, N, L, estride, lines, lstride, W, inv, line_fast);
        break;
    }
}

// Forward (DIT, innermost radix first) or inverse (DIF, outermost first) transform of
// every line of one dimension.  f: radices, outermost first.
template <bool ANY>
__device__ void gfft_dim(float2 *buf, const int *f, int nf, int N, int estride, int lines, int lstride,
                         const float2 *W, bool inv, bool line_fast)
{
    if (!inv) {
        int L = 1;
        for (int s = nf - 1; s >= 0; --s) {
            L *= f[s];
            gstage_r<ANY>(buf, f[s], N, L, estride, lines, lstride, W, false, line_fast);
            __syncthreads();
        }
    } else {
        int L = N;
        for (int s = 0; s < nf; ++s) {
            gstage_r<ANY>(buf, f[s], N, L, estride, lines, lstride, W, true, line_fast);
            __syncthreads();
            L /= f[s];
        }
    }
}

// position of natural index n in the digit-reversed order of radices f (outermost first)
__device__ __forceinline__ int gperm(int n, const int *f, int nf, int N)
{
    int pos = 0, size = N;
    for (int s = 0; s < nf; ++s) {
        const int M = size / f[s];
        pos += (n % f[s]) * M;
        n /= f[s];
        size = M;
    }
    return pos;
}

__device__ __forceinline__ bool gbetter(float v1, int i1, float v2, int i2)
{
    return v1 > v2 || (v1 == v2 && i1 < i2);
}

// block-wide best (value desc, index asc) and, optionally, sum; every thread gets them
__device__ __forceinline__ void gblock_best(float &v, int &i, int &cnt, float *rv, int *ri, int *rc)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_down_sync(0xffffffffu, v, o);
        const int oi = __shfl_down_sync(0xffffffffu, i, o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        if (gbetter(ov, oi, v, i)) {
            v = ov;
            i = oi;
        }
    }
    __syncthreads();  // the previous round's readers are done with rv/ri/rc
    if (lane == 0) {
        rv[warp] = v;
        ri[warp] = i;
        rc[warp] = cnt;
    }
    __syncthreads();
    v = rv[0];
    i = ri[0];
    cnt = rc[0];
    for (int q = 1; q < nw; ++q) {
        if (gbetter(rv[q], ri[q], v, i)) {
            v = rv[q];
            i = ri[q];
        }
        cnt += rc[q];
    }
}

}  // namespace

template <bool DEF, bool ANY>
__global__ void __launch_bounds__(kGenThreads) xcorr_generic_kernel(const XcorrArgs a, const GenericPlan pl,
                                                                    float2 *gplane)
{
    const GridGeom &g = a.g;
    const int nx = g.ws_x, ny = g.ws_y, N = nx * ny, tid = threadIdx.x;
    extern __shared__ __align__(16) unsigned char gsm[];
    float2 *Wx = reinterpret_cast<float2 *>(gsm);
    float2 *Wy = Wx + nx;
    int *Sx = reinterpret_cast<int *>(Wy + ny);  // shifted column -> storage column
    int *Sy = Sx + nx;                            // shifted row -> storage row offset
    float *rv = reinterpret_cast<float *>(Sy + ny);
    int *ri = reinterpret_cast<int *>(rv + 32);
    int *rc = ri + 32;
    float *pv = reinterpret_cast<float *>(rc + 32);  // the window's picks
    int *pi = reinterpret_cast<int *>(pv + g.Nps);
    float2 *plane = pl.in_smem ? reinterpret_cast<float2 *>(
                                     gsm + (((size_t)(nx + ny) * 16 + 96 * 4 + (size_t)g.Nps * 8 + 15) & ~(size_t)15))
                               : gplane + (size_t)blockIdx.x * N;

    // tables: forward twiddles (FP64, rounded once) and the shifted-index maps
    for (int t = tid; t < nx; t += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)t / (double)nx, &s, &c);
        Wx[t] = make_float2((float)c, (float)(-s));
        Sx[t] = gperm((t + nx / 2) % nx, pl.fx, pl.nfx, nx);
    }
    for (int t = tid; t < ny; t += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)t / (double)ny, &s, &c);
        Wy[t] = make_float2((float)c, (float)(-s));
        Sy[t] = gperm((t + ny / 2) % ny, pl.fy, pl.nfy, ny) * nx;
    }
    __syncthreads();

    const float tiny = __int_as_float(1);  // v >= max(neighbours, tiny)  <=>  v > 0 and a local maximum
    const int ilo = g.bx > 1 ? g.bx : 1, ihi = min(nx - 1 - g.bx, nx - 2);
    const int jlo = g.by > 1 ? g.by : 1, jhi = min(ny - 1 - g.by, ny - 2);
    const int rw = ihi - ilo + 1, rh = jhi - jlo + 1, region = (rw > 0 && rh > 0) ? rw * rh : 0;

    for (int w = a.w_first + blockIdx.x; w < a.w_end; w += gridDim.x) {
        const int iy = w / g.Nx_vec, ix = w - iy * g.Nx_vec;
        // ---- load at the digit-reversed positions of the forward transform ----
        for (int t = tid; t < N; t += blockDim.x) {
            const int r = t / nx, i = t - r * nx;
            const int x0 = ix * g.sp_x - g.Nx_left + a.f1.mx, y1 = iy * g.sp_y + r - g.Ny_left + a.f1.my;
            const float v1 = (float)a.f1.base[(size_t)y1 * a.f1.pitch + x0 + i];
            float v2;
            if constexpr (DEF) v2 = a.def[(size_t)(iy * g.sp_y + r) * a.def_pitch + ix * g.sp_x + i];
            else v2 = (float)a.f2.base[(size_t)y1 * a.f2.pitch + x0 + i];
            plane[(size_t)gperm(r, pl.fy, pl.nfy, ny) * nx + gperm(i, pl.fx, pl.nfx, nx)] = make_float2(v1, v2);
        }
        __syncthreads();
        // ---- forward 2D transform: rows (x), then columns (y) ----
        gfft_dim<ANY>(plane, pl.fx, pl.nfx, nx, 1, ny, nx, Wx, false, false);
        gfft_dim<ANY>(plane, pl.fy, pl.nfy, ny, nx, nx, 1, Wy, false, true);
        // ---- cross spectrum, in place over (k, -k) pairs.  Z(0,0) = (sum f1, sum f2) is
        //      exactly zero iff a frame's window is all zero; the reference's correlation is
        //      then exactly 0 (no candidate), so the spectrum is set to 0 ----
        const float2 dc = plane[0];
        const bool dead = dc.x == 0.f || dc.y == 0.f;
        __syncthreads();  // every thread has read the DC term before it is overwritten
        for (int t = tid; t < N; t += blockDim.x) {
            const int ky = t / nx, kx = t - ky * nx;
            const int tm = ((ny - ky) % ny) * nx + (nx - kx) % nx;
            if (tm < t) continue;
            const float2 A = plane[t], M = plane[tm];
            const float2 C = dead ? make_float2(0.f, 0.f)
                                  : make_float2(0.5f * (A.x * M.y + A.y * M.x),
                                                0.25f * ((M.x * M.x + M.y * M.y) - (A.x * A.x + A.y * A.y)));
            plane[t] = C;
            if (tm != t) plane[tm] = make_float2(C.x, -C.y);
        }
        __syncthreads();
        // ---- inverse 2D transform (natural in, digit-reversed out), then |.|/N ----
        gfft_dim<ANY>(plane, pl.fy, pl.nfy, ny, nx, nx, 1, Wy, true, true);
        gfft_dim<ANY>(plane, pl.fx, pl.nfx, nx, 1, ny, nx, Wx, true, false);
        for (int t = tid; t < N; t += blockDim.x) {
            const float2 z = plane[t];
            plane[t].x = __fdiv_rn(sqrtf(z.x * z.x + z.y * z.y), (float)N);
        }
        __syncthreads();
        auto P = [&](int i, int j) -> float { return plane[Sy[j] + Sx[i]].x; };
        if (a.cc_dump) {
            float *dst = a.cc_dump + (size_t)(w - a.w_first) * N;
            for (int t = tid; t < N; t += blockDim.x) {
                const int j = t / nx, i = t - j * nx;
                dst[t] = P(i, j);
            }
            __syncthreads();
            continue;
        }
        // ---- peaks: Npeak_save rounds of a block arg-max over the local maxima ----
        float prev_v = FLT_MAX;
        int prev_i = -1, cnt = 0;
        for (int k = 0; k < g.Nps; ++k) {
            float bv = -1.f;
            int bi = INT_MAX, c = 0;
            if (prev_v > 0.f) {
                for (int t = tid; t < region; t += blockDim.x) {
                    const int jj = t / rw, j = jlo + jj, i = ilo + (t - jj * rw);
                    const float v = P(i, j);
                    const float m = fmaxf(fmaxf(P(i - 1, j), P(i + 1, j)), fmaxf(fmaxf(P(i, j - 1), P(i, j + 1)), tiny));
                    if (!(v >= m)) continue;
                    if (k == 0) ++c;
                    const int idx = j * nx + i;
                    if (gbetter(prev_v, prev_i, v, idx) && gbetter(v, idx, bv, bi)) {
                        bv = v;
                        bi = idx;
                    }
                }
            }
            gblock_best(bv, bi, c, rv, ri, rc);
            if (k == 0) cnt = c;
            if (tid == 0) {
                pv[k] = bv;
                pi[k] = bi;
            }
            prev_v = bv;
            prev_i = bi;
        }
        __syncthreads();
        // ---- fit and store (same arithmetic as the fused kernels' peak_fit_store) ----
        const float pred_x = a.pred_x[w], pred_y = a.pred_y[w];
        for (int k = tid; k < g.Nps; k += blockDim.x) {
            const float v = pv[k];
            const int idx = pi[k];
            float ox = 0.f, oy = 0.f;
            bool ok = false;
            if (v > 0.f) {
                const int j = idx / nx, i = idx - j * nx;
                if (i != 0 && i != nx - 1 && j != 0 && j != ny - 1) {
                    float sh[2];
                    for (int comp = 0; comp < 2; ++comp) {
                        const float f0 = comp ? P(i, j - 1) : P(i - 1, j);
                        const float f2 = comp ? P(i, j + 1) : P(i + 1, j);
                        const double dv = (double)v * (double)v;
                        const float nn = logf(f0) - logf(f2);
                        const double den = log(((double)f0 * (double)f2) / dv);
                        sh[comp] = (float)((double)nn / den / 2.0);
                    }
                    ox = (float)i + sh[0] - (float)nx / 2 + pred_x;
                    oy = (float)j + sh[1] - (float)ny / 2 + pred_y;
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
            }
            const size_t o = (size_t)w * g.Nps + k;
            a.cdx[o] = ox;
            a.cdy[o] = oy;
            a.cvalid[o] = ok ? 1 : 0;
            a.pidx[o] = (v > 0.f) ? idx : -1;
            a.pval[o] = (v > 0.f) ? v : 0.f;
        }
        if (tid == 0) a.count[w] = cnt;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------

namespace {
int radices(int n, int *f)
{
    int nf = 0;
    while (n % 4 == 0 && n > 4) {
        f[nf++] = 4;
        n /= 4;
    }
    for (int p = 2; n > 1; ++p)
        while (n % p == 0) {
            f[nf++] = p;
            n /= p;
        }
    return nf;
}

size_t table_bytes(int nx, int ny, int nps)
{
    return (((size_t)(nx + ny) * 16 + 96 * 4 + (size_t)nps * 8 + 15) & ~(size_t)15);
}
}  // namespace

GenericPlan generic_plan(int wsx, int wsy)
{
    GenericPlan pl{};
    pl.nfx = radices(wsx, pl.fx);
    pl.nfy = radices(wsy, pl.fy);
    pl.in_smem = wsx * wsy <= kGenSmemPlane ? 1 : 0;
    pl.any = 0;
    for (int s = 0; s < pl.nfx; ++s) pl.any |= pl.fx[s] > 7;
    for (int s = 0; s < pl.nfy; ++s) pl.any |= pl.fy[s] > 7;
    return pl;
}

bool xcorr_generic_needs_workspace(int wsx, int wsy) { return wsx * wsy > kGenSmemPlane; }

int xcorr_generic_ctas(int wsx, int wsy, int nps)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    if (xcorr_generic_needs_workspace(wsx, wsy)) return 2 * sms;
    const size_t smem = table_bytes(wsx, wsy, nps) + (size_t)wsx * wsy * sizeof(float2);
    const int by_smem = (int)((227 * 1024) / (smem + 1024));
    const int per_sm = by_smem < 1 ? 1 : (by_smem > 8 ? 8 : by_smem);
    return per_sm * sms;
}

cudaError_t launch_xcorr_generic(const XcorrArgs &a, bool deformed, float2 *workspace, int workspace_ctas,
                                 cudaStream_t s)
{
    const int n = a.w_end - a.w_first;
    if (n <= 0) return cudaSuccess;
    const GenericPlan pl = generic_plan(a.g.ws_x, a.g.ws_y);
    if (!pl.in_smem && (!workspace || workspace_ctas < 1)) return cudaErrorInvalidValue;
    const size_t smem = table_bytes(a.g.ws_x, a.g.ws_y, a.g.Nps) +
                        (pl.in_smem ? (size_t)a.g.ws_x * a.g.ws_y * sizeof(float2) : 0);
    int ctas = pl.in_smem ? xcorr_generic_ctas(a.g.ws_x, a.g.ws_y, a.g.Nps) : workspace_ctas;
    if (ctas > n) ctas = n;
    cudaError_t e = cudaSuccess;
    auto go = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return;
        kern<<<ctas, kGenThreads, smem, s>>>(a, pl, workspace);
        e = cudaGetLastError();
    };
    if (pl.any) {
        if (deformed) go(xcorr_generic_kernel<true, true>);
        else go(xcorr_generic_kernel<false, true>);
    } else {
        if (deformed) go(xcorr_generic_kernel<true, false>);
        else go(xcorr_generic_kernel<false, false>);
    }
    return e;
}

}  // namespace piv
