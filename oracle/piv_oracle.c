/*
 * piv_oracle.c -- CPU restatement of the xinzhixue/PIV_xcorr2d_V1.0 hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): see piv_oracle.h for
 * who may call it and for the precision contract.  Built with -ffp-contract=off so
 * that every FP32 expression rounds exactly as written, like the reference's C.
 *
 * The oracle deliberately mirrors the reference's own data layout (zero-padded
 * aug_ex frames, the edge-replicated "_ex" vector field, Npeak candidate slots with
 * the two-stage arg-max tree) so that it is an independent restatement of the
 * reference rather than of the CUDA engine's design.
 */
#include "piv_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_PI 3.14159265358979323846

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }
static int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

int or_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------- */
/* Geometry: xcorr2d_multi::init, X/xcorr2d_multi_grid.cu:751-920             */
/* ------------------------------------------------------------------------- */

/* Vector count along one axis: the tmp1/tmp2 loop at X/xcorr2d_multi_grid.cu:771-777. */
static int vec_count(int N, int sp)
{
    int t1 = (N - sp / 2 - 1) / sp;
    int t2 = N - (sp / 2 + 1 + t1 * sp);
    while (t2 < (sp / 2 - 1)) {
        t1 = t1 - 1;
        t2 = t2 + sp;
    }
    return t1 + 1;
}

int or_geometry(const or_params *p, or_geom *g)
{
    if (!p || !g) return OR_ERR_ARG;
    memset(g, 0, sizeof(*g));
    if (p->Nx < 1 || p->Ny < 1 || p->Nsec_cc < 1 || p->Npeak_save < 1) return OR_ERR_ARG;
    for (int k = 0; k < 2; ++k) {
        if (p->sp_x[k] < 1 || p->sp_y[k] < 1) return OR_ERR_ARG;
        /* window validation, X/xcorr2d_multi_grid.cu:896-920 */
        if (p->ws_x[k] < 4 || p->ws_y[k] < 4) return OR_ERR_GEOMETRY;
        if (p->ws_x[k] > 1024 || p->ws_y[k] > 1024) return OR_ERR_GEOMETRY;
        if (p->ws_x[k] % 4 != 0 || p->ws_y[k] % 4 != 0) return OR_ERR_GEOMETRY;
    }
    for (int k = 0; k < 2; ++k) {
        int wsx = p->ws_x[k], wsy = p->ws_y[k], spx = p->sp_x[k], spy = p->sp_y[k];
        /* :751-754 */
        g->border_x[k] = imax(1, wsx / 2 - (int)roundf((float)wsx * p->pct_x[k]));
        g->border_y[k] = imax(1, wsy / 2 - (int)roundf((float)wsy * p->pct_y[k]));
        /* :761-769 */
        g->hfws_x[k] = wsx / 2;
        g->hfws_y[k] = wsy / 2;
        g->Npeak[k] = wsx * wsy / 4 / 4;
        /* :771-803 */
        g->Nx_vec[k] = vec_count(p->Nx, spx);
        g->Ny_vec[k] = vec_count(p->Ny, spy);
        g->Nt_vec[k] = g->Nx_vec[k] * g->Ny_vec[k];
        if (g->Nx_vec[k] < 1 || g->Ny_vec[k] < 1) return OR_ERR_GEOMETRY;
        /* :805-829 sectioning.  Nsec_cc > Nt_vec would loop forever in the reference. */
        int Nt = g->Nt_vec[k], Nsec = p->Nsec_cc;
        if (Nsec > Nt) return OR_ERR_ARG;
        if (Nt % Nsec == 0) {
            g->Neach[k] = Nt / Nsec;
            g->Nlast[k] = g->Neach[k];
        } else {
            g->Neach[k] = Nt / Nsec;
            g->Nlast[k] = Nt - (Nsec - 1) * g->Neach[k];
            while (g->Nlast[k] > g->Neach[k]) {
                g->Nlast[k] -= g->Neach[k];
                Nsec += 1;
            }
        }
        g->Nsec[k] = Nsec;
        /* :831-880 padding */
        int hx = g->hfws_x[k], hy = g->hfws_y[k];
        g->Nx_left[k] = (spx / 2 < hx) ? hx - spx / 2 : 0;
        g->Ny_left[k] = (spy / 2 < hy) ? hy - spy / 2 : 0;
        g->Nx_right[k] = ((p->Nx - spx / 2 - 1 - (g->Nx_vec[k] - 1) * spx) < (hx - 1))
                             ? spx / 2 + 1 + (g->Nx_vec[k] - 1) * spx + hx - 1 - p->Nx
                             : 0;
        g->Ny_right[k] = ((p->Ny - spy / 2 - 1 - (g->Ny_vec[k] - 1) * spy) < (hy - 1))
                             ? spy / 2 + 1 + (g->Ny_vec[k] - 1) * spy + hy - 1 - p->Ny
                             : 0;
        /* :882-894 */
        g->Nx_aug[k] = p->Nx + g->Nx_left[k] + g->Nx_right[k];
        g->Ny_aug[k] = p->Ny + g->Ny_left[k] + g->Ny_right[k];
        g->Nx_aug_ex[k] = g->Nx_aug[k] + wsx;
        g->Ny_aug_ex[k] = g->Ny_aug[k] + wsy;
    }
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* MHE: X/MHE7_4_gpu.cu:5-137 kernels, :149-253 host                          */
/* ------------------------------------------------------------------------- */
int or_mhe(const uint8_t *in, int Nx, int Ny, int ws, float thresh, uint8_t *out)
{
    if (!in || !out || Nx < 1 || Ny < 1 || ws < 1) return OR_ERR_ARG;
    int width, height, xs, ys;
    /* mhe_gpu::init :157-178 */
    if (Nx % ws == 0 && Ny % ws == 0) {
        height = Ny;
        width = Nx;
        xs = 0;
        ys = 0;
    } else {
        width = ws * (Nx / ws);
        xs = (Nx - width) / 2;
        height = ws * (Ny / ws);
        ys = (Ny - height) / 2;
    }
    int maxI = height / ws, maxJ = width / ws;
    if (maxI < 1 || maxJ < 1) return OR_ERR_ARG;
    int Ntrash = (int)roundf((float)(ws * ws) * thresh);
    int Nnontrash = ws * ws - Ntrash;
    if (Nnontrash <= 0) return OR_ERR_ARG; /* the reference divides by zero here */
    int Nw = maxI * maxJ;
    int *levels = (int *)calloc((size_t)(maxI + 2) * (maxJ + 2) * 256, sizeof(int));
    int *lut = (int *)malloc((size_t)Nw * 256 * sizeof(int));
    if (!levels || !lut) {
        free(levels);
        free(lut);
        return OR_ERR_ARG;
    }
    /* MakeHist_kernel :66-83 (zero-ringed tile grid) */
    for (int idy = 0; idy < height; ++idy)
        for (int idx = 0; idx < width; ++idx) {
            int pix = in[(size_t)(idy + ys) * Nx + xs + idx];
            int t = (maxJ + 2) * (idy / ws + 1) + 1 + idx / ws;
            levels[(size_t)t * 256 + pix] += 1;
        }
    for (int w = 0; w < Nw; ++w) {
        int ty = w / maxJ, tx = w - ty * maxJ;
        /* Calc_cnt_neigh_kernel :45-64 with (Nx, Ny) = (maxJ, maxI) */
        int cnt;
        if (tx >= 1 && tx <= maxJ - 2 && ty >= 1 && ty <= maxI - 2)
            cnt = 9;
        else if ((tx == 0 && ty == 0) || (tx == 0 && ty == maxI - 1) || (tx == maxJ - 1 && ty == 0) ||
                 (tx == maxJ - 1 && ty == maxI - 1))
            cnt = 4;
        else
            cnt = 6;
        /* CreateTransfer_kernel :85-101 */
        int c = (ty + 1) * (maxJ + 2) + 1 + tx;
        const int nb[9] = {c, c - 1, c + 1, c - maxJ - 2, c - maxJ - 1, c - maxJ - 3, c + maxJ + 2, c + maxJ + 1,
                           c + maxJ + 3};
        int cum = 0;
        for (int b = 0; b < 256; ++b) {
            int tr = 0;
            for (int q = 0; q < 9; ++q) tr += levels[(size_t)nb[q] * 256 + b];
            /* prescan_kernel :5-43: exclusive scan shifted by one = inclusive prefix sum */
            cum += tr;
            /* Calc_Enhanced_value_kernel :103-119 */
            int v = cum - cnt * Ntrash;
            v = (v >= 0) ? v : 0;
            v = imin(255, v * 255 / (cnt * Nnontrash));
            if (b == 0) v = 0;
            if (b == 255) v = 255;
            lut[(size_t)w * 256 + b] = v;
        }
    }
    /* Enhanced_kernel :121-137 into a zero-initialised output (mhe_gpu::init :197) */
    memset(out, 0, (size_t)Nx * Ny);
    for (int idy = 0; idy < height; ++idy)
        for (int idx = 0; idx < width; ++idx) {
            size_t pi = (size_t)(idy + ys) * Nx + xs + idx;
            int w = (idy / ws) * maxJ + idx / ws;
            out[pi] = (uint8_t)lut[(size_t)w * 256 + in[pi]];
        }
    free(levels);
    free(lut);
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* FP64 mixed-radix FFT (own implementation; the reference uses cuFFT C2C)     */
/* ------------------------------------------------------------------------- */
typedef struct {
    double re, im;
} cpx;

/* Decimation-in-time mixed-radix FFT of x[0], x[istride], ..., length n.
 * sign = -1 forward (cuFFT FORWARD), +1 inverse (unnormalised, cuFFT INVERSE).
 * tw[t] = exp(sign*2*pi*i*t/N0) for the top-level length N0, tstep = N0/n. */
static void fft_rec(const cpx *x, int istride, cpx *out, int n, const cpx *tw, int tstep, int N0)
{
    if (n == 1) {
        out[0] = x[0];
        return;
    }
    int p = 0;
    for (int f = 2; f * f <= n; ++f)
        if (n % f == 0) {
            p = f;
            break;
        }
    if (p == 0) p = n; /* prime length: direct DFT */
    int m = n / p;
    if (m == 1) {
        for (int k = 0; k < n; ++k) {
            double sr = 0, si = 0;
            for (int r = 0; r < n; ++r) {
                int t = (int)(((long)r * k % n) * tstep % N0);
                double a = x[r * istride].re, b = x[r * istride].im;
                sr += a * tw[t].re - b * tw[t].im;
                si += a * tw[t].im + b * tw[t].re;
            }
            out[k].re = sr;
            out[k].im = si;
        }
        return;
    }
    cpx *sub = (cpx *)malloc(sizeof(cpx) * (size_t)n);
    for (int r = 0; r < p; ++r) fft_rec(x + r * istride, istride * p, sub + r * m, m, tw, tstep * p, N0);
    for (int k = 0; k < m; ++k)
        for (int s = 0; s < p; ++s) {
            int kk = k + m * s;
            double sr = 0, si = 0;
            for (int r = 0; r < p; ++r) {
                int t = (int)(((long)r * kk % n) * tstep % N0);
                double a = sub[r * m + k].re, b = sub[r * m + k].im;
                sr += a * tw[t].re - b * tw[t].im;
                si += a * tw[t].im + b * tw[t].re;
            }
            out[kk].re = sr;
            out[kk].im = si;
        }
    free(sub);
}

static void twiddles(int N, int sign, cpx *tw)
{
    for (int t = 0; t < N; ++t) {
        double a = 2.0 * OR_PI * (double)t / (double)N;
        tw[t].re = cos(a);
        tw[t].im = sign * sin(a);
    }
}

/* 2D unnormalised transform of a [ny][nx] array, in place. */
static void fft2d(cpx *a, int nx, int ny, int sign)
{
    cpx *twx = (cpx *)malloc(sizeof(cpx) * (size_t)nx), *twy = (cpx *)malloc(sizeof(cpx) * (size_t)ny);
    cpx *tmp = (cpx *)malloc(sizeof(cpx) * (size_t)(nx > ny ? nx : ny));
    twiddles(nx, sign, twx);
    twiddles(ny, sign, twy);
    for (int j = 0; j < ny; ++j) {
        fft_rec(a + (size_t)j * nx, 1, tmp, nx, twx, 1, nx);
        memcpy(a + (size_t)j * nx, tmp, sizeof(cpx) * (size_t)nx);
    }
    for (int i = 0; i < nx; ++i) {
        fft_rec(a + i, nx, tmp, ny, twy, 1, ny);
        for (int j = 0; j < ny; ++j) a[(size_t)j * nx + i] = tmp[j];
    }
    free(twx);
    free(twy);
    free(tmp);
}

/* ------------------------------------------------------------------------- */
/* Correlation plane: organize_data -> FFT x2 -> multiply_conjugate -> IFFT ->  */
/* complex2amp -> fftshift row/col (X/xcorr2d_multi_grid.cu:497-583, 1315-1365) */
/* ------------------------------------------------------------------------- */
void or_xcorr_plane(const double *w1, const double *w2, int wsx, int wsy, double *cc, int direct)
{
    int N = wsx * wsy;
    if (direct) {
        /* IFFT(conj(F1) F2)[p]/N = sum_n f1[n] f2[n+p] (circular): exact for integer data. */
        for (int j = 0; j < wsy; ++j)
            for (int i = 0; i < wsx; ++i) {
                int py = (j + wsy / 2) % wsy, px = (i + wsx / 2) % wsx;
                double s = 0;
                for (int b = 0; b < wsy; ++b) {
                    int b2 = (b + py) % wsy;
                    for (int a = 0; a < wsx; ++a) s += w1[b * wsx + a] * w2[b2 * wsx + (a + px) % wsx];
                }
                cc[j * wsx + i] = fabs(s);
            }
        return;
    }
    cpx *A = (cpx *)malloc(sizeof(cpx) * (size_t)N), *B = (cpx *)malloc(sizeof(cpx) * (size_t)N);
    for (int n = 0; n < N; ++n) {
        A[n].re = w1[n];
        A[n].im = 0;
        B[n].re = w2[n];
        B[n].im = 0;
    }
    fft2d(A, wsx, wsy, -1);
    fft2d(B, wsx, wsy, -1);
    for (int n = 0; n < N; ++n) {
        /* multiply_conjugate :519-534: d1 <- conj(d1) * d2 */
        double x1 = A[n].re, y1 = A[n].im, x2 = B[n].re, y2 = B[n].im;
        A[n].re = x1 * x2 + y1 * y2;
        A[n].im = x1 * y2 - x2 * y1;
    }
    fft2d(A, wsx, wsy, +1);
    for (int j = 0; j < wsy; ++j)
        for (int i = 0; i < wsx; ++i) {
            /* fftshift row then column: shifted[j][i] = unshifted[(j+wsy/2)%wsy][(i+wsx/2)%wsx] */
            const cpx *v = &A[((j + wsy / 2) % wsy) * wsx + (i + wsx / 2) % wsx];
            /* complex2amp_xcorr2d :536-545: magnitude / (ws_x*ws_y) */
            cc[j * wsx + i] = sqrt(v->re * v->re + v->im * v->im) / (double)N;
        }
    free(A);
    free(B);
}

/* ------------------------------------------------------------------------- */
/* Peak search of one window (reference semantics)                             */
/* ------------------------------------------------------------------------- */

static int cmp_desc(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x < y) - (x > y);
}

static int next_pow2(int v)
{
    int b = 1;
    while (b < v) b <<= 1;
    return b;
}

/* One block of reduce_max_index_general/final (X/xcorr2d_multi_grid.cu:32-172): arg-max
 * of q values padded with zeros to the block size bn; `>=` keeps the lower lane.
 * Returns the winning value (sdata[0]) and the clamped lane min(q-1, index[0]). */
static double tree_argmax(const double *val, int q, int *lane)
{
    int bn = next_pow2(q);
    double s[1024];
    int ix[1024];
    for (int t = 0; t < bn; ++t) {
        s[t] = (t < q) ? val[t] : 0.0;
        ix[t] = t;
    }
    for (int off = bn / 2; off >= 1; off >>= 1)
        for (int t = 0; t < off; ++t) {
            ix[t] = (s[t] >= s[t + off]) ? ix[t] : ix[t + off];
            s[t] = (s[t] >= s[t + off]) ? s[t] : s[t + off]; /* fmaxf, no NaNs here */
        }
    *lane = imin(q - 1, ix[0]);
    return s[0];
}

void or_peaks_window(const double *cc, int wsx, int wsy, int bx, int by, int Npeak, int Nps, float pred_x,
                     float pred_y, float lx1, float lx2, float ly1, float ly2, float *dx, float *dy,
                     uint8_t *valid, int32_t *count_out, int32_t *pidx, float *pval, uint8_t *flags)
{
    double *sval = (double *)calloc((size_t)Npeak, sizeof(double));
    int *sidx = (int *)calloc((size_t)Npeak, sizeof(int));
    double *allv = (double *)malloc(sizeof(double) * (size_t)wsx * wsy);
    int count = 0;
    /* find_local_max_2d :585-606, candidates appended in raster order */
    for (int j = by; j <= wsy - 1 - by; ++j)
        for (int i = bx; i <= wsx - 1 - bx; ++i) {
            int t = j * wsx + i;
            double v = cc[t];
            if (v > 0 && v >= cc[t - 1] && v >= cc[t + 1] && v >= cc[t - wsx] && v >= cc[t + wsx]) {
                int slot = imin(count, Npeak - 1);
                sval[slot] = v;
                sidx[slot] = t;
                allv[count] = v;
                count++;
            }
        }
    uint8_t fl = 0;
    if (count > Npeak) fl |= 1;
    /* exact ties among the top Nps+1 values make the reference's pick order-dependent */
    {
        qsort(allv, (size_t)count, sizeof(double), cmp_desc);
        int top = imin(count, Nps + 1);
        for (int q = 1; q < top; ++q)
            if (allv[q] == allv[q - 1]) fl |= 2;
    }
    if (flags) *flags = fl;
    if (count_out) *count_out = count;

    int qx = wsx / 4, qy = wsy / 4;
    double part_v[256];
    int part_s[256];
    for (int k = 0; k < Nps; ++k) {
        /* reduce_max_index_general: one block per row of qx slots */
        for (int b = 0; b < qy; ++b) {
            int lane;
            part_v[b] = tree_argmax(sval + b * qx, qx, &lane);
            part_s[b] = b * qx + lane;
        }
        /* reduce_max_index_final over the qy partials */
        int lane;
        double v = tree_argmax(part_v, qy, &lane);
        int slot = part_s[lane];
        int li = sidx[slot]; /* d_index_local_tot[...]: 0 for an empty slot */
        /* replace_local_max_2d :298-307 (not after the last round) */
        if (k < Nps - 1) sval[slot] = -1000000.0;

        /* peak_subpixel_4peak_2d :309-350 */
        int iy = li / wsx, ix = li - iy * wsx;
        float ox = 0.f, oy = 0.f;
        uint8_t ok;
        if (ix == 0 || ix == wsx - 1 || iy == 0 || iy == wsy - 1 || v <= 0) {
            ok = 0;
        } else {
            ok = 1;
            double f1 = log(v), f0 = log(cc[li - 1]), f2 = log(cc[li + 1]);
            double ddx = (double)ix + (f0 - f2) / (f0 + f2 - 2.0 * f1) / 2.0 - (double)wsx / 2.0 + (double)pred_x;
            f0 = log(cc[li - wsx]);
            f2 = log(cc[li + wsx]);
            double ddy = (double)iy + (f0 - f2) / (f0 + f2 - 2.0 * f1) / 2.0 - (double)wsy / 2.0 + (double)pred_y;
            ox = (float)ddx;
            oy = (float)ddy;
            if (ox < lx1 || ox > lx2 || oy < ly1 || oy > ly2) {
                ok = 0;
                ox = 0.f;
                oy = 0.f;
            }
        }
        /* kernel_remove_nan :457-471 */
        if (isnan(ox) || isnan(oy) || isinf(ox) || isinf(oy)) {
            ox = 0.f;
            oy = 0.f;
            ok = 0;
        }
        dx[k] = ox;
        dy[k] = oy;
        valid[k] = ok;
        if (pidx) pidx[k] = (v > 0) ? li : -1;
        if (pval) pval[k] = (v > 0) ? (float)v : 0.f;
    }
    free(sval);
    free(sidx);
    free(allv);
}

/* ------------------------------------------------------------------------- */
/* Zero-padded frame for grid g: prep_img_data (X/xcorr2d_multi_grid.cu:1271-1282) */
/* ------------------------------------------------------------------------- */
static uint8_t *make_aug_ex(const uint8_t *img, const or_params *p, const or_geom *g, int k)
{
    size_t W = (size_t)g->Nx_aug_ex[k], H = (size_t)g->Ny_aug_ex[k];
    uint8_t *a = (uint8_t *)calloc(W * H, 1);
    if (!a) return NULL;
    for (int j = 0; j < p->Ny; ++j)
        memcpy(a + (size_t)(j + g->Ny_left[k] + g->hfws_y[k]) * W + g->Nx_left[k] + g->hfws_x[k],
               img + (size_t)j * p->Nx, (size_t)p->Nx);
    return a;
}

/* Edge-replicated field with a 3-cell border: extend_filtered_vecfield_p{1,2}
 * (X/xcorr2d_multi_grid.cu:1547-1576, 1589-1618). */
static float *make_ext(const float *f, int Nxv, int Nyv)
{
    int B = 3, Nxe = Nxv + 2 * B, Nye = Nyv + 2 * B;
    float *e = (float *)malloc(sizeof(float) * (size_t)Nxe * Nye);
    for (int n = 0; n < Nye; ++n)
        for (int m = 0; m < Nxe; ++m) e[(size_t)n * Nxe + m] = f[(size_t)iclamp(n - B, 0, Nyv - 1) * Nxv + iclamp(m - B, 0, Nxv - 1)];
    return e;
}

static float ext_at(const float *e, int Nxe, int Nye, int m, int n, long *oob)
{
    if (m < 0 || m >= Nxe || n < 0 || n >= Nye) {
        (*oob)++;
        m = iclamp(m, 0, Nxe - 1);
        n = iclamp(n, 0, Nye - 1);
    }
    return e[(size_t)n * Nxe + m];
}

long or_deform(const uint8_t *img2, const or_params *p, const or_geom *g, int k, const float *fx, const float *fy,
               float *out)
{
    uint8_t *aug = make_aug_ex(img2, p, g, k);
    int Nxv = g->Nx_vec[k], Nyv = g->Ny_vec[k], Nxe = Nxv + 6, Nye = Nyv + 6;
    float *ex = make_ext(fx, Nxv, Nyv), *ey = make_ext(fy, Nxv, Nyv);
    int Nx_aug = g->Nx_aug[k], Ny_aug = g->Ny_aug[k], W = g->Nx_aug_ex[k];
    long Nt_ex = (long)W * g->Ny_aug_ex[k];
    /* launch arguments of :1300 / :1624 */
    int x_st_inten = -g->hfws_x[k], y_st_inten = -g->hfws_y[k];
    float x_st_vec = (float)(g->hfws_x[k] - p->sp_x[k] * 3), y_st_vec = (float)(g->hfws_y[k] - p->sp_y[k] * 3);
    float spx = (float)p->sp_x[k], spy = (float)p->sp_y[k];
    long oob = 0;
#pragma omp parallel for reduction(+ : oob) schedule(static)
    for (int idy = 0; idy < Ny_aug; ++idy) {
        for (int idx = 0; idx < Nx_aug; ++idx) {
            /* Kernel_Window_Deformation_2d :608-652 */
            float a_x = ((float)idx - x_st_vec) / spx;
            float a_y = ((float)idy - y_st_vec) / spy;
            int i_x = (int)floorf(a_x);
            int i_y = (int)floorf(a_y);
            a_x = a_x - (float)i_x;
            a_y = a_y - (float)i_y;
            float ce1 = (1 - a_x) * (1 - a_y);
            float ce2 = a_x * (1 - a_y);
            float ce3 = (1 - a_x) * a_y;
            float ce4 = a_x * a_y;
            float u1 = ext_at(ex, Nxe, Nye, i_x, i_y, &oob), u2 = ext_at(ex, Nxe, Nye, i_x + 1, i_y, &oob);
            float u3 = ext_at(ex, Nxe, Nye, i_x, i_y + 1, &oob), u4 = ext_at(ex, Nxe, Nye, i_x + 1, i_y + 1, &oob);
            float v1 = ext_at(ey, Nxe, Nye, i_x, i_y, &oob), v2 = ext_at(ey, Nxe, Nye, i_x + 1, i_y, &oob);
            float v3 = ext_at(ey, Nxe, Nye, i_x, i_y + 1, &oob), v4 = ext_at(ey, Nxe, Nye, i_x + 1, i_y + 1, &oob);
            a_x = (float)idx + ce1 * u1 + ce2 * u2 + ce3 * u3 + ce4 * u4;
            a_y = (float)idy + ce1 * v1 + ce2 * v2 + ce3 * v3 + ce4 * v4;
            i_x = (int)floorf(a_x);
            i_y = (int)floorf(a_y);
            a_x = a_x - (float)i_x;
            a_y = a_y - (float)i_y;
            i_x = i_x - x_st_inten;
            i_y = i_y - y_st_inten;
            long i1 = (long)i_y * W + i_x, i2 = i1 + 1, i3 = i1 + W, i4 = i3 + 1;
            ce1 = (1 - a_x) * (1 - a_y);
            ce2 = a_x * (1 - a_y);
            ce3 = (1 - a_x) * a_y;
            ce4 = a_x * a_y;
            float p1 = 0, p2 = 0, p3 = 0, p4 = 0;
            if (i1 >= 0 && i1 < Nt_ex) p1 = aug[i1]; else oob++;
            if (i2 >= 0 && i2 < Nt_ex) p2 = aug[i2]; else oob++;
            if (i3 >= 0 && i3 < Nt_ex) p3 = aug[i3]; else oob++;
            if (i4 >= 0 && i4 < Nt_ex) p4 = aug[i4]; else oob++;
            out[(size_t)idy * Nx_aug + idx] = ce1 * p1 + ce2 * p2 + ce3 * p3 + ce4 * p4;
        }
    }
    free(aug);
    free(ex);
    free(ey);
    return oob;
}

void or_upsample(const or_params *p, const or_geom *g, const float *fx1, const float *fy1, float *fx2, float *fy2)
{
    int Nx1 = g->Nx_vec[0], Ny1 = g->Ny_vec[0], Nxe = Nx1 + 6, Nye = Ny1 + 6;
    float *ex = make_ext(fx1, Nx1, Ny1), *ey = make_ext(fy1, Nx1, Ny1);
    /* launch arguments of Upsampling_vector_field :1580-1581 */
    float x_st_vec1 = (float)(p->sp_x[0] / 2 - 3 * p->sp_x[0]);
    float y_st_vec1 = (float)(p->sp_y[0] / 2 - 3 * p->sp_y[0]);
    float sp1x = (float)p->sp_x[0], sp1y = (float)p->sp_y[0];
    int sp2x = p->sp_x[1], sp2y = p->sp_y[1];
    long oob = 0;
    for (int l = 0; l < g->Ny_vec[1]; ++l)
        for (int kx = 0; kx < g->Nx_vec[1]; ++kx) {
            /* Upsampling_vecfield_kernel_2d :675-704 */
            int idx = kx * sp2x + sp2x / 2;
            int idy = l * sp2y + sp2y / 2;
            float a_x = (float)(idx - x_st_vec1) / sp1x;
            float a_y = (float)(idy - y_st_vec1) / sp1y;
            int i_x = (int)floorf(a_x);
            int i_y = (int)floorf(a_y);
            a_x = a_x - (float)i_x;
            a_y = a_y - (float)i_y;
            float ce1 = (1 - a_x) * (1 - a_y);
            float ce2 = a_x * (1 - a_y);
            float ce3 = (1 - a_x) * a_y;
            float ce4 = a_x * a_y;
            size_t o = (size_t)l * g->Nx_vec[1] + kx;
            fx2[o] = ce1 * ext_at(ex, Nxe, Nye, i_x, i_y, &oob) + ce2 * ext_at(ex, Nxe, Nye, i_x + 1, i_y, &oob) +
                     ce3 * ext_at(ex, Nxe, Nye, i_x, i_y + 1, &oob) + ce4 * ext_at(ex, Nxe, Nye, i_x + 1, i_y + 1, &oob);
            fy2[o] = ce1 * ext_at(ey, Nxe, Nye, i_x, i_y, &oob) + ce2 * ext_at(ey, Nxe, Nye, i_x + 1, i_y, &oob) +
                     ce3 * ext_at(ey, Nxe, Nye, i_x, i_y + 1, &oob) + ce4 * ext_at(ey, Nxe, Nye, i_x + 1, i_y + 1, &oob);
        }
    free(ex);
    free(ey);
}

/* ------------------------------------------------------------------------- */
/* Correlation pass of one grid                                               */
/* ------------------------------------------------------------------------- */
static int peaks_common(const float *cc_f32, const uint8_t *img1, const uint8_t *img2, const float *deformed,
                        const or_params *p, const or_geom *g, int k, const float *pred_x, const float *pred_y,
                        int direct, or_candidates *out)
{
    int wsx = p->ws_x[k], wsy = p->ws_y[k], N = wsx * wsy, Nps = p->Npeak_save;
    uint8_t *a1 = NULL, *a2 = NULL;
    if (!cc_f32) {
        a1 = make_aug_ex(img1, p, g, k);
        if (!deformed) a2 = make_aug_ex(img2, p, g, k);
    }
    int W = g->Nx_aug_ex[k], Wd = g->Nx_aug[k];
    long Nt_ex = (long)W * g->Ny_aug_ex[k], Nt_aug = (long)g->Nx_aug[k] * g->Ny_aug[k];
    int bad = 0;
#pragma omp parallel
    {
        double *w1 = (double *)malloc(sizeof(double) * N), *w2 = (double *)malloc(sizeof(double) * N);
        double *cc = (double *)malloc(sizeof(double) * N);
#pragma omp for schedule(dynamic, 16)
        for (int w = 0; w < g->Nt_vec[k]; ++w) {
            int ix_w = w % g->Nx_vec[k], iy_w = w / g->Nx_vec[k];
            if (cc_f32) {
                for (int n = 0; n < N; ++n) cc[n] = (double)cc_f32[(size_t)w * N + n];
            } else {
                for (int j = 0; j < wsy; ++j)
                    for (int i = 0; i < wsx; ++i) {
                        /* organize_data_fft2d_multi :497-517 (border = hfws, Nx_img = Nx_aug_ex) */
                        long id = (long)(iy_w * p->sp_y[k] + j + g->hfws_y[k]) * W + ix_w * p->sp_x[k] + i + g->hfws_x[k];
                        if (id < 0 || id >= Nt_ex) {
#pragma omp atomic write
                            bad = 1;
                            id = 0;
                        }
                        w1[j * wsx + i] = a1[id];
                        if (!deformed) {
                            w2[j * wsx + i] = a2[id];
                        } else {
                            /* organize_data_fft2d_multi_deformed :654-673 (Nx_img = Nx_aug) */
                            long jd = (long)(iy_w * p->sp_y[k] + j) * Wd + ix_w * p->sp_x[k] + i;
                            if (jd < 0 || jd >= Nt_aug) {
#pragma omp atomic write
                                bad = 1;
                                jd = 0;
                            }
                            w2[j * wsx + i] = (double)deformed[jd];
                        }
                    }
                or_xcorr_plane(w1, w2, wsx, wsy, cc, direct);
            }
            size_t o = (size_t)w * Nps;
            or_peaks_window(cc, wsx, wsy, g->border_x[k], g->border_y[k], g->Npeak[k], Nps, pred_x ? pred_x[w] : 0.f,
                            pred_y ? pred_y[w] : 0.f, p->lim_x1, p->lim_x2, p->lim_y1, p->lim_y2, out->dx + o,
                            out->dy + o, out->valid + o, out->count ? out->count + w : NULL,
                            out->peak_index ? out->peak_index + o : NULL, out->peak_value ? out->peak_value + o : NULL,
                            out->flags ? out->flags + w : NULL);
        }
        free(w1);
        free(w2);
        free(cc);
    }
    free(a1);
    free(a2);
    return bad ? OR_ERR_GEOMETRY : OR_OK;
}

int or_correlate_grid(const uint8_t *img1, const uint8_t *img2, const float *deformed, const or_params *p,
                      const or_geom *g, int k, const float *pred_x, const float *pred_y, int direct,
                      or_candidates *out)
{
    if (!img1 || !p || !g || !out || (!deformed && !img2) || k < 0 || k > 1) return OR_ERR_ARG;
    return peaks_common(NULL, img1, img2, deformed, p, g, k, pred_x, pred_y, direct, out);
}

int or_peaks_from_planes(const float *cc, const or_params *p, const or_geom *g, int k, const float *pred_x,
                         const float *pred_y, or_candidates *out)
{
    if (!cc || !p || !g || !out || k < 0 || k > 1) return OR_ERR_ARG;
    return peaks_common(cc, NULL, NULL, NULL, p, g, k, pred_x, pred_y, 0, out);
}

/* ------------------------------------------------------------------------- */
/* Validation (FP32, as written in the reference)                             */
/* ------------------------------------------------------------------------- */

/* Calc_median :174-207: (N+2)/2 bubble passes carry the largest values to the end;
 * the middle element(s) are then in place. */
static float median_bubble(float *d, int n)
{
    int cnt = n;
    for (int i = 0; i < (n + 2) / 2; i++) {
        cnt -= 1;
        float t1 = d[0];
        for (int j = 0; j < cnt; j++) {
            float t2 = d[1 + j];
            if (t1 > t2) {
                d[1 + j] = t1;
                d[j] = t2;
            } else {
                t1 = t2;
            }
        }
    }
    if (n % 2 == 0) return (d[n / 2] + d[n / 2 - 1]) / 2;
    return d[(n - 1) / 2];
}

int or_validate(const float *cdx, const float *cdy, const uint8_t *cvalid, int Nxv, int Nyv, int Nps, int wx_med,
                int wy_med, int wx_sm, int wy_sm, const or_valid_cfg *cfg, float *fx, float *fy, uint8_t *fvalid,
                int *fill_iters)
{
    if (!cdx || !cdy || !cvalid || !cfg || !fx || !fy || !fvalid || wx_med < 1 || wy_med < 1 || wx_sm < 1 || wy_sm < 1)
        return OR_ERR_ARG;
    int Nt = Nxv * Nyv, Ntm = wx_med * wy_med, Nts = wx_sm * wy_sm;
    const float epsilon = 0.1f; /* X/xcorr2d_multi_grid.cuh:192 */
    float *nx = (float *)malloc(sizeof(float) * Nt), *ny = (float *)malloc(sizeof(float) * Nt);
    uint8_t *nv = (uint8_t *)malloc(Nt);
    /* median_filter_data_prep :484-495 */
    for (int v = 0; v < Nt; ++v) {
        fvalid[v] = cvalid[(size_t)v * Nps];
        fx[v] = cdx[(size_t)v * Nps];
        fy[v] = cdy[(size_t)v * Nps];
    }
    int hfwx = (wx_med - 1) / 2, hfwy = (wy_med - 1) / 2;
    for (int pass = 0; pass < cfg->Npass_median; ++pass) {
#pragma omp parallel
        {
            float *xs = (float *)malloc(sizeof(float) * Ntm), *ys = (float *)malloc(sizeof(float) * Ntm);
#pragma omp for schedule(static)
            for (int v = 0; v < Nt; ++v) {
                int vy = v / Nxv, vx = v - vy * Nxv, n = 0;
                /* organize_median_filter_data :255-283 (raster stencil order, centre slot skipped) */
                for (int t = 0; t < Ntm; ++t) {
                    if (t == (Ntm - 1) / 2) continue;
                    int ty = t / wx_med, tx = t - ty * wx_med;
                    int x = vx - hfwx + tx, y = vy - hfwy + ty;
                    if (x >= 0 && x <= Nxv - 1 && y >= 0 && y <= Nyv - 1 && fvalid[y * Nxv + x]) {
                        xs[n] = fx[y * Nxv + x];
                        ys[n] = fy[y * Nxv + x];
                        n++;
                    }
                }
                /* median_validity :285-296; an empty neighbourhood never counts */
                int vm = (n >= cfg->minNneigh) && n >= 1;
                nx[v] = 0;
                ny[v] = 0;
                nv[v] = 0;
                if (vm) {
                    float mx = median_bubble(xs, n), my = median_bubble(ys, n);
                    /* Calc_devi :209-223 */
                    for (int q = 0; q < n; ++q) {
                        xs[q] = fabsf(xs[q] - mx);
                        ys[q] = fabsf(ys[q] - my);
                    }
                    float dmx = median_bubble(xs, n), dmy = median_bubble(ys, n);
                    /* median_filtering :225-253 */
                    for (int i = 0; i < Nps; ++i) {
                        size_t c = (size_t)v * Nps + i;
                        if (!cvalid[c]) continue;
                        float devix = fabsf(cdx[c] - mx) / (dmx + epsilon);
                        float deviy = fabsf(cdy[c] - my) / (dmy + epsilon);
                        if (devix < cfg->insert_threshold && deviy < cfg->insert_threshold) {
                            nv[v] = 1;
                            nx[v] = cdx[c];
                            ny[v] = cdy[c];
                            break;
                        }
                    }
                }
            }
            free(xs);
            free(ys);
        }
        memcpy(fx, nx, sizeof(float) * Nt);
        memcpy(fy, ny, sizeof(float) * Nt);
        memcpy(fvalid, nv, Nt);
    }
    /* fill_blank_vecfield + _update :352-397, loop of :1514-1528 */
    int iters = 0;
    if (cfg->iffill) {
        uint8_t *filled = (uint8_t *)malloc(Nt);
        for (;;) {
            long nfill = 0;
            for (int v = 0; v < Nt; ++v) {
                filled[v] = 0;
                if (fvalid[v]) continue;
                int vy = v / Nxv, vx = v - vy * Nxv, cnt = 0;
                float sx = 0, sy = 0;
                for (int j = imax(0, vy - 1); j <= imin(Nyv - 1, vy + 1); j++)
                    for (int k = imax(0, vx - 1); k <= imin(Nxv - 1, vx + 1); k++) {
                        int id = j * Nxv + k;
                        if (fvalid[id]) {
                            cnt += 1;
                            sx += fx[id];
                            sy += fy[id];
                        }
                    }
                if (cnt > 0) {
                    nfill++;
                    filled[v] = 1;
                    fx[v] = sx / (float)cnt;
                    fy[v] = sy / (float)cnt;
                }
            }
            for (int v = 0; v < Nt; ++v)
                if (filled[v]) fvalid[v] = 1;
            iters++;
            if (nfill == 0) break;
        }
        free(filled);
    }
    if (fill_iters) *fill_iters = iters;
    /* organize_smooth_filter_data + smoothing_tophat :399-443, raster summation order */
    int hsx = (wx_sm - 1) / 2, hsy = (wy_sm - 1) / 2;
    for (int pass = 0; pass < cfg->Npass_smooth; ++pass) {
#pragma omp parallel for schedule(static)
        for (int v = 0; v < Nt; ++v) {
            int vy = v / Nxv, vx = v - vy * Nxv, n = 0;
            float sx = 0, sy = 0;
            for (int t = 0; t < Nts; ++t) {
                int ty = t / wx_sm, tx = t - ty * wx_sm;
                int x = vx - hsx + tx, y = vy - hsy + ty;
                if (x >= 0 && x <= Nxv - 1 && y >= 0 && y <= Nyv - 1) {
                    sx += fx[y * Nxv + x];
                    sy += fy[y * Nxv + x];
                    n++;
                }
            }
            nx[v] = sx / (float)n;
            ny[v] = sy / (float)n;
        }
        memcpy(fx, nx, sizeof(float) * Nt);
        memcpy(fy, ny, sizeof(float) * Nt);
    }
    free(nx);
    free(ny);
    free(nv);
    return OR_OK;
}

/* ------------------------------------------------------------------------- */
/* Whole pair, X/main.cpp:288-376                                              */
/* ------------------------------------------------------------------------- */
static int alloc_cands(or_candidates *c, int Nt, int Nps)
{
    c->dx = (float *)calloc((size_t)Nt * Nps, sizeof(float));
    c->dy = (float *)calloc((size_t)Nt * Nps, sizeof(float));
    c->valid = (uint8_t *)calloc((size_t)Nt * Nps, 1);
    c->count = (int32_t *)calloc((size_t)Nt, sizeof(int32_t));
    c->peak_index = (int32_t *)calloc((size_t)Nt * Nps, sizeof(int32_t));
    c->peak_value = (float *)calloc((size_t)Nt * Nps, sizeof(float));
    c->flags = (uint8_t *)calloc((size_t)Nt, 1);
    return (c->dx && c->dy && c->valid && c->count && c->peak_index && c->peak_value && c->flags) ? 0 : -1;
}

static void free_cands(or_candidates *c)
{
    free(c->dx);
    free(c->dy);
    free(c->valid);
    free(c->count);
    free(c->peak_index);
    free(c->peak_value);
    free(c->flags);
}

static void copy_cands(or_candidates *dst, const or_candidates *src, int Nt, int Nps)
{
    if (!dst) return;
    size_t n = (size_t)Nt * Nps;
    if (dst->dx) memcpy(dst->dx, src->dx, n * sizeof(float));
    if (dst->dy) memcpy(dst->dy, src->dy, n * sizeof(float));
    if (dst->valid) memcpy(dst->valid, src->valid, n);
    if (dst->count) memcpy(dst->count, src->count, (size_t)Nt * sizeof(int32_t));
    if (dst->peak_index) memcpy(dst->peak_index, src->peak_index, n * sizeof(int32_t));
    if (dst->peak_value) memcpy(dst->peak_value, src->peak_value, n * sizeof(float));
    if (dst->flags) memcpy(dst->flags, src->flags, (size_t)Nt);
}

int or_run_pair(const uint8_t *img1, const uint8_t *img2, const or_params *p, const or_valid_cfg *vc1,
                const or_valid_cfg *vc2, int direct, or_pair_out *out)
{
    or_geom g;
    int rc = or_geometry(p, &g);
    if (rc) return rc;
    int Nps = p->Npeak_save;
    int Nt1 = g.Nt_vec[0], Nt2 = g.Nt_vec[1];
    or_candidates c1, c2;
    memset(&c1, 0, sizeof(c1));
    memset(&c2, 0, sizeof(c2));
    float *fx1 = (float *)calloc(Nt1, sizeof(float)), *fy1 = (float *)calloc(Nt1, sizeof(float));
    uint8_t *fv1 = (uint8_t *)calloc(Nt1, 1);
    float *fx2 = (float *)calloc(Nt2, sizeof(float)), *fy2 = (float *)calloc(Nt2, sizeof(float));
    uint8_t *fv2 = (uint8_t *)calloc(Nt2, 1);
    size_t nd = (size_t)imax(g.Nx_aug[0] * g.Ny_aug[0], g.Nx_aug[1] * g.Ny_aug[1]);
    float *def = (float *)malloc(sizeof(float) * nd);
    long oob = 0;
    if (alloc_cands(&c1, Nt1, Nps) || alloc_cands(&c2, Nt2, Nps) || !def) {
        rc = OR_ERR_ARG;
        goto done;
    }
    or_valid_cfg v1 = *vc1;
    v1.iffill = 1; /* MedianFilter_Smoothing_p1 always fills (:1514) */
    for (int j = 0; j < p->Npass[0]; ++j) {
        if (j == 0) {
            /* Calc_cc_map_p1(0) zeroes the grid-1 predictor (:1287-1298) */
            memset(fx1, 0, sizeof(float) * Nt1);
            memset(fy1, 0, sizeof(float) * Nt1);
            rc = or_correlate_grid(img1, img2, NULL, p, &g, 0, fx1, fy1, direct, &c1);
        } else {
            oob += or_deform(img2, p, &g, 0, fx1, fy1, def);
            rc = or_correlate_grid(img1, img2, def, p, &g, 0, fx1, fy1, direct, &c1);
        }
        if (rc) goto done;
        or_validate(c1.dx, c1.dy, c1.valid, g.Nx_vec[0], g.Ny_vec[0], Nps, p->wx_med[0], p->wy_med[0], p->wx_sm[0],
                    p->wy_sm[0], &v1, fx1, fy1, fv1, NULL);
    }
    if (p->Npass[1] > 0) {
        or_upsample(p, &g, fx1, fy1, fx2, fy2);
        or_valid_cfg v2 = *vc2;
        v2.iffill = 1; /* main.cpp:319 passes iffill = 1 in the loop */
        for (int j = 0; j < p->Npass[1]; ++j) {
            oob += or_deform(img2, p, &g, 1, fx2, fy2, def);
            rc = or_correlate_grid(img1, img2, def, p, &g, 1, fx2, fy2, direct, &c2);
            if (rc) goto done;
            or_validate(c2.dx, c2.dy, c2.valid, g.Nx_vec[1], g.Ny_vec[1], Nps, p->wx_med[1], p->wy_med[1],
                        p->wx_sm[1], p->wy_sm[1], &v2, fx2, fy2, fv2, NULL);
        }
    }
    if (out) {
        copy_cands(&out->raw[0], &c1, Nt1, Nps);
        if (out->fx[0]) memcpy(out->fx[0], fx1, sizeof(float) * Nt1);
        if (out->fy[0]) memcpy(out->fy[0], fy1, sizeof(float) * Nt1);
        if (out->fvalid[0]) memcpy(out->fvalid[0], fv1, Nt1);
        if (p->Npass[1] > 0) {
            copy_cands(&out->raw[1], &c2, Nt2, Nps);
            if (out->fx[1]) memcpy(out->fx[1], fx2, sizeof(float) * Nt2);
            if (out->fy[1]) memcpy(out->fy[1], fy2, sizeof(float) * Nt2);
            if (out->fvalid[1]) memcpy(out->fvalid[1], fv2, Nt2);
            if (out->fx2_median || out->fy2_median || out->fvalid2_median) {
                /* main.cpp:363: median test only (smooth 0, fill 0) on the last raw grid-2 candidates */
                or_valid_cfg vm = *vc2;
                vm.Npass_smooth = 0;
                vm.iffill = 0;
                float *mx = (float *)malloc(sizeof(float) * Nt2), *my = (float *)malloc(sizeof(float) * Nt2);
                uint8_t *mv = (uint8_t *)malloc(Nt2);
                or_validate(c2.dx, c2.dy, c2.valid, g.Nx_vec[1], g.Ny_vec[1], Nps, p->wx_med[1], p->wy_med[1],
                            p->wx_sm[1], p->wy_sm[1], &vm, mx, my, mv, NULL);
                if (out->fx2_median) memcpy(out->fx2_median, mx, sizeof(float) * Nt2);
                if (out->fy2_median) memcpy(out->fy2_median, my, sizeof(float) * Nt2);
                if (out->fvalid2_median) memcpy(out->fvalid2_median, mv, Nt2);
                free(mx);
                free(my);
                free(mv);
            }
        }
        out->deform_oob = oob;
    }
done:
    free_cands(&c1);
    free_cands(&c2);
    free(fx1);
    free(fy1);
    free(fv1);
    free(fx2);
    free(fy2);
    free(fv2);
    free(def);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* Tecplot ASCII writer, X/xcorr2d_multi_grid.cu:1865-1973                     */
/* ------------------------------------------------------------------------- */
int or_write_tecplot(const char *path, int Nxv, int Nyv, int spx, int spy, int raw, int Nps, const float *dx,
                     const float *dy)
{
    FILE *f = fopen(path, "wb");
    if (!f) return OR_ERR_ARG;
    int Nt = Nxv * Nyv;
    fprintf(f, "TITLE = \"B00001\"\n");
    if (raw)
        fprintf(f, "VARIABLES = \"x\", \"y\", \"dx1\", \"dy1\", \"dx2\", \"dy2\", \"dx3\", \"dy3\", \"dx4\", \"dy4\"\n");
    else
        fprintf(f, "VARIABLES = \"x\", \"y\", \"displacement-x\", \"displacement-y\"\n");
    fprintf(f, "ZONE T=\"Frame 0\", I=%d, J=%d\n", Nxv, Nyv);
    long n = (long)Nt * (raw ? Nps : 1);
    for (int i = 0; i < Nt; ++i) {
        int j = i / Nxv, k = i - j * Nxv;
        fprintf(f, "%.2f\t%.2f", (double)(float)(spx / 2 + k * spx), (double)(float)(spy / 2 + j * spy));
        if (raw) {
            for (int c = 0; c < 4; ++c) {
                long q = (long)i * Nps + c;
                fprintf(f, "\t%.2f\t%.2f", q < n ? (double)dx[q] : 0.0, q < n ? (double)dy[q] : 0.0);
            }
        } else {
            fprintf(f, "\t%.2f\t%.2f", (double)dx[i], (double)dy[i]);
        }
        fprintf(f, "\n");
    }
    fclose(f);
    return OR_OK;
}
