/*
 * ref_capi.cu -- a C-ABI around the reference engine (class xcorr2d_multi,
 * X/xcorr2d_multi_grid.cuh:12-208, and class mhe_gpu, X/MHE7_4_gpu.h:7-40) compiled
 * unmodified for sm_100a.  TEST AND BASELINE INFRASTRUCTURE ONLY: it lets the tests
 * pin the oracle to the reference's real outputs and lets bench.py time the
 * reference arm.  It drives the public methods in the order of X/main.cpp:263-376.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>

#include "MHE7_4_gpu.h"
#include "xcorr2d_multi_grid.cuh"

/* Numeric lines 7..50 of the reference parameter file, in file order (X/main.cpp:103-146). */
struct ref_params {
    int device_id, ifmhe, mhe_ws;
    float mhe_thresh;
    int Nx, Ny;
    int ws_x1, ws_y1, spacing_x1, spacing_y1, Npass1;
    int ws_x2, ws_y2, spacing_x2, spacing_y2, Npass2;
    int Nsec_cc;
    int wx1_median, wy1_median, Npass1_median, minNneigh_p1;
    float residual_threshold_p1, insert_threshold_p1;
    int wx1_smooth, wy1_smooth, Npass1_smooth;
    int wx2_median, wy2_median, Npass2_median, minNneigh_p2;
    float residual_threshold_p2, insert_threshold_p2;
    int wx2_smooth, wy2_smooth, Npass2_smooth;
    float max_dispx_win_percent1, max_dispy_win_percent1, max_dispx_win_percent2, max_dispy_win_percent2;
    int Npeak_save;
    float dispx_lim1, dispx_lim2, dispy_lim1, dispy_lim2;
};

struct ref_engine {
    ref_params p;
    mhe_gpu mhe;
    xcorr2d_multi x;
    unsigned char *d_img_org = nullptr;
    bool mhe_ok = false, x_ok = false;
};

extern "C" {

int ref_create(const ref_params *p, ref_engine **out)
{
    if (!p || !out) return -1;
    *out = nullptr;
    if (cudaSetDevice(p->device_id) != cudaSuccess) return -4;
    ref_engine *e = new (std::nothrow) ref_engine();
    if (!e) return -5;
    e->p = *p;
    /* X/main.cpp:67-72 launch configuration */
    e->mhe.setupgridblockdim(10000, 1, 1, 512, 1, 1);
    e->x.setupgridblockdim(10000, 1, 1, 512, 1, 1);
    if (!e->mhe.init(p->Nx, p->Ny, p->mhe_ws, p->mhe_thresh)) {
        e->mhe.freemem();
        delete e;
        return -2;
    }
    e->mhe_ok = true;
    if (!e->x.init(p->Nx, p->Ny, p->Nsec_cc, p->ws_x1, p->ws_y1, p->spacing_x1, p->spacing_y1, p->Npass1, p->ws_x2,
                   p->ws_y2, p->spacing_x2, p->spacing_y2, p->Npass2, p->wx1_median, p->wy1_median, p->wx2_median,
                   p->wy2_median, p->wx1_smooth, p->wy1_smooth, p->wx2_smooth, p->wy2_smooth, p->Npeak_save,
                   p->max_dispx_win_percent1, p->max_dispy_win_percent1, p->max_dispx_win_percent2,
                   p->max_dispy_win_percent2, p->dispx_lim1, p->dispx_lim2, p->dispy_lim1, p->dispy_lim2)) {
        e->x.freemem();
        e->mhe.freemem();
        delete e;
        return -2;
    }
    e->x_ok = true;
    if (cudaMalloc((void **)&e->d_img_org, (size_t)p->Nx * p->Ny) != cudaSuccess) {
        e->x.freemem();
        e->mhe.freemem();
        delete e;
        return -5;
    }
    *out = e;
    return 0;
}

void ref_destroy(ref_engine *e)
{
    if (!e) return;
    cudaFree(e->d_img_org);
    if (e->mhe_ok) e->mhe.freemem();
    if (e->x_ok) e->x.freemem();
    delete e;
}

/* One frame through mhe_gpu::processsing (X/main.cpp:268-274): host in -> host out. */
int ref_mhe(ref_engine *e, const uint8_t *in, uint8_t *out)
{
    size_t n = (size_t)e->p.Nx * e->p.Ny;
    cudaMemcpy(e->d_img_org, in, n, cudaMemcpyHostToDevice);
    if (!e->mhe.processsing(e->d_img_org)) return -4;
    cudaMemcpy(out, e->mhe.d_enhanced, n, cudaMemcpyDeviceToHost);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

static void copy_field(float *dst, const float *src, int n)
{
    if (dst) cudaMemcpy(dst, src, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
}

/* The per-pair body of X/main.cpp:263-326: frames into the engine's pinned buffers,
 * optional MHE round trip, prep, grid-1 and grid-2 pass loops.  pred1x/y, pred2x/y
 * (optional) receive the filtered field each grid's last pass starts from (its
 * predictor and deformation field). */
int ref_run_pair_recording(ref_engine *e, const uint8_t *f1, const uint8_t *f2, float *pred1x, float *pred1y,
                           float *pred2x, float *pred2y);

int ref_run_pair(ref_engine *e, const uint8_t *f1, const uint8_t *f2)
{
    return ref_run_pair_recording(e, f1, f2, nullptr, nullptr, nullptr, nullptr);
}

int ref_run_pair_recording(ref_engine *e, const uint8_t *f1, const uint8_t *f2, float *pred1x, float *pred1y,
                           float *pred2x, float *pred2y)
{
    xcorr2d_multi &x = e->x;
    size_t n = (size_t)e->p.Nx * e->p.Ny;
    std::memcpy(x.h_img1_org, f1, n);
    std::memcpy(x.h_img2_org, f2, n);
    if (e->p.ifmhe == 1) {
        cudaMemcpy(e->d_img_org, x.h_img1_org, n, cudaMemcpyHostToDevice);
        if (!e->mhe.processsing(e->d_img_org)) return -4;
        cudaMemcpy(x.h_img1_org, e->mhe.d_enhanced, n, cudaMemcpyDeviceToHost);
        cudaMemcpy(e->d_img_org, x.h_img2_org, n, cudaMemcpyHostToDevice);
        if (!e->mhe.processsing(e->d_img_org)) return -4;
        cudaMemcpy(x.h_img2_org, e->mhe.d_enhanced, n, cudaMemcpyDeviceToHost);
    }
    x.prep_img_data();
    for (int j = 0; j < x.Npass1; j++) {
        if (j > 0) x.extend_filtered_vecfield_p1();
        if (j == x.Npass1 - 1 && j > 0) {
            copy_field(pred1x, x.d_disp_x_filter_p1, x.Nt1_vec);
            copy_field(pred1y, x.d_disp_y_filter_p1, x.Nt1_vec);
        }
        if (!x.Calc_cc_map_p1(j)) return -4;
        if (!x.MedianFilter_Smoothing_p1(e->p.Npass1_median, e->p.minNneigh_p1, e->p.residual_threshold_p1,
                                         e->p.insert_threshold_p1, e->p.Npass1_smooth))
            return -4;
    }
    if (x.Npass2 > 0) {
        x.extend_filtered_vecfield_p1();
        if (!x.Upsampling_vector_field()) return -4;
        for (int j = 0; j < x.Npass2; j++) {
            x.extend_filtered_vecfield_p2();
            if (j == x.Npass2 - 1) {
                copy_field(pred2x, x.d_disp_x_filter_p2, x.Nt2_vec);
                copy_field(pred2y, x.d_disp_y_filter_p2, x.Nt2_vec);
            }
            if (!x.Calc_cc_map_p2()) return -4;
            if (!x.MedianFilter_Smoothing_p2(e->p.Npass2_median, e->p.minNneigh_p2, e->p.residual_threshold_p2,
                                             e->p.insert_threshold_p2, e->p.Npass2_smooth, 1))
                return -4;
        }
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

/* X/main.cpp:363: median test only (no smoothing, no fill) on the grid-2 candidates. */
int ref_median_only(ref_engine *e)
{
    if (!e->x.MedianFilter_Smoothing_p2(e->p.Npass2_median, e->p.minNneigh_p2, e->p.residual_threshold_p2,
                                        e->p.insert_threshold_p2, 0, 0))
        return -4;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

/* Host -> the reference's raw candidate arrays of a grid ([Nt*Npeak_save] each), so that
 * its validation can be run on candidates from elsewhere (the engine's). */
int ref_set_raw(ref_engine *e, int grid, const float *dx, const float *dy, const uint8_t *valid)
{
    xcorr2d_multi &x = e->x;
    size_t n = (size_t)(grid ? x.Nt2_vec : x.Nt1_vec) * x.Npeak_save;
    cudaMemcpy(grid ? x.d_disp_x_p2 : x.d_disp_x_p1, dx, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(grid ? x.d_disp_y_p2 : x.d_disp_y_p1, dy, n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(grid ? (void *)x.d_valid_p2 : (void *)x.d_valid_p1, valid, n, cudaMemcpyHostToDevice);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

/* MedianFilter_Smoothing_p1 / _p2 (X/xcorr2d_multi_grid.cu:1451, :1766) on the current raw
 * candidates of a grid; grid 1 always fills (the reference's p1 form has no switch). */
int ref_validate(ref_engine *e, int grid, int Npass_median, int minN, float rthr, float ithr, int Npass_smooth,
                 int iffill)
{
    bool ok = grid ? e->x.MedianFilter_Smoothing_p2(Npass_median, minN, rthr, ithr, Npass_smooth, iffill)
                   : e->x.MedianFilter_Smoothing_p1(Npass_median, minN, rthr, ithr, Npass_smooth);
    if (!ok) return -4;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -4;
}

/* Device state -> host.  grid 0/1; raw candidates [Nt*Npeak_save] and the filtered field [Nt]. */
int ref_get_raw(ref_engine *e, int grid, float *dx, float *dy, uint8_t *valid)
{
    xcorr2d_multi &x = e->x;
    size_t n = (size_t)(grid ? x.Nt2_vec : x.Nt1_vec) * x.Npeak_save;
    if (dx) cudaMemcpy(dx, grid ? x.d_disp_x_p2 : x.d_disp_x_p1, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (dy) cudaMemcpy(dy, grid ? x.d_disp_y_p2 : x.d_disp_y_p1, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (valid) cudaMemcpy(valid, grid ? x.d_valid_p2 : x.d_valid_p1, n, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

int ref_get_filtered(ref_engine *e, int grid, float *dx, float *dy, uint8_t *valid)
{
    xcorr2d_multi &x = e->x;
    size_t n = (size_t)(grid ? x.Nt2_vec : x.Nt1_vec);
    if (dx) cudaMemcpy(dx, grid ? x.d_disp_x_filter_p2 : x.d_disp_x_filter_p1, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (dy) cudaMemcpy(dy, grid ? x.d_disp_y_filter_p2 : x.d_disp_y_filter_p1, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (valid) cudaMemcpy(valid, grid ? x.d_valid_filter_p2 : x.d_valid_filter_p1, n, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

/* Peak bookkeeping of the last section of the last pass of a grid (valid for all
 * windows when Nsec_cc = 1): local-maximum counts, the chosen cc-plane indices
 * (in-window, shifted) and their values. */
int ref_get_peaks(ref_engine *e, int grid, int32_t *count, int32_t *pidx, float *pval)
{
    xcorr2d_multi &x = e->x;
    int Neach = grid ? x.Neach2 : x.Neach1, Npeak = grid ? x.Npeak2 : x.Npeak1, Ntws = grid ? x.Nt_ws2 : x.Nt_ws1;
    int Nps = x.Npeak_save;
    size_t nslot = (size_t)Neach * Npeak, n4 = (size_t)Neach * Nps;
    int32_t *h_loc = new int32_t[nslot];
    int32_t *h_four = new int32_t[n4];
    float *h_val = new float[n4];
    cudaMemcpy(h_loc, grid ? x.d_index_local_tot2 : x.d_index_local_tot1, nslot * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(h_four, grid ? x.d_index_four_peaks_p2 : x.d_index_four_peaks_p1, n4 * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(h_val, grid ? x.d_max_four_peaks_p2 : x.d_max_four_peaks_p1, n4 * 4, cudaMemcpyDeviceToHost);
    if (count) cudaMemcpy(count, grid ? x.d_posi_count_p2 : x.d_posi_count_p1, (size_t)Neach * 4, cudaMemcpyDeviceToHost);
    for (size_t t = 0; t < n4; ++t) {
        int w = (int)(t / Nps);
        float v = h_val[t];
        int li = h_loc[h_four[t]] - w * Ntws;
        if (pidx) pidx[t] = (v > 0) ? li : -1;
        if (pval) pval[t] = (v > 0) ? v : 0.f;
    }
    delete[] h_loc;
    delete[] h_four;
    delete[] h_val;
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

/* Shifted correlation planes left in d_cc by the last section of the last pass. */
int ref_get_cc(ref_engine *e, int grid, int first, int nwin, float *out)
{
    xcorr2d_multi &x = e->x;
    int Ntws = grid ? x.Nt_ws2 : x.Nt_ws1;
    cudaMemcpy(out, x.d_cc + (size_t)first * Ntws, (size_t)nwin * Ntws * 4, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

/* Deformed frame 2 of the last pass of a grid ([Ny_aug][Nx_aug] floats). */
int ref_get_deformed(ref_engine *e, int grid, float *out)
{
    xcorr2d_multi &x = e->x;
    size_t n = grid ? (size_t)x.Nt2_aug : (size_t)x.Nt1_aug;
    cudaMemcpy(out, grid ? x.d_img_deform_p2 : x.d_img_deform_p1, n * 4, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

int ref_write_tecplot(ref_engine *e, const char *path, int selection)
{
    return e->x.write_vec_data_general(CString(path), selection) ? 0 : -6;
}

}  // extern "C"
