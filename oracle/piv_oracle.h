/*
 * piv_oracle.h -- CPU restatement of the multi-grid PIV correlation path of
 * xinzhixue/PIV_xcorr2d_V1.0 (xcorr2d_V1.0/xcorr2d_multi_grid.cu, MHE7_4_gpu.cu).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine in
 * piv_xcorr2d_v1.0_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product path never calls it.
 *
 * Precision contract:
 *   - geometry, candidate search, top-N rounds, validation decisions, MHE: integer
 *     or FP32 arithmetic written exactly as the reference writes it (no FMA
 *     contraction: gcc on x86-64 without -mfma), so decisions are reproducible;
 *   - correlation planes: FP64 (own mixed-radix FFT, or an exact direct sum);
 *   - 3-point Gaussian fit: FP64.
 * Every function cites the reference file:line it restates (paths relative to the
 * reference project root, X/ = xcorr2d_V1.0/).
 */
#ifndef PIV_ORACLE_H
#define PIV_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Numeric part of the 50-line parameter file (X/main.cpp:97-146), grid g in {0,1}. */
typedef struct {
    int Nx, Ny, Nsec_cc;
    int ws_x[2], ws_y[2], sp_x[2], sp_y[2], Npass[2];
    int wx_med[2], wy_med[2], wx_sm[2], wy_sm[2];
    int Npeak_save;
    float pct_x[2], pct_y[2];
    float lim_x1, lim_x2, lim_y1, lim_y2;
} or_params;

/* Derived geometry of xcorr2d_multi::init (X/xcorr2d_multi_grid.cu:751-894). */
typedef struct {
    int border_x[2], border_y[2];
    int hfws_x[2], hfws_y[2];
    int Npeak[2];
    int Nx_vec[2], Ny_vec[2], Nt_vec[2];
    int Neach[2], Nlast[2], Nsec[2];
    int Nx_left[2], Nx_right[2], Ny_left[2], Ny_right[2];
    int Nx_aug[2], Ny_aug[2], Nx_aug_ex[2], Ny_aug_ex[2];
} or_geom;

/* Validation settings of MedianFilter_Smoothing_p{1,2} (X/xcorr2d_multi_grid.cu:1451,1766). */
typedef struct {
    int Npass_median, minNneigh;
    float insert_threshold;
    int Npass_smooth, iffill;
} or_valid_cfg;

/* Per-grid candidate outputs of one correlation pass. */
typedef struct {
    float *dx, *dy;        /* [Nt_vec * Npeak_save] */
    uint8_t *valid;        /* [Nt_vec * Npeak_save] */
    int32_t *count;        /* [Nt_vec]  local-maximum count (d_posi_count) */
    int32_t *peak_index;   /* [Nt_vec * Npeak_save] shifted in-window index j*ws_x+i, -1 if empty */
    float *peak_value;     /* [Nt_vec * Npeak_save] */
    uint8_t *flags;        /* [Nt_vec] bit0: slot overflow (count > Npeak), bit1: exact tie among top N+1 */
} or_candidates;

/* Status codes (same meaning as the engine's). */
#define OR_OK 0
#define OR_ERR_ARG (-1)
#define OR_ERR_GEOMETRY (-2)

int or_geometry(const or_params *p, or_geom *g);

/* MHE7_4_gpu.cu:149-253 -- integer, bit-exact. out must be Nx*Ny (pixels outside the
 * centred crop are written 0, like the zero-initialised d_enhanced). */
int or_mhe(const uint8_t *in, int Nx, int Ny, int ws, float thresh, uint8_t *out);

/* FP64 circular cross-correlation magnitude of one window pair, fftshifted
 * (X/xcorr2d_multi_grid.cu:519-583 semantics).  direct!=0 uses the exact O(N^2) sum. */
void or_xcorr_plane(const double *w1, const double *w2, int wsx, int wsy, double *cc_shifted, int direct);

/* Candidate search + top-N rounds + Gaussian fit of one window from a given plane
 * (X/xcorr2d_multi_grid.cu:585-606, 32-172, 298-350, 457-471). */
void or_peaks_window(const double *cc, int wsx, int wsy, int bx, int by, int Npeak, int Npeak_save,
                     float pred_x, float pred_y, float lx1, float lx2, float ly1, float ly2,
                     float *dx, float *dy, uint8_t *valid, int32_t *count, int32_t *pidx, float *pval,
                     uint8_t *flags);

/* Window deformation of frame 2 on grid g (X/xcorr2d_multi_grid.cu:608-652, 1300, 1624)
 * from the filtered field (extended by edge replication, :1547-1618).  out is
 * Nx_aug*Ny_aug floats.  Returns the number of bilinear taps that fell outside the
 * reference's zero-padded aug_ex buffer (the reference reads unchecked there). */
long or_deform(const uint8_t *img2, const or_params *p, const or_geom *g, int grid,
               const float *fx, const float *fy, float *out);

/* Bilinear upsampling of the grid-1 field onto grid 2 (X/xcorr2d_multi_grid.cu:675-704, 1578). */
void or_upsample(const or_params *p, const or_geom *g, const float *fx1, const float *fy1,
                 float *fx2, float *fy2);

/* One correlation pass of grid g (Calc_cc_map_p1/p2, X/xcorr2d_multi_grid.cu:1284-1449, 1620-1764).
 * deformed: NULL for the undeformed first grid-1 pass, else the deformed frame 2.
 * pred_x/pred_y: the predictor field (filtered field before the pass). */
int or_correlate_grid(const uint8_t *img1, const uint8_t *img2, const float *deformed,
                      const or_params *p, const or_geom *g, int grid,
                      const float *pred_x, const float *pred_y, int direct, or_candidates *out);

/* Same, but from caller-provided shifted planes (e.g. the engine's FP32 planes):
 * cc is [Nt_vec][ws_y][ws_x] floats. */
int or_peaks_from_planes(const float *cc, const or_params *p, const or_geom *g, int grid,
                         const float *pred_x, const float *pred_y, or_candidates *out);

/* Normalized median test + candidate replacement, hole fill, top-hat smoothing
 * (X/xcorr2d_multi_grid.cu:174-296, 352-443, 484-495, 1451-1545, 1766-1863), FP32.
 * fx/fy/fvalid: in = ignored (prepared from candidate 0), out = filtered field. */
int or_validate(const float *cdx, const float *cdy, const uint8_t *cvalid, int Nx_vec, int Ny_vec,
                int Npeak_save, int wx_med, int wy_med, int wx_sm, int wy_sm, const or_valid_cfg *cfg,
                float *fx, float *fy, uint8_t *fvalid, int *fill_iters);

/* Whole pair (X/main.cpp:288-376 order).  Outputs may be NULL.
 * raw[g] candidates of the last pass of grid g; filt[g] filtered field after the
 * loop of grid g; filt2_median: grid-2 median-only field (smooth 0, fill 0). */
typedef struct {
    or_candidates raw[2];
    float *fx[2], *fy[2];
    uint8_t *fvalid[2];
    float *fx2_median, *fy2_median;
    uint8_t *fvalid2_median;
    long deform_oob;      /* out-of-aug_ex taps over all deformations */
} or_pair_out;

int or_run_pair(const uint8_t *img1, const uint8_t *img2, const or_params *p,
                const or_valid_cfg *vc1, const or_valid_cfg *vc2, int direct, or_pair_out *out);

/* write_vec_data_general (X/xcorr2d_multi_grid.cu:1865-1973) for one field. raw!=0:
 * 4 candidate columns from a [Nt*Npeak_save] array; else one (dx, dy) column. */
int or_write_tecplot(const char *path, int Nx_vec, int Ny_vec, int sp_x, int sp_y, int raw,
                     int Npeak_save, const float *dx, const float *dy);

int or_num_threads(void);
void or_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
