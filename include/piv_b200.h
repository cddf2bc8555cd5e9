/*
 * piv_b200.h -- C-ABI of the B200-native multi-grid PIV correlation engine.
 *
 * A drop-in for the engine surface of xinzhixue/PIV_xcorr2d_V1.0 (paths below are
 * relative to that project; X/ = xcorr2d_V1.0/):
 *   class xcorr2d_multi  X/xcorr2d_multi_grid.cuh:12-208
 *   class mhe_gpu        X/MHE7_4_gpu.h:7-40
 * driven in the order of X/main.cpp:248-380.  Every entry point returns an int
 * status (PIV_OK = 0, negative = error); piv_last_error() gives the message the
 * reference would have printed.  One host thread per engine; calls on one engine
 * are not re-entrant.  All device work is queued on the engine's own CUDA stream.
 * Plain pointers and sizes only: no CUDA or C++ types cross this boundary.
 */
#ifndef PIV_B200_H
#define PIV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIV_B200_ABI_VERSION 1

/* Status codes. */
#define PIV_OK 0
#define PIV_ERR_ARG (-1)          /* invalid argument or parameter value */
#define PIV_ERR_GEOMETRY (-2)     /* rejected by the window-size checks of xcorr2d_multi::init */
#define PIV_ERR_UNSUPPORTED (-3)  /* valid for the reference but not built into this engine */
#define PIV_ERR_CUDA (-4)         /* a CUDA runtime call failed */
#define PIV_ERR_ALLOC (-5)        /* device or pinned allocation failed */
#define PIV_ERR_IO (-6)           /* file could not be opened / parsed */
#define PIV_ERR_STATE (-7)        /* call out of order (e.g. a pass before piv_prep) */
#define PIV_ERR_DEVICE (-8)       /* a kernel reported an error status (iteration cap hit) */

typedef struct piv_engine piv_engine;
typedef struct piv_mhe piv_mhe;

/* Numeric lines 7..50 of the reference's 50-line parameter file, in file order
 * (X/main.cpp:103-146, X/Parameter_Instructions_xcorr2d_V1.0.txt:38-136). */
typedef struct piv_params {
    int device_id;                 /* 7  */
    int if_mhe;                    /* 8  */
    int mhe_ws;                    /* 9  */
    float mhe_thresh;              /* 10 */
    int Nx, Ny;                    /* 11, 12 */
    int ws_x1, ws_y1;              /* 13, 14 */
    int spacing_x1, spacing_y1;    /* 15, 16 */
    int Npass1;                    /* 17 */
    int ws_x2, ws_y2;              /* 18, 19 */
    int spacing_x2, spacing_y2;    /* 20, 21 */
    int Npass2;                    /* 22 */
    int Nsec_cc;                   /* 23 */
    int wx1_median, wy1_median;    /* 24, 25 */
    int Npass1_median;             /* 26 */
    int minNneigh_p1;              /* 27 */
    float residual_threshold_p1;   /* 28 (read, unused: as in the reference) */
    float insert_threshold_p1;     /* 29 */
    int wx1_smooth, wy1_smooth;    /* 30, 31 */
    int Npass1_smooth;             /* 32 */
    int wx2_median, wy2_median;    /* 33, 34 */
    int Npass2_median;             /* 35 */
    int minNneigh_p2;              /* 36 */
    float residual_threshold_p2;   /* 37 (read, unused) */
    float insert_threshold_p2;     /* 38 */
    int wx2_smooth, wy2_smooth;    /* 39, 40 */
    int Npass2_smooth;             /* 41 */
    float max_dispx_win_percent1;  /* 42 */
    float max_dispy_win_percent1;  /* 43 */
    float max_dispx_win_percent2;  /* 44 */
    float max_dispy_win_percent2;  /* 45 */
    int Npeak_save;                /* 46 */
    float dispx_lim1, dispx_lim2;  /* 47, 48 */
    float dispy_lim1, dispy_lim2;  /* 49, 50 */
} piv_params;

/* Lines 1..6 of the parameter file (file-name prefixes/suffixes, pair list, output folder). */
typedef struct piv_paths {
    char prefix_f1[1024], suffix_f1[256];
    char prefix_f2[1024], suffix_f2[256];
    char dir_index[1024];
    char folder_result[1024];
} piv_paths;

/* Derived geometry, bit-identical to xcorr2d_multi::init (X/xcorr2d_multi_grid.cu:751-894). */
typedef struct piv_geometry {
    int border_x[2], border_y[2];
    int hfws_x[2], hfws_y[2];
    int Npeak[2];
    int Nx_vec[2], Ny_vec[2], Nt_vec[2];
    int Neach[2], Nlast[2], Nsec[2];
    int Nx_left[2], Nx_right[2], Ny_left[2], Ny_right[2];
    int Nx_aug[2], Ny_aug[2], Nx_aug_ex[2], Ny_aug_ex[2];
} piv_geometry;

/* ---- parameter file, geometry ------------------------------------------------ */

/* Parses the 50-line positional parameter file (X/main.cpp:93-158).  Returns
 * PIV_ERR_IO if it cannot be opened and PIV_ERR_ARG if a line is missing
 * ("Parameter missing in Parameter.dat!").  paths may be NULL. */
int piv_params_read(const char *path, piv_params *out, piv_paths *paths);

/* Geometry without allocating an engine (same checks as xcorr2d_multi::init). */
int piv_geometry_compute(const piv_params *p, piv_geometry *out);

/* Message for a status code without an engine handle. */
const char *piv_status_string(int status);

/* ---- engine: xcorr2d_multi + mhe_gpu --------------------------------------- */

/* mhe_gpu::init + xcorr2d_multi::init (X/MHE7_4_gpu.cu:149, X/xcorr2d_multi_grid.cu:716):
 * selects p->device_id, validates the geometry, allocates all device buffers and
 * the pinned host frame buffers, creates the engine stream.  Every window shape the
 * reference accepts runs (ws_x, ws_y multiples of 4 in [4, 1024]): the fused register-FFT
 * kernels cover 8..64 px in 13 shapes with up to 8 saved peaks, a generic-size kernel
 * every other shape and Npeak_save up to 1024 (PIV_ERR_ARG above).  A pair's results do
 * not depend on the tile variant, Nsec_cc, or whether it runs alone or in a batch.
 * Fault injection (off unless set in the environment): PIV_TEST_FAIL_ALLOC=k fails the
 * engine's k-th device allocation (PIV_ERR_ALLOC, everything freed); PIV_TEST_FILL_CAP=n
 * caps the hole fill at n iterations (piv_synchronize then returns PIV_ERR_DEVICE). */
int piv_create(const piv_params *p, piv_engine **out);

/* xcorr2d_multi::freemem + mhe_gpu::freemem. */
int piv_destroy(piv_engine *e);

/* Message of the last failing call on this engine (empty if none). */
const char *piv_last_error(const piv_engine *e);

int piv_get_geometry(const piv_engine *e, piv_geometry *out);

/* The parameters the engine was created with. */
int piv_get_params(const piv_engine *e, piv_params *out);

/* Engine-owned pinned host frame buffers, Nx*Ny bytes each, row-major without
 * padding (the public h_img1_org / h_img2_org, X/xcorr2d_multi_grid.cuh:104-105). */
int piv_host_images(piv_engine *e, uint8_t **f1, uint8_t **f2);

/* Copies two host frames (Nx*Ny bytes each, rows of `pitch` bytes; pitch 0 = Nx)
 * into the engine's pinned buffers. */
int piv_set_images(piv_engine *e, const uint8_t *f1, const uint8_t *f2, size_t pitch);

/* Uses two frames already resident in device memory (Nx*Ny bytes each, row-major)
 * instead of the pinned host buffers for the next piv_prep. The pointers must stay
 * valid until piv_prep has run. NULL, NULL switches back to the host buffers. */
int piv_set_device_images(piv_engine *e, const uint8_t *d_f1, const uint8_t *d_f2);

/* Pipelined input (no counterpart in the reference, whose main loop uploads a pair and
 * then computes it): queues the upload of the next pair's frames (Nx*Ny bytes each,
 * row-major host memory; pinned memory lets the copy overlap) into one of two device
 * input slots on the engine's copy stream and returns at once.  The next piv_run_pair
 * computes that pair, after the upload, while the caller may already queue the pair
 * after it: the upload of pair k+1 then overlaps the computation of pair k.  A slot is
 * refilled only after the pair that read it has finished.  PIV_ERR_STATE if a queued
 * pair has not been run yet; piv_set_images / piv_set_device_images discard a queued
 * pair.  The host buffers must stay valid until the upload is done (piv_run_pair of
 * that pair returned and its results were read, or piv_synchronize). */
int piv_queue_images(piv_engine *e, const uint8_t *f1, const uint8_t *f2);

/* Page-locked host memory for the frames a caller feeds to piv_queue_images (uploads
 * from it overlap the computation); release with piv_host_free. */
int piv_host_alloc(size_t bytes, void **ptr);
int piv_host_free(void *ptr);

/* prep_img_data (X/xcorr2d_multi_grid.cu:1271-1282) fused with the optional MHE of
 * both frames (X/main.cpp:267-283, mhe_gpu::processsing): uploads the frames (one
 * asynchronous copy per frame from the pinned buffers, or a device-to-device copy),
 * enhances them on the device when if_mhe == 1 and places them into the padded
 * frame buffers.  No host round trip. */
int piv_prep(piv_engine *e);

/* Calc_cc_map_p1(idx_pass) (X/xcorr2d_multi_grid.cu:1284-1449), including the
 * extend_filtered_vecfield_p1 that precedes it for idx_pass > 0. */
int piv_pass_grid1(piv_engine *e, int idx_pass);

/* MedianFilter_Smoothing_p1 (X/xcorr2d_multi_grid.cu:1451-1545). */
int piv_validate_grid1(piv_engine *e, int Npass_median, int minNneigh, float residual_threshold,
                       float insert_threshold, int Npass_smooth);

/* extend_filtered_vecfield_p1 + Upsampling_vector_field (X/xcorr2d_multi_grid.cu:1547-1587). */
int piv_upsample(piv_engine *e);

/* extend_filtered_vecfield_p2 + Calc_cc_map_p2 (X/xcorr2d_multi_grid.cu:1589-1764). */
int piv_pass_grid2(piv_engine *e);

/* MedianFilter_Smoothing_p2 (X/xcorr2d_multi_grid.cu:1766-1863). */
int piv_validate_grid2(piv_engine *e, int Npass_median, int minNneigh, float residual_threshold,
                       float insert_threshold, int Npass_smooth, int iffill);

/* The per-pair body of X/main.cpp:288-326 with the engine's parameters: prep (+MHE),
 * the grid-1 passes and validations, upsampling, the grid-2 passes and validations.
 * Replayed from a CUDA graph captured on the first call.  Asynchronous: follow with
 * piv_synchronize or a piv_get_* call. */
int piv_run_pair(piv_engine *e);

/* Waits for the engine stream and reports any device-side error status. */
int piv_synchronize(piv_engine *e);

/* Field readback (synchronises).  selection as write_vec_data_general:
 *   0 grid-1 raw candidates, 1 grid-1 filtered, 2 grid-2 raw candidates, 3 grid-2 filtered.
 * For raw selections dx, dy, valid hold Nt_vec*Npeak_save values (candidate-major per
 * vector); for filtered ones Nt_vec.  x, y receive the grid coordinates (Nt_vec).
 * Any output pointer may be NULL. */
int piv_get_field(piv_engine *e, int selection, float *x, float *y, float *dx, float *dy, uint8_t *valid);

/* Asynchronous readback (no counterpart in the reference, which reads each field back
 * before the next pair starts).  piv_field_async queues, behind the work already queued on
 * the engine stream, the copy of a selection (0..3, as piv_get_field) into one of two
 * engine-owned pinned slots, together with the device status word of that work, and
 * returns at once with a ticket.  piv_field_wait waits for that copy, reports a device
 * error of its pair (PIV_ERR_DEVICE), and copies the arrays out (any pointer may be NULL).
 * A caller thus keeps the next pair queued while it reads the previous one:
 *   queue(0); for k: run(k); t[k] = field_async(k); queue(k+1); field_wait(t[k-1]).
 * At most two readbacks are pending (PIV_ERR_STATE otherwise). */
int piv_field_async(piv_engine *e, int selection, int *ticket);
int piv_field_wait(piv_engine *e, int ticket, float *x, float *y, float *dx, float *dy, uint8_t *valid);

/* write_vec_data_general (X/xcorr2d_multi_grid.cu:1865-1973): Tecplot ASCII file. */
int piv_write_tecplot(piv_engine *e, const char *path, int selection);

/* The Tecplot writer on caller arrays (raw != 0: dx, dy hold Nt_vec*Npeak_save values and
 * four candidate columns are printed, as the reference always does). */
int piv_tecplot_write_arrays(const char *path, int Nx_vec, int Ny_vec, int spacing_x, int spacing_y, int raw,
                             int Npeak_save, const float *dx, const float *dy);

/* Binary sidecar (no counterpart in the reference): a float32 array of `ndim` dimensions
 * as a NumPy .npy file (format 1.0, little-endian, C order). */
int piv_npy_write_f32(const char *path, const float *data, int ndim, const int *shape);

/* Baseline TIFF (CImageIO, X/ImageIOPkg.cpp:124-428 and :641): uncompressed, 8-bit grey,
 * strip-organised, either byte order.  piv_tiff_read8 needs the file to be exactly Nx x Ny
 * (PIV_ERR_ARG otherwise, PIV_ERR_UNSUPPORTED for other bit depths or compression). */
int piv_tiff_info(const char *path, int *Nx, int *Ny, int *bits);
int piv_tiff_read8(const char *path, uint8_t *out, int Nx, int Ny);
int piv_tiff_write8(const char *path, const uint8_t *img, int Nx, int Ny);

/* Output file name of X/main.cpp:327-369 for pair index `idx`:
 * kind 0 grid-1 raw, 1 grid-1 filtered, 2 grid-2 raw, 3 grid-2 filtered, 4 grid-2 median-only. */
int piv_output_name(const piv_params *p, const char *folder, int idx, int kind, char *out, size_t cap);

/* ---- parity / diagnostics taps ---------------------------------------------- */

/* Peak bookkeeping of the last pass of a grid: local-maximum count per vector
 * (d_posi_count), chosen peak index in the shifted window (j*ws_x+i, -1 = none) and
 * value, Npeak_save per vector.  Any pointer may be NULL. */
int piv_get_peaks(piv_engine *e, int grid, int32_t *count, int32_t *peak_index, float *peak_value);

/* Replaces the filtered field of a grid (the predictor of the next pass). */
int piv_set_field(piv_engine *e, int grid, const float *dx, const float *dy, const uint8_t *valid);

/* Replaces the raw candidates of a grid (input of the next validation). */
int piv_set_candidates(piv_engine *e, int grid, const float *dx, const float *dy, const uint8_t *valid);

/* Frames as placed by piv_prep (after MHE), Nx*Ny each. */
int piv_get_frames(piv_engine *e, uint8_t *f1, uint8_t *f2);

/* Deformed frame 2 of the last pass of a grid, [Ny_aug][Nx_aug] floats. */
int piv_get_deformed(piv_engine *e, int grid, float *out);

/* Re-runs the correlation of the last pass of `grid` for windows [first, first+n) and
 * returns their shifted correlation planes ([n][ws_y][ws_x] floats).  Candidates and
 * fields are not touched. */
int piv_debug_cc_planes(piv_engine *e, int grid, int first, int n, float *out);

/* Device time of the kernels of the last piv_run_pair, by stage (ms): [0] prep+MHE,
 * [1] deformation, [2] correlation, [3] validation, [4] total. Needs PIV_TIMING=1 in the
 * environment at piv_create; otherwise returns PIV_ERR_STATE. */
int piv_stage_times(piv_engine *e, float *ms5);

/* ---- measurement ------------------------------------------------------------ */

/* The engine's CUDA stream (a cudaStream_t), for callers that order their own work
 * (events, copies) against the engine. */
int piv_get_stream(const piv_engine *e, void **stream);

/* The fused correlation kernel configuration the autotuner chose for a grid at
 * piv_create (windows per CTA, threads per CTA) and its measured time per launch on
 * the tuning input (0 if not tuned; PIV_AUTOTUNE=0/off/false/no keeps the defaults,
 * PIV_XCORR_VARIANT=v1,v2 fixes them).  The variants compute the same bits, so the
 * choice changes speed only.  32x32 windows have one more variant after their row-major
 * ones (index 5): two horizontally adjacent window pairs of two consecutive window rows per
 * CTA, sharing their overlapping pixel rows' gathers and row transforms, reported as
 * (4, 128).  A grid on the generic-size kernel reports (1, 256, 0). */
int piv_xcorr_config(const piv_engine *e, int grid, int *windows_per_cta, int *threads_per_cta, float *tuned_ms);

/* Correlation path of a grid (0 = grid 1, 1 = grid 2).  PIV_XCORR_SIMT: register FFTs in FP32 on the CUDA cores
 * (default).  PIV_XCORR_TC_SPLIT: the transforms as DFT products on the tcgen05 tensor
 * cores with split-BF16 operands (hi*hi + hi*lo + lo*hi, FP32 accumulation).
 * PIV_XCORR_TC_BF16: one BF16 product per step (precision study only).
 * PIV_XCORR_TC_SPLIT_F16 / PIV_XCORR_TC_F16: the same with FP16 operands (about 22
 * significant bits per split operand, 11 for one product; the passes' operands are scaled
 * by exact powers of two that keep them in FP16's range).  The tensor-core paths cover
 * 16x16, 32x32, 64x64, 48x24 and 24x48 windows with up to 8 saved peaks
 * (PIV_ERR_UNSUPPORTED otherwise).  PIV_XCORR_PATH=tc|tc1|tch|tch1 in the environment at piv_create selects
 * them for every grid they cover.  At 16x16 and 32x32 with spacing up to half the window,
 * a tile's windows of one grid row are staged into shared memory by TMA tensor-map copies
 * (identical results to direct loads; PIV_TC_STAGING=0 at piv_create turns it off). */
#define PIV_XCORR_SIMT 0
#define PIV_XCORR_TC_SPLIT 1
#define PIV_XCORR_TC_BF16 2
#define PIV_XCORR_TC_SPLIT_F16 3
#define PIV_XCORR_TC_F16 4
int piv_set_xcorr_path(piv_engine *e, int grid, int path);
int piv_get_xcorr_path(const piv_engine *e, int grid, int *path);

/* Kernels that one piv_run_pair launches with the engine's parameters. */
int piv_kernel_launches_per_pair(const piv_engine *e, int *n);

/* Re-launches one stage `reps` times on the engine stream on the current state (the
 * stage is idempotent on its inputs) and returns the mean device time per launch from
 * CUDA events on that stream.  which: 0 grid-1 correlation kernel (last pass's mode),
 * 1 grid-2 correlation kernel, 2 grid-2 deformation, 3 grid-2 validation (median passes
 * + fill + smoothing with the engine's parameters), 4 MHE of one frame. */
int piv_time_stage(piv_engine *e, int which, int reps, float *ms_per_launch);

/* Measured FP32 FMA throughput of the current device (TFLOP/s, 2 flops per FMA), from a
 * dependent-chain FMA kernel over every SM; the SIMT roofline of the FP32 correlation path. */
int piv_probe_fp32_peak(float *tflops);

/* Tensor-core self-check: D[128][N] = A[128][K] * B[N][K]^T computed by tcgen05 MMAs
 * with BF16 operands staged in shared memory (a_mn / b_mn: operand in the MN-major
 * instead of the K-major layout) and FP32 accumulation in tensor memory; nprod 1 uses
 * the rounded operands, 3 the split hi*hi + hi*lo + lo*hi.  Host arrays, row-major.
 * N and K: multiples of 16 in [16, 128].  PIV_ERR_UNSUPPORTED on a device other than
 * compute capability 10.x. */
int piv_tc_gemm_check(const float *A, const float *B, float *D, int N, int K, int a_mn, int b_mn, int nprod);

/* ---- standalone MHE (mhe_gpu) --------------------------------------------- */

/* mhe_gpu::init (X/MHE7_4_gpu.cu:149-212) on the current device. */
int piv_mhe_create(int Nx, int Ny, int ws, float thresh, piv_mhe **out);
/* mhe_gpu::processsing (X/MHE7_4_gpu.cu:214-253): d_in -> d_out, both Nx*Ny device bytes;
 * pixels outside the centred crop are written 0.  stream: a cudaStream_t or NULL. */
int piv_mhe_process(piv_mhe *m, const uint8_t *d_in, uint8_t *d_out, void *stream);
int piv_mhe_destroy(piv_mhe *m);

/* MHE of one frame without any allocation (no counterpart in the reference).  For callers
 * that cannot call cudaMalloc where they enhance a frame: real-time acquisition callbacks
 * that must not wait on the allocator, and applications whose own pool owns all device
 * memory after start-up.  Same result as piv_mhe_process (d_in -> d_out, Nx*Ny device
 * bytes each, outside the centred crop written 0), but the tile histograms live in a
 * fixed device array of the library: PIV_MHE_NOALLOC_MAX_TILES tiles including the
 * one-tile border ring, i.e. (Ny/ws + 2) * (Nx/ws + 2) <= 24576 (24 MiB, held by every GPU
 * that loads the library until exit).  Larger requests return PIV_ERR_ARG with a message
 * on stderr.  The first call on a device (and the first after that device's context was
 * re-created, e.g. by cudaDeviceReset) looks up the array's device address; make that
 * first call before any stream capture.  All calls share the array and each clears the
 * part it uses: calls whose work overlaps on the GPU (other streams, other threads) race
 * and must be serialised by the caller. */
#define PIV_MHE_NOALLOC_MAX_TILES 24576
int piv_mhe_process_noalloc(const uint8_t *d_in, uint8_t *d_out, int Nx, int Ny, int ws, float thresh,
                            void *stream);

/* ---- synthetic particle-image pairs (no reference counterpart) -------------- */

/* Displacement field models. */
#define PIV_FIELD_UNIFORM 0   /* (a, b) */
#define PIV_FIELD_VORTEX 1    /* Lamb-Oseen vortex: peak speed a, core radius b, plus shear c*(y-Ny/2) in x */
#define PIV_FIELD_FOURIER 2   /* sum of 8 seeded Fourier modes, wavelengths in [a, b] px, max |u| c */

typedef struct piv_synth_params {
    int Nx, Ny;
    double ppp;            /* particles per pixel */
    double sigma;          /* Gaussian spot sigma, px */
    double i_min, i_max;   /* peak intensity U(i_min, i_max) */
    double background;     /* additive background */
    double noise_sigma;    /* additive Gaussian noise sigma */
    int field;             /* PIV_FIELD_* */
    double a, b, c;        /* field parameters */
    uint64_t seed;
} piv_synth_params;

/* Renders frame 1 (particles at x) and frame 2 (particles at x + u(x)) as uint8, Nx*Ny
 * each; deterministic for a given seed (Philox4x32-10 counter RNG).  Host-only. */
int piv_synth_pair(const piv_synth_params *s, uint8_t *f1, uint8_t *f2);

/* The displacement field of s evaluated at n points. */
int piv_synth_field(const piv_synth_params *s, const float *x, const float *y, int n, float *u, float *v);

/* The same pair rendered on the GPU from the same random streams (particles, field,
 * noise); the float accumulation order differs, so a pixel may differ from the host
 * generator by one grey level at a rounding tie.  d_f1, d_f2: Nx*Ny bytes each (device);
 * d_scratch: 2*Nx*Ny floats (device); stream: cudaStream_t or NULL.  Asynchronous. */
int piv_synth_pair_device(const piv_synth_params *s, uint8_t *d_f1, uint8_t *d_f2, float *d_scratch, void *stream);

/* ---- batches of uneven pairs (no reference counterpart) ----------------------------
 * n pairs of any sizes and window shapes (params[i]; every pair must have the same
 * Npass1 and Npass2), one engine each.  piv_batch_run runs every pair's pass loop as one
 * captured graph: per pass, the pairs' deformations and validations on parallel
 * branches and ONE persistent correlation launch per (grid, window shape, top-K width)
 * group over all pairs in it, instead of one launch per pair.  The first run autotunes
 * each group's tile variant on the batch's data (PIV_BATCH_VARIANT=v fixes it).  A pair
 * whose engine is set to a tensor-core path (piv_set_xcorr_path), or whose shape runs on
 * the generic-size kernel, correlates with its own launch on its branch of the graph.
 * Results are bit-identical to piv_run_pair on each engine.  Frames: set on each engine (piv_batch_engine +
 * piv_set_images / piv_set_device_images / piv_host_images) before piv_batch_run; read
 * fields from the engines after piv_batch_synchronize.  Asynchronous. */
typedef struct piv_batch piv_batch;
int piv_batch_create(const piv_params *params, int n, piv_batch **out);
int piv_batch_destroy(piv_batch *b);
const char *piv_batch_last_error(const piv_batch *b);
int piv_batch_engine(piv_batch *b, int i, piv_engine **e);
int piv_batch_run(piv_batch *b);
int piv_batch_synchronize(piv_batch *b);
int piv_batch_stream(const piv_batch *b, void **stream);
/* The correlation groups (up to max): window shape, grid (0/1), deformed pass or not,
 * pairs in the group, chosen tile variant and its windows per CTA; *n_groups = count. */
int piv_batch_groups(const piv_batch *b, int max, int *wsx, int *wsy, int *grid, int *deformed, int *pairs,
                     int *variant, int *windows_per_cta, int *n_groups);

/* ---- learned grid-1 predictor (no reference counterpart) --------------------------
 * Replaces the plain grid-1 passes (X/main.cpp:290-300 driving Calc_cc_map_p1 and
 * MedianFilter_Smoothing_p1) as the deformation predictor of the grid-2 passes.
 *   features: both frames box-averaged 4x4 (grey/255, global mean removed); at every
 *     grid-1 vector a (ws_x1/4 x ws_y1/4) window of frame 1 correlated with frame 2 at
 *     the 81 integer shifts |dx|,|dy| <= 4 of the downsampled grid, normalised by the
 *     windows' energies -> input [81][Ny1_vec][Nx1_vec];
 *   network: 4-level U-Net on the grid-1 vector grid (3x3 convolutions, LeakyReLU 0.1,
 *     stride-2 down, nearest-up + skip concatenation, 881,922 parameters), BF16 weights,
 *     FP32 activations and accumulation; output [2][Ny1_vec][Nx1_vec] in downsampled
 *     pixels (x4 = image pixels).
 * Training (piv_net_loss_grad + piv_net_adam_step) and inference run on hand-written
 * kernels; the net is bound to the device current at piv_net_create. */
typedef struct piv_net piv_net;
#define PIV_NET_IN_CHANNELS 81
#define PIV_NET_LAYERS 13
int piv_net_create(uint64_t seed, piv_net **out);
int piv_net_destroy(piv_net *n);
const char *piv_net_last_error(const piv_net *n);
int piv_net_num_params(const piv_net *n, int64_t *count);
/* Layer `layer` (0..12): input/output channels, stride, offsets of its weights
 * [cout][cin][3][3] and biases [cout] in the flat parameter vector. */
int piv_net_layout(int layer, int *cin, int *cout, int *stride, int *weight_offset, int *bias_offset);
int piv_net_get_params(piv_net *n, float *host, int64_t count);
int piv_net_set_params(piv_net *n, const float *host, int64_t count);  /* resets Adam */
int piv_net_get_grads(piv_net *n, float *host, int64_t count);
int piv_net_save(piv_net *n, const char *path);
int piv_net_load(piv_net *n, const char *path);
/* [N][81][H][W] -> [N][2][H][W] (device pointers); stream NULL = the net's own. */
int piv_net_forward(piv_net *n, const float *d_in, int N, int H, int W, float *d_out, void *stream);
/* Forward, Charbonnier loss against d_label [N][2][H][W] (downsampled px) over the
 * vectors with d_mask [N][H][W] = 1 (mean over them), backward into the net's gradient
 * buffer (overwritten).  Synchronous; *loss receives the loss. */
int piv_net_loss_grad(piv_net *n, const float *d_in, const float *d_label, const float *d_mask, int N, int H, int W,
                      float *loss);
int piv_net_adam_step(piv_net *n, float lr);  /* Adam, beta 0.9/0.999, eps 1e-8 */
int piv_net_synchronize(piv_net *n);

/* The predictor input of the engine's current (prepared) frames at grid 1, written to
 * d_out [81][Ny1_vec][Nx1_vec] on the engine's stream (asynchronous). */
int piv_net_features(piv_engine *e, piv_net *n, float *d_out);
/* The learned form of a pair: prep, features, network -> grid-1 field (all valid),
 * upsampling, the Npass2 grid-2 passes with their validation (the grid's correlation
 * path, piv_set_xcorr_path), then the judge: the fraction of grid-2 vectors the last
 * median test rejected and the RMS difference between the upsampled prediction and the
 * final grid-2 field.  Above max_reject_frac or max_rms_px, the pair is run again by the
 * plain method (piv_run_pair) and *fell_back = 1.  Synchronous (the judge is read on the
 * host).  Requires Npass2 > 0. */
int piv_run_pair_learned(piv_engine *e, piv_net *n, float max_reject_frac, float max_rms_px, int *fell_back,
                         float *reject_frac, float *rms_px);

#ifdef __cplusplus
}
#endif
#endif
