// engine.cu -- host engine behind the C-ABI of include/piv_b200.h.
//
// Device layout (one engine = one image-pair pipeline on one GPU):
//   frames      2 x uint8, zero-padded (margin mx/my, pitch a multiple of 128 B); the
//               image pixel (x, y) sits at [(y+my)*pitch + x+mx].  Replaces the four
//               aug_ex buffers of the reference (one per frame per grid).
//   staging     2 x uint8 Nx*Ny, only when MHE is on (raw upload, MHE input).
//   deformed    per grid, float [Ny_aug][pitch] (Kernel_Window_Deformation_2d output).
//   per grid    candidates dx/dy/valid [Nt_vec][Npeak_save], peak taps (count, index,
//               value), filtered field fx/fy/valid [Nt_vec] + a ping-pong copy, the
//               fill work list.
// There are no correlation-plane buffers: the fused kernel keeps them on chip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "learned.cuh"
#include "piv_common.cuh"

namespace piv {

static int imax(int a, int b) { return a > b ? a : b; }

// PIV_AUTOTUNE, read the same way by the engine's and the batch's tuners: unset, or any
// value other than 0 / off / false / no (any case), leaves tuning on.  Every tile variant
// of a shape computes the same bits, so tuning changes speed only.
static bool autotune_enabled()
{
    const char *env = getenv("PIV_AUTOTUNE");
    if (!env) return true;
    std::string v(env);
    for (char &c : v) c = (char)tolower((unsigned char)c);
    return !(v == "0" || v == "off" || v == "false" || v == "no");
}

static int vec_count(int N, int sp)
{
    // X/xcorr2d_multi_grid.cu:771-777
    int t1 = (N - sp / 2 - 1) / sp;
    int t2 = N - (sp / 2 + 1 + t1 * sp);
    while (t2 < (sp / 2 - 1)) {
        t1 = t1 - 1;
        t2 = t2 + sp;
    }
    return t1 + 1;
}

int compute_geometry(const piv_params &p, piv_geometry &g, const char **why)
{
    std::memset(&g, 0, sizeof(g));
    auto fail = [&](int code, const char *msg) {
        if (why) *why = msg;
        return code;
    };
    if (p.Nx < 1 || p.Ny < 1) return fail(PIV_ERR_ARG, "image size must be positive");
    if (p.Nsec_cc < 1) return fail(PIV_ERR_ARG, "Nsec_cc must be >= 1");
    if (p.Npeak_save < 1) return fail(PIV_ERR_ARG, "Npeak_save must be >= 1");
    const int wsx[2] = {p.ws_x1, p.ws_x2}, wsy[2] = {p.ws_y1, p.ws_y2};
    const int spx[2] = {p.spacing_x1, p.spacing_x2}, spy[2] = {p.spacing_y1, p.spacing_y2};
    const float pcx[2] = {p.max_dispx_win_percent1, p.max_dispx_win_percent2};
    const float pcy[2] = {p.max_dispy_win_percent1, p.max_dispy_win_percent2};
    // window validation of X/xcorr2d_multi_grid.cu:896-920 (same messages)
    if (wsx[0] < 4 || wsy[0] < 4) return fail(PIV_ERR_GEOMETRY, "The interrogation window size (1st grid) is too small!");
    if (wsx[0] > 1024 || wsy[0] > 1024) return fail(PIV_ERR_GEOMETRY, "The interrogation window size (1st grid) is too big!");
    if (wsx[1] < 4 || wsy[1] < 4) return fail(PIV_ERR_GEOMETRY, "The interrogation window size (2nd grid) is too small!");
    if (wsx[1] > 1024 || wsy[1] > 1024) return fail(PIV_ERR_GEOMETRY, "The interrogation window size (2nd grid) is too big!");
    if (wsx[0] % 4 != 0 || wsx[1] % 4 != 0) return fail(PIV_ERR_GEOMETRY, "The window x-dimension is not divisible by 4!");
    if (wsy[0] % 4 != 0 || wsy[1] % 4 != 0) return fail(PIV_ERR_GEOMETRY, "The window y-dimension is not divisible by 4!");
    for (int k = 0; k < 2; ++k) {
        if (spx[k] < 1 || spy[k] < 1) return fail(PIV_ERR_ARG, "vector spacing must be >= 1");
        g.border_x[k] = imax(1, wsx[k] / 2 - (int)roundf((float)wsx[k] * pcx[k]));
        g.border_y[k] = imax(1, wsy[k] / 2 - (int)roundf((float)wsy[k] * pcy[k]));
        g.hfws_x[k] = wsx[k] / 2;
        g.hfws_y[k] = wsy[k] / 2;
        g.Npeak[k] = wsx[k] * wsy[k] / 4 / 4;
        g.Nx_vec[k] = vec_count(p.Nx, spx[k]);
        g.Ny_vec[k] = vec_count(p.Ny, spy[k]);
        if (g.Nx_vec[k] < 1 || g.Ny_vec[k] < 1) return fail(PIV_ERR_GEOMETRY, "image smaller than one vector spacing");
        g.Nt_vec[k] = g.Nx_vec[k] * g.Ny_vec[k];
        // sectioning, X/xcorr2d_multi_grid.cu:805-829 (Nsec_cc > Nt_vec never terminates there)
        int Nt = g.Nt_vec[k], Nsec = p.Nsec_cc;
        if (Nsec > Nt) return fail(PIV_ERR_ARG, "Nsec_cc exceeds the number of vectors");
        if (Nt % Nsec == 0) {
            g.Neach[k] = Nt / Nsec;
            g.Nlast[k] = g.Neach[k];
        } else {
            g.Neach[k] = Nt / Nsec;
            g.Nlast[k] = Nt - (Nsec - 1) * g.Neach[k];
            while (g.Nlast[k] > g.Neach[k]) {
                g.Nlast[k] -= g.Neach[k];
                Nsec += 1;
            }
        }
        g.Nsec[k] = Nsec;
        const int hx = g.hfws_x[k], hy = g.hfws_y[k];
        g.Nx_left[k] = (spx[k] / 2 < hx) ? hx - spx[k] / 2 : 0;
        g.Ny_left[k] = (spy[k] / 2 < hy) ? hy - spy[k] / 2 : 0;
        g.Nx_right[k] = ((p.Nx - spx[k] / 2 - 1 - (g.Nx_vec[k] - 1) * spx[k]) < (hx - 1))
                            ? spx[k] / 2 + 1 + (g.Nx_vec[k] - 1) * spx[k] + hx - 1 - p.Nx
                            : 0;
        g.Ny_right[k] = ((p.Ny - spy[k] / 2 - 1 - (g.Ny_vec[k] - 1) * spy[k]) < (hy - 1))
                            ? spy[k] / 2 + 1 + (g.Ny_vec[k] - 1) * spy[k] + hy - 1 - p.Ny
                            : 0;
        g.Nx_aug[k] = p.Nx + g.Nx_left[k] + g.Nx_right[k];
        g.Ny_aug[k] = p.Ny + g.Ny_left[k] + g.Ny_right[k];
        g.Nx_aug_ex[k] = g.Nx_aug[k] + wsx[k];
        g.Ny_aug_ex[k] = g.Ny_aug[k] + wsy[k];
    }
    return PIV_OK;
}

}  // namespace piv

using namespace piv;

struct GridState {
    GridGeom gg{};
    float *cdx = nullptr, *cdy = nullptr;
    uint8_t *cv = nullptr;
    int32_t *count = nullptr, *pidx = nullptr;
    float *pval = nullptr;
    float *fx = nullptr, *fy = nullptr, *tx = nullptr, *ty = nullptr;
    uint8_t *fv = nullptr, *tv = nullptr;
    int *list = nullptr;
    float *def = nullptr;
    int def_pitch = 0;
    bool last_deformed = false;
    bool has_pass = false;
    int variant = 0;          // fused-kernel instantiation chosen by the autotuner
    int path = PIV_XCORR_SIMT;  // correlation path (PIV_XCORR_*)
    // generic-size kernel (xcorr_generic.cu): shapes without a fused instance, or more
    // than 8 saved peaks; planes above 20,480 points live in a workspace of gws_ctas slabs
    bool generic = false;
    float2 *gws = nullptr;
    int gws_ctas = 0;
    float tuned_ms[8] = {};   // measured time per variant (0 = not measured)
    int n_tuned = 0;
    // TMA staging maps of the tensor-core kernels, built at their first launch (the frame and
    // deformed-frame buffers live as long as the engine): [0] the undeformed pass, [1] the
    // deformed pass
    TcStaging stage[2];
    bool stage_built[2] = {false, false};
};

struct piv_engine {
    piv_params p{};
    piv_geometry g{};
    int device = 0;
    cudaStream_t stream = nullptr;
    uint8_t *h_f1 = nullptr, *h_f2 = nullptr;
    const uint8_t *d_in1 = nullptr, *d_in2 = nullptr;  // caller's device frames
    uint8_t *d_stage1 = nullptr, *d_stage2 = nullptr;
    uint8_t *d_f1 = nullptr, *d_f2 = nullptr;
    int mx = 0, my = 0, pitch = 0, rows = 0;
    bool tc_staging = true;  // tensor-core kernels stage window rows through TMA where they can
    GridState grid[2];
    MheGeom mg{};
    int *d_levels = nullptr;
    int *d_status = nullptr, *d_list_n = nullptr;
    int *h_status = nullptr;
    bool prepared = false;
    // captured pair graphs, one per input-frame address pair (the host path, caller
    // frames, and the two upload slots each get their own)
    struct PairGraph {
        cudaGraphExec_t exec = nullptr;
        const uint8_t *in1 = nullptr, *in2 = nullptr;
    };
    PairGraph graphs[4];
    int n_graphs = 0;
    // pipelined input (piv_queue_images): two device slots filled on the copy stream;
    // ev_up[s] marks slot s uploaded, ev_done[s] the end of the last pair that read it
    cudaStream_t copy_stream = nullptr;
    uint8_t *d_slot[2][2] = {};
    cudaEvent_t ev_up[2] = {}, ev_done[2] = {};
    bool slot_read[2] = {};
    int next_slot = 0, pending_slot = -1, reading_slot = -1;
    // asynchronous readback (piv_field_async / piv_field_wait): two pinned result slots
    struct ResultSlot {
        float *dx = nullptr, *dy = nullptr;
        uint8_t *valid = nullptr;
        int *status = nullptr;
        size_t cap = 0;       // elements the slot holds
        int sel = 0, seq = 0;
        bool pending = false;
        cudaEvent_t ev = nullptr;
    };
    ResultSlot results[2];
    int result_seq = 0;
    // learned form (piv_run_pair_learned): its captured graph, keyed by input frames and
    // net; the upsampled prediction kept for the judge; the judge's two numbers
    cudaGraphExec_t learned_exec = nullptr;
    const uint8_t *learned_in1 = nullptr, *learned_in2 = nullptr;
    const piv_net *learned_net = nullptr;
    unsigned learned_gen = 0;
    float *d_pred2 = nullptr, *d_judge = nullptr, *h_judge = nullptr;
    std::string err;
    // fault injection, read from the environment at piv_create (off by default):
    // PIV_TEST_FAIL_ALLOC=k fails the engine's k-th device allocation (counted from piv_create),
    // PIV_TEST_FILL_CAP=n caps the hole fill at n iterations
    int fail_alloc_at = 0, n_allocs = 0, fill_cap = 0;
    bool timing = false;
    cudaEvent_t ev[6] = {};
    float stage_ms[5] = {};
    bool have_times = false;
};

struct piv_mhe {
    MheGeom mg{};
    int *d_levels = nullptr;
    int device = 0;
};

namespace {

int set_err(piv_engine *e, int code, const char *fmt, ...)
{
    if (e) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        e->err = buf;
    }
    return code;
}

#define CK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t _e = (call);                                                                           \
        if (_e != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));   \
    } while (0)

template <typename T>
int dalloc(piv_engine *e, T **ptr, size_t n)
{
    if (n == 0) n = 1;
    if (e->fail_alloc_at > 0 && ++e->n_allocs == e->fail_alloc_at) {
        *ptr = nullptr;
        return set_err(e, PIV_ERR_ALLOC, "cudaMalloc ERROR! (%zu bytes: injected failure)", n * sizeof(T));
    }
    cudaError_t c = cudaMalloc((void **)ptr, n * sizeof(T));
    if (c != cudaSuccess) {
        *ptr = nullptr;
        return set_err(e, PIV_ERR_ALLOC, "cudaMalloc ERROR! (%zu bytes: %s)", n * sizeof(T), cudaGetErrorString(c));
    }
    return PIV_OK;
}

void free_all(piv_engine *e)
{
    for (int i = 0; i < e->n_graphs; ++i) cudaGraphExecDestroy(e->graphs[i].exec);
    e->n_graphs = 0;
    if (e->learned_exec) cudaGraphExecDestroy(e->learned_exec);
    e->learned_exec = nullptr;
    cudaFree(e->d_pred2);
    cudaFree(e->d_judge);
    cudaFreeHost(e->h_judge);
    for (int q = 0; q < 2; ++q) {
        cudaFree(e->d_slot[q][0]);
        cudaFree(e->d_slot[q][1]);
        if (e->ev_up[q]) cudaEventDestroy(e->ev_up[q]);
        if (e->ev_done[q]) cudaEventDestroy(e->ev_done[q]);
    }
    if (e->copy_stream) cudaStreamDestroy(e->copy_stream);
    for (auto &r : e->results) {
        cudaFreeHost(r.dx);
        cudaFreeHost(r.dy);
        cudaFreeHost(r.valid);
        cudaFreeHost(r.status);
        if (r.ev) cudaEventDestroy(r.ev);
    }
    cudaFreeHost(e->h_f1);
    cudaFreeHost(e->h_f2);
    cudaFreeHost(e->h_status);
    cudaFree(e->d_stage1);
    cudaFree(e->d_stage2);
    cudaFree(e->d_f1);
    cudaFree(e->d_f2);
    cudaFree(e->d_levels);
    cudaFree(e->d_status);
    cudaFree(e->d_list_n);
    for (auto &gs : e->grid) {
        cudaFree(gs.gws);
        cudaFree(gs.cdx);
        cudaFree(gs.cdy);
        cudaFree(gs.cv);
        cudaFree(gs.count);
        cudaFree(gs.pidx);
        cudaFree(gs.pval);
        cudaFree(gs.fx);
        cudaFree(gs.fy);
        cudaFree(gs.tx);
        cudaFree(gs.ty);
        cudaFree(gs.fv);
        cudaFree(gs.tv);
        cudaFree(gs.list);
        cudaFree(gs.def);
    }
    for (auto &ev : e->ev)
        if (ev) cudaEventDestroy(ev);
    if (e->stream) cudaStreamDestroy(e->stream);
}

int round_up(int v, int m) { return (v + m - 1) / m * m; }

Frame8 frame_of(const piv_engine *e, const uint8_t *base)
{
    Frame8 f;
    f.base = base;
    f.pitch = e->pitch;
    f.mx = e->mx;
    f.my = e->my;
    f.cols = e->pitch;
    f.rows = e->rows;
    return f;
}

int check_ready(piv_engine *e, bool need_prep)
{
    if (!e) return PIV_ERR_ARG;
    if (cudaSetDevice(e->device) != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "cudaSetDevice failed");
    if (need_prep && !e->prepared) return set_err(e, PIV_ERR_STATE, "piv_prep has not run");
    return PIV_OK;
}

// ---- pipeline stages (queue work on e->stream; no host synchronisation) ----

int do_prep(piv_engine *e)
{
    const piv_params &p = e->p;
    cudaStream_t s = e->stream;
    for (int f = 0; f < 2; ++f) {
        const uint8_t *din = f ? e->d_in2 : e->d_in1;
        uint8_t *dst = f ? e->d_f2 : e->d_f1;
        uint8_t *host = f ? e->h_f2 : e->h_f1;
        if (p.if_mhe == 1) {
            const uint8_t *src = din;
            if (!src) {
                uint8_t *stage = f ? e->d_stage2 : e->d_stage1;
                CK(cudaMemcpyAsync(stage, host, (size_t)p.Nx * p.Ny, cudaMemcpyHostToDevice, s));
                src = stage;
            }
            CK(launch_mhe(e->mg, src, p.Nx, e->d_levels, dst, e->pitch, e->mx, e->my, s));
        } else if (din) {
            CK(cudaMemcpy2DAsync(dst + (size_t)e->my * e->pitch + e->mx, e->pitch, din, p.Nx, p.Nx, p.Ny,
                                 cudaMemcpyDeviceToDevice, s));
        } else {
            CK(cudaMemcpy2DAsync(dst + (size_t)e->my * e->pitch + e->mx, e->pitch, host, p.Nx, p.Nx, p.Ny,
                                 cudaMemcpyHostToDevice, s));
        }
    }
    e->prepared = true;
    return PIV_OK;
}

// Arguments of grid k's correlation launch over all its windows.
XcorrArgs xcorr_args(piv_engine *e, int k)
{
    GridState &gs = e->grid[k];
    XcorrArgs a;
    a.g = gs.gg;
    a.f1 = frame_of(e, e->d_f1);
    a.f2 = frame_of(e, e->d_f2);
    a.def = gs.def;
    a.def_pitch = gs.def_pitch;
    a.pred_x = gs.fx;
    a.pred_y = gs.fy;
    a.cdx = gs.cdx;
    a.cdy = gs.cdy;
    a.cvalid = gs.cv;
    a.count = gs.count;
    a.pidx = gs.pidx;
    a.pval = gs.pval;
    a.cc_dump = nullptr;
    a.status = e->d_status;
    a.w_first = 0;
    a.w_end = gs.gg.Nt_vec;
    return a;
}

// The generic-size kernel's plane workspace of grid k, for planes too large for shared
// memory (allocated at piv_create for the grids with passes, else at the first pass).
int ensure_workspace(piv_engine *e, int k)
{
    GridState &gs = e->grid[k];
    if (!gs.generic || gs.gws || !xcorr_generic_needs_workspace(gs.gg.ws_x, gs.gg.ws_y)) return PIV_OK;
    gs.gws_ctas = imax(1, std::min(gs.gg.Nt_vec, xcorr_generic_ctas(gs.gg.ws_x, gs.gg.ws_y, gs.gg.Nps)));
    return dalloc(e, &gs.gws, (size_t)gs.gws_ctas * gs.gg.ws_x * gs.gg.ws_y);
}

int do_xcorr(piv_engine *e, int k, bool deformed, int first, int end, float *dump)
{
    GridState &gs = e->grid[k];
    XcorrArgs a;
    a.g = gs.gg;
    a.f1 = frame_of(e, e->d_f1);
    a.f2 = frame_of(e, e->d_f2);
    a.def = gs.def;
    a.def_pitch = gs.def_pitch;
    a.pred_x = gs.fx;
    a.pred_y = gs.fy;
    a.cdx = gs.cdx;
    a.cdy = gs.cdy;
    a.cvalid = gs.cv;
    a.count = gs.count;
    a.pidx = gs.pidx;
    a.pval = gs.pval;
    a.cc_dump = dump;
    a.status = e->d_status;
    const char *why = nullptr;
    auto launch = [&]() {
        if (gs.generic) return launch_xcorr_generic(a, deformed, gs.gws, gs.gws_ctas, e->stream);
        if (gs.path == PIV_XCORR_SIMT) return launch_xcorr(a, deformed, e->stream, &why, gs.variant);
        const bool split = gs.path == PIV_XCORR_TC_SPLIT || gs.path == PIV_XCORR_TC_SPLIT_F16;
        const bool f16 = gs.path == PIV_XCORR_TC_SPLIT_F16 || gs.path == PIV_XCORR_TC_F16;
        const TcStaging *stage = nullptr;
        if (gs.gg.ws_x == gs.gg.ws_y && e->tc_staging) {
            const int d = deformed ? 1 : 0;
            if (!gs.stage_built[d]) {
                tc_staging_build(gs.stage[d], gs.gg.ws_x, gs.gg.sp_x, e->d_f1, e->d_f2, e->pitch, e->rows,
                                 deformed ? gs.def : nullptr, gs.def_pitch, gs.gg.Ny_aug);
                gs.stage_built[d] = true;
            }
            stage = &gs.stage[d];
        }
        return launch_xcorr_tc(a, deformed, e->stream, &why, split ? 3 : 1, f16, stage);
    };
    if (dump) {
        a.w_first = first;
        a.w_end = end;
        cudaError_t c = launch();
        if (c != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "correlation kernel: %s", why ? why : cudaGetErrorString(c));
        return PIV_OK;
    }
    // Nsec_cc sections (X/xcorr2d_multi_grid.cu:1308-1441); the results do not depend on it
    const int Nsec = e->g.Nsec[k], Neach = e->g.Neach[k], Nlast = e->g.Nlast[k];
    for (int i = 0; i < Nsec; ++i) {
        a.w_first = i * Neach;
        a.w_end = a.w_first + (i == Nsec - 1 ? Nlast : Neach);
        cudaError_t c = launch();
        if (c != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "correlation kernel: %s", why ? why : cudaGetErrorString(c));
    }
    return PIV_OK;
}

int do_deform(piv_engine *e, int k)
{
    GridState &gs = e->grid[k];
    DeformArgs d;
    d.f2 = frame_of(e, e->d_f2);
    d.out = gs.def;
    d.out_pitch = gs.def_pitch;
    d.Nx_aug = e->g.Nx_aug[k];
    d.Ny_aug = e->g.Ny_aug[k];
    d.fx = gs.fx;
    d.fy = gs.fy;
    d.Nx_vec = gs.gg.Nx_vec;
    d.Ny_vec = gs.gg.Ny_vec;
    d.sp_x = gs.gg.sp_x;
    d.sp_y = gs.gg.sp_y;
    d.hfws_x = gs.gg.hfws_x;
    d.hfws_y = gs.gg.hfws_y;
    d.Nx_left = gs.gg.Nx_left;
    d.Ny_left = gs.gg.Ny_left;
    CK(launch_deform(d, e->stream));
    return PIV_OK;
}

int do_pass(piv_engine *e, int k, int idx_pass)
{
    GridState &gs = e->grid[k];
    bool deformed = true;
    if (k == 0 && idx_pass == 0) {
        // Calc_cc_map_p1(0): zero predictor, undeformed frame 2 (X/xcorr2d_multi_grid.cu:1287-1298)
        CK(cudaMemsetAsync(gs.fx, 0, sizeof(float) * gs.gg.Nt_vec, e->stream));
        CK(cudaMemsetAsync(gs.fy, 0, sizeof(float) * gs.gg.Nt_vec, e->stream));
        deformed = false;
    } else {
        int rc = do_deform(e, k);
        if (rc) return rc;
    }
    int rc = do_xcorr(e, k, deformed, 0, 0, nullptr);
    if (rc) return rc;
    gs.last_deformed = deformed;
    gs.has_pass = true;
    return PIV_OK;
}

int do_validate(piv_engine *e, int k, int Npass_median, int minN, float thr, int Npass_smooth, int iffill)
{
    GridState &gs = e->grid[k];
    const int wxm = k ? e->p.wx2_median : e->p.wx1_median, wym = k ? e->p.wy2_median : e->p.wy1_median;
    const int wxs = k ? e->p.wx2_smooth : e->p.wx1_smooth, wys = k ? e->p.wy2_smooth : e->p.wy1_smooth;
    if (Npass_median < 0 || Npass_smooth < 0) return set_err(e, PIV_ERR_ARG, "negative pass count");
    if (Npass_median > 0 && (wxm < 1 || wym < 1)) return set_err(e, PIV_ERR_ARG, "median window must be >= 1");
    if (Npass_smooth > 0 && (wxs < 1 || wys < 1)) return set_err(e, PIV_ERR_ARG, "smoothing window must be >= 1");
    ValidateArgs v;
    v.cdx = gs.cdx;
    v.cdy = gs.cdy;
    v.cvalid = gs.cv;
    v.Nps = e->p.Npeak_save;
    v.Nx_vec = gs.gg.Nx_vec;
    v.Ny_vec = gs.gg.Ny_vec;
    v.fx = gs.fx;
    v.fy = gs.fy;
    v.fv = gs.fv;
    v.tx = gs.tx;
    v.ty = gs.ty;
    v.tv = gs.tv;
    v.wx_med = wxm;
    v.wy_med = wym;
    v.Npass_median = Npass_median;
    v.minNneigh = minN;
    v.insert_threshold = thr;
    v.wx_sm = wxs;
    v.wy_sm = wys;
    v.Npass_smooth = Npass_smooth;
    v.iffill = iffill;
    v.list = gs.list;
    v.list_n = e->d_list_n;
    v.status = e->d_status;
    v.fill_cap = e->fill_cap;
    CK(launch_validate(v, e->stream));
    return PIV_OK;
}

int do_upsample(piv_engine *e)
{
    UpsampleArgs u;
    u.fx1 = e->grid[0].fx;
    u.fy1 = e->grid[0].fy;
    u.Nx1 = e->grid[0].gg.Nx_vec;
    u.Ny1 = e->grid[0].gg.Ny_vec;
    u.sp_x1 = e->p.spacing_x1;
    u.sp_y1 = e->p.spacing_y1;
    u.fx2 = e->grid[1].fx;
    u.fy2 = e->grid[1].fy;
    u.Nx2 = e->grid[1].gg.Nx_vec;
    u.Ny2 = e->grid[1].gg.Ny_vec;
    u.sp_x2 = e->p.spacing_x2;
    u.sp_y2 = e->p.spacing_y2;
    CK(launch_upsample(u, e->stream));
    return PIV_OK;
}

// X/main.cpp:288-326.  `ev` (optional) records stage boundaries for piv_stage_times.
int do_pair(piv_engine *e, bool with_events)
{
    const piv_params &p = e->p;
    int rc;
    auto mark = [&](int i) {
        if (with_events) cudaEventRecord(e->ev[i], e->stream);
    };
    mark(0);
    if ((rc = do_prep(e))) return rc;
    mark(1);
    for (int j = 0; j < p.Npass1; ++j) {
        if ((rc = do_pass(e, 0, j))) return rc;
        if ((rc = do_validate(e, 0, p.Npass1_median, p.minNneigh_p1, p.insert_threshold_p1, p.Npass1_smooth, 1)))
            return rc;
    }
    mark(2);
    if (p.Npass2 > 0) {
        if ((rc = do_upsample(e))) return rc;
        for (int j = 0; j < p.Npass2; ++j) {
            if ((rc = do_pass(e, 1, j))) return rc;
            if ((rc = do_validate(e, 1, p.Npass2_median, p.minNneigh_p2, p.insert_threshold_p2, p.Npass2_smooth, 1)))
                return rc;
        }
    }
    mark(3);
    return PIV_OK;
}

// Features of the prepared frames at grid 1 into `out` (the predictor input).
int do_features(piv_engine *e, piv_net *n, float *out)
{
    learned::FeatArgs f;
    f.f1 = e->d_f1 + (size_t)e->my * e->pitch + e->mx;
    f.f2 = e->d_f2 + (size_t)e->my * e->pitch + e->mx;
    f.pitch = e->pitch;
    f.Nx = e->p.Nx;
    f.Ny = e->p.Ny;
    f.g = e->grid[0].gg;
    f.down = learned::net_feature_down(n);
    f.sums = learned::net_feature_sums(n);
    f.out = out;
    CK(learned::launch_features(f, e->stream));
    return PIV_OK;
}

// The learned form of a pair up to the judge (captured as one graph): prep, features,
// network, grid-1 field, upsampling, the grid-2 passes, judge.
int do_learned(piv_engine *e, piv_net *n)
{
    const piv_params &p = e->p;
    int rc;
    if ((rc = do_prep(e))) return rc;
    GridState &g1 = e->grid[0], &g2 = e->grid[1];
    const int H = g1.gg.Ny_vec, W = g1.gg.Nx_vec;
    if ((rc = do_features(e, n, learned::net_input(n)))) return rc;
    CK(learned::net_forward(n, learned::net_input(n), 1, H, W, nullptr, e->stream));
    CK(learned::launch_field_from_net(learned::net_output(n), g1.gg.Nt_vec, g1.fx, g1.fy, g1.fv, e->stream));
    if ((rc = do_upsample(e))) return rc;
    const size_t nt2 = (size_t)g2.gg.Nt_vec;
    CK(cudaMemcpyAsync(e->d_pred2, g2.fx, nt2 * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
    CK(cudaMemcpyAsync(e->d_pred2 + nt2, g2.fy, nt2 * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
    for (int j = 0; j < p.Npass2; ++j) {
        if ((rc = do_pass(e, 1, j))) return rc;
        if ((rc = do_validate(e, 1, p.Npass2_median, p.minNneigh_p2, p.insert_threshold_p2, p.Npass2_smooth, 1)))
            return rc;
    }
    CK(learned::launch_judge(e->d_pred2, e->d_pred2 + nt2, g2.fx, g2.fy, g2.gg.Nt_vec, e->d_list_n, e->d_judge,
                             e->stream));
    return PIV_OK;
}

// The autotuner: every instantiated variant (windows per CTA, threads per CTA) of each
// grid's window shape is timed on this engine's own geometry, with the frames (and the
// deformed frame, the mode most passes run in) holding a particle-like pattern; the
// fastest variant is kept.  PIV_AUTOTUNE=0 keeps the defaults; PIV_XCORR_VARIANT=v1,v2
// fixes the variants by index.
int tune_xcorr(piv_engine *e)
{
    if (const char *fixed = getenv("PIV_XCORR_VARIANT")) {
        // "v1,v2": the grids' variants by index, no timing (profiling a chosen variant)
        int v[2] = {0, 0};
        if (sscanf(fixed, "%d,%d", &v[0], &v[1]) != 2) return set_err(e, PIV_ERR_ARG, "PIV_XCORR_VARIANT wants v1,v2");
        for (int k = 0; k < 2; ++k) {
            GridState &gs = e->grid[k];
            if (gs.generic) continue;  // one form only
            if (v[k] < 0 || v[k] >= xcorr_variants(gs.gg.ws_x, gs.gg.ws_y))
                return set_err(e, PIV_ERR_ARG, "PIV_XCORR_VARIANT: grid %d has %d variants", k + 1,
                               xcorr_variants(gs.gg.ws_x, gs.gg.ws_y));
            gs.variant = v[k];
        }
        return PIV_OK;
    }
    if (!autotune_enabled()) return PIV_OK;
    const piv_params &p = e->p;
    cudaStream_t s = e->stream;
    CK(launch_pattern(e->d_f1, nullptr, e->pitch, e->pitch, e->rows, 1u, s));
    CK(launch_pattern(e->d_f2, nullptr, e->pitch, e->pitch, e->rows, 2u, s));
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    int rc = PIV_OK;
    for (int k = 0; k < 2 && !rc; ++k) {
        GridState &gs = e->grid[k];
        if ((k == 0 ? p.Npass1 : p.Npass2) < 1 || gs.generic) continue;
        const int nv = xcorr_variants(gs.gg.ws_x, gs.gg.ws_y);
        if (nv <= 1) continue;
        const bool deformed = gs.def != nullptr;
        if (deformed) CK(launch_pattern(nullptr, gs.def, gs.def_pitch, gs.gg.Nx_aug, gs.gg.Ny_aug, 3u + k, s));
        float best = 1e30f;
        int best_v = 0;
        for (int v = 0; v < nv && v < 8 && !rc; ++v) {
            gs.variant = v;
            if ((rc = do_xcorr(e, k, deformed, 0, 0, nullptr))) break;  // warm-up
            cudaEventRecord(a, s);
            for (int r = 0; r < 2 && !rc; ++r) rc = do_xcorr(e, k, deformed, 0, 0, nullptr);
            cudaEventRecord(b, s);
            if (cudaEventSynchronize(b) != cudaSuccess) {
                rc = set_err(e, PIV_ERR_CUDA, "autotune timing failed");
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            gs.tuned_ms[v] = ms / 2;
            if (ms < best) {
                best = ms;
                best_v = v;
            }
        }
        gs.variant = best_v;
        gs.n_tuned = nv < 8 ? nv : 8;
        // leave no trace of the tuning input
        if (deformed) CK(cudaMemsetAsync(gs.def, 0, (size_t)gs.def_pitch * gs.gg.Ny_aug * sizeof(float), s));
        const size_t Nt = (size_t)gs.gg.Nt_vec, Nc = Nt * p.Npeak_save;
        CK(cudaMemsetAsync(gs.cdx, 0, Nc * sizeof(float), s));
        CK(cudaMemsetAsync(gs.cdy, 0, Nc * sizeof(float), s));
        CK(cudaMemsetAsync(gs.cv, 0, Nc, s));
        CK(cudaMemsetAsync(gs.count, 0, Nt * sizeof(int), s));
        CK(cudaMemsetAsync(gs.pidx, 0xff, Nc * sizeof(int), s));
        CK(cudaMemsetAsync(gs.pval, 0, Nc * sizeof(float), s));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaMemsetAsync(e->d_f1, 0, (size_t)e->pitch * e->rows, s));
    CK(cudaMemsetAsync(e->d_f2, 0, (size_t)e->pitch * e->rows, s));
    CK(cudaStreamSynchronize(s));
    return rc;
}

int validate_params(piv_engine *e, const piv_params &p)
{
    const char *why = nullptr;
    int rc = compute_geometry(p, e->g, &why);
    if (rc) return set_err(e, rc, "%s", why ? why : "invalid parameters");
    // every shape the geometry accepts runs: the fused kernels or the generic-size one
    if (p.Npeak_save > kGenericMaxPeaks)
        return set_err(e, PIV_ERR_ARG, "Npeak_save above %d is not supported", kGenericMaxPeaks);
    if (p.Npass1 < 0 || p.Npass2 < 0) return set_err(e, PIV_ERR_ARG, "negative pass count");
    if (p.if_mhe == 1 && !mhe_geometry(p.Nx, p.Ny, p.mhe_ws, p.mhe_thresh, e->mg))
        return set_err(e, PIV_ERR_ARG, "invalid MHE window/threshold");
    return PIV_OK;
}

}  // namespace

// ==================================================================================
// C-ABI
// ==================================================================================
extern "C" {

const char *piv_status_string(int s)
{
    switch (s) {
    case PIV_OK: return "ok";
    case PIV_ERR_ARG: return "invalid argument";
    case PIV_ERR_GEOMETRY: return "invalid window geometry";
    case PIV_ERR_UNSUPPORTED: return "not built into this engine";
    case PIV_ERR_CUDA: return "CUDA error";
    case PIV_ERR_ALLOC: return "allocation failed";
    case PIV_ERR_IO: return "I/O error";
    case PIV_ERR_STATE: return "call out of order";
    case PIV_ERR_DEVICE: return "device-side error status";
    default: return "unknown status";
    }
}

int piv_geometry_compute(const piv_params *p, piv_geometry *out)
{
    if (!p || !out) return PIV_ERR_ARG;
    return compute_geometry(*p, *out, nullptr);
}

int piv_create(const piv_params *p, piv_engine **out)
{
    if (!p || !out) return PIV_ERR_ARG;
    *out = nullptr;
    piv_engine *e = new piv_engine();
    e->p = *p;
    e->device = p->device_id;
    int rc = validate_params(e, *p);
    if (rc) {
        fprintf(stderr, "piv_create: %s\n", e->err.c_str());
        delete e;
        return rc;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        delete e;
        return PIV_ERR_CUDA;
    }
    if (e->device < 0 || e->device >= ndev || cudaSetDevice(e->device) != cudaSuccess) {
        delete e;
        return PIV_ERR_ARG;
    }
    const piv_geometry &g = e->g;
    auto bail = [&](int code) {
        fprintf(stderr, "piv_create: %s\n", e->err.c_str());
        free_all(e);
        delete e;
        return code;
    };
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(set_err(e, PIV_ERR_CUDA, "stream creation failed"));
    if (const char *v = getenv("PIV_TEST_FAIL_ALLOC")) e->fail_alloc_at = atoi(v);
    if (const char *v = getenv("PIV_TEST_FILL_CAP")) e->fill_cap = atoi(v);
    if (const char *v = getenv("PIV_TC_STAGING")) e->tc_staging = atoi(v) != 0;  // 0: direct row loads
    // frame padding: every window of both grids reads inside the buffer
    int mx = 0, my = 0;
    const int wsx[2] = {p->ws_x1, p->ws_x2}, wsy[2] = {p->ws_y1, p->ws_y2};
    const int spx[2] = {p->spacing_x1, p->spacing_x2}, spy[2] = {p->spacing_y1, p->spacing_y2};
    for (int k = 0; k < 2; ++k) {
        int xlo = -g.Nx_left[k], xhi = (g.Nx_vec[k] - 1) * spx[k] + wsx[k] - 1 - g.Nx_left[k];
        int ylo = -g.Ny_left[k], yhi = (g.Ny_vec[k] - 1) * spy[k] + wsy[k] - 1 - g.Ny_left[k];
        mx = imax(mx, imax(-xlo, xhi - (p->Nx - 1)));
        my = imax(my, imax(-ylo, yhi - (p->Ny - 1)));
    }
    e->mx = round_up(mx + 8, 16);
    e->my = my + 8;
    e->pitch = round_up(p->Nx + 2 * e->mx, 128);
    e->rows = p->Ny + 2 * e->my;
    const size_t fbytes = (size_t)e->pitch * e->rows, npix = (size_t)p->Nx * p->Ny;
    if (cudaHostAlloc((void **)&e->h_f1, npix, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void **)&e->h_f2, npix, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc((void **)&e->h_status, sizeof(int), cudaHostAllocDefault) != cudaSuccess)
        return bail(set_err(e, PIV_ERR_ALLOC, "pinned allocation failed"));
    std::memset(e->h_f1, 0, npix);
    std::memset(e->h_f2, 0, npix);
    if ((rc = dalloc(e, &e->d_f1, fbytes)) || (rc = dalloc(e, &e->d_f2, fbytes))) return bail(rc);
    if (cudaMemset(e->d_f1, 0, fbytes) != cudaSuccess || cudaMemset(e->d_f2, 0, fbytes) != cudaSuccess)
        return bail(set_err(e, PIV_ERR_CUDA, "memset failed"));
    if (p->if_mhe == 1) {
        if ((rc = dalloc(e, &e->d_stage1, npix)) || (rc = dalloc(e, &e->d_stage2, npix))) return bail(rc);
        const size_t nlev = (size_t)(e->mg.maxI + 2) * (e->mg.maxJ + 2) * 256;
        if ((rc = dalloc(e, &e->d_levels, nlev))) return bail(rc);
        if (cudaMemset(e->d_levels, 0, nlev * sizeof(int)) != cudaSuccess)
            return bail(set_err(e, PIV_ERR_CUDA, "memset failed"));
    }
    if ((rc = dalloc(e, &e->d_status, 1)) || (rc = dalloc(e, &e->d_list_n, 1))) return bail(rc);
    cudaMemset(e->d_status, 0, sizeof(int));
    const int Nps = p->Npeak_save;
    for (int k = 0; k < 2; ++k) {
        GridState &gs = e->grid[k];
        GridGeom &gg = gs.gg;
        gg.ws_x = wsx[k];
        gg.ws_y = wsy[k];
        gg.sp_x = spx[k];
        gg.sp_y = spy[k];
        gg.Nx_vec = g.Nx_vec[k];
        gg.Ny_vec = g.Ny_vec[k];
        gg.Nt_vec = g.Nt_vec[k];
        gg.bx = g.border_x[k];
        gg.by = g.border_y[k];
        gg.Nx_left = g.Nx_left[k];
        gg.Ny_left = g.Ny_left[k];
        gg.Nx_aug = g.Nx_aug[k];
        gg.Ny_aug = g.Ny_aug[k];
        gg.hfws_x = g.hfws_x[k];
        gg.hfws_y = g.hfws_y[k];
        gg.Nps = Nps;
        gg.lx1 = p->dispx_lim1;
        gg.lx2 = p->dispx_lim2;
        gg.ly1 = p->dispy_lim1;
        gg.ly2 = p->dispy_lim2;
        const size_t Nt = (size_t)gg.Nt_vec, Nc = Nt * Nps;
        if ((rc = dalloc(e, &gs.cdx, Nc)) || (rc = dalloc(e, &gs.cdy, Nc)) || (rc = dalloc(e, &gs.cv, Nc)) ||
            (rc = dalloc(e, &gs.count, Nt)) || (rc = dalloc(e, &gs.pidx, Nc)) || (rc = dalloc(e, &gs.pval, Nc)) ||
            (rc = dalloc(e, &gs.fx, Nt)) || (rc = dalloc(e, &gs.fy, Nt)) || (rc = dalloc(e, &gs.tx, Nt)) ||
            (rc = dalloc(e, &gs.ty, Nt)) || (rc = dalloc(e, &gs.fv, Nt)) || (rc = dalloc(e, &gs.tv, Nt)) ||
            (rc = dalloc(e, &gs.list, Nt)))
            return bail(rc);
        cudaMemset(gs.cdx, 0, Nc * sizeof(float));
        cudaMemset(gs.cdy, 0, Nc * sizeof(float));
        cudaMemset(gs.cv, 0, Nc);
        cudaMemset(gs.count, 0, Nt * sizeof(int));
        cudaMemset(gs.pidx, 0xff, Nc * sizeof(int));
        cudaMemset(gs.pval, 0, Nc * sizeof(float));
        cudaMemset(gs.fx, 0, Nt * sizeof(float));
        cudaMemset(gs.fy, 0, Nt * sizeof(float));
        cudaMemset(gs.fv, 0, Nt);
        // deformed frame 2: every window row/column it serves lies inside [Ny_aug][Nx_aug]
        const int need_x = (gg.Nx_vec - 1) * gg.sp_x + gg.ws_x, need_y = (gg.Ny_vec - 1) * gg.sp_y + gg.ws_y;
        if (need_x > gg.Nx_aug || need_y > gg.Ny_aug)
            return bail(set_err(e, PIV_ERR_GEOMETRY, "window extent exceeds the padded frame"));
        const bool used = (k == 0) ? p->Npass1 > 1 : p->Npass2 > 0;
        gs.def_pitch = round_up(gg.Nx_aug, 32);
        if (used) {
            const size_t nd = (size_t)gs.def_pitch * gg.Ny_aug;
            if ((rc = dalloc(e, &gs.def, nd))) return bail(rc);
            cudaMemset(gs.def, 0, nd * sizeof(float));
        }
        const char *force = getenv("PIV_XCORR_GENERIC");  // the generic kernel for every shape
        gs.generic = !xcorr_supported(gg.ws_x, gg.ws_y) || Nps > 8 || (force && atoi(force) == 1);
        if (((k == 0) ? p->Npass1 > 0 : p->Npass2 > 0) && (rc = ensure_workspace(e, k))) return bail(rc);
    }
    if ((rc = tune_xcorr(e))) return bail(rc);
    if (const char *path = getenv("PIV_XCORR_PATH")) {
        // "tc": split-BF16 tensor-core path, "tc1": single-product BF16 (precision study),
        // for every grid whose window shape the tensor-core path covers
        const int want = !strcmp(path, "tc") ? PIV_XCORR_TC_SPLIT : !strcmp(path, "tc1") ? PIV_XCORR_TC_BF16
                         : !strcmp(path, "tch") ? PIV_XCORR_TC_SPLIT_F16 : !strcmp(path, "tch1") ? PIV_XCORR_TC_F16
                                                                                               : PIV_XCORR_SIMT;
        for (int k = 0; k < 2; ++k)
            if (xcorr_tc_supported(e->grid[k].gg.ws_x, e->grid[k].gg.ws_y) && !e->grid[k].generic)
                e->grid[k].path = want;
    }
    if (getenv("PIV_TIMING") && atoi(getenv("PIV_TIMING")) == 1) {
        e->timing = true;
        for (auto &ev : e->ev) cudaEventCreate(&ev);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(set_err(e, PIV_ERR_CUDA, "initialisation failed"));
    *out = e;
    return PIV_OK;
}

int piv_destroy(piv_engine *e)
{
    if (!e) return PIV_ERR_ARG;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_all(e);
    delete e;
    return PIV_OK;
}

const char *piv_last_error(const piv_engine *e) { return e ? e->err.c_str() : "null engine"; }

int piv_get_geometry(const piv_engine *e, piv_geometry *out)
{
    if (!e || !out) return PIV_ERR_ARG;
    *out = e->g;
    return PIV_OK;
}

int piv_get_params(const piv_engine *e, piv_params *out)
{
    if (!e || !out) return PIV_ERR_ARG;
    *out = e->p;
    return PIV_OK;
}

int piv_host_images(piv_engine *e, uint8_t **f1, uint8_t **f2)
{
    if (!e) return PIV_ERR_ARG;
    if (f1) *f1 = e->h_f1;
    if (f2) *f2 = e->h_f2;
    return PIV_OK;
}

int piv_set_images(piv_engine *e, const uint8_t *f1, const uint8_t *f2, size_t pitch)
{
    if (!e || !f1 || !f2) return PIV_ERR_ARG;
    const size_t Nx = (size_t)e->p.Nx;
    if (pitch == 0) pitch = Nx;
    if (pitch < Nx) return set_err(e, PIV_ERR_ARG, "pitch smaller than Nx");
    // the pinned buffers may still feed an asynchronous upload
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "stream sync failed");
    for (int j = 0; j < e->p.Ny; ++j) {
        std::memcpy(e->h_f1 + j * Nx, f1 + j * pitch, Nx);
        std::memcpy(e->h_f2 + j * Nx, f2 + j * pitch, Nx);
    }
    e->d_in1 = e->d_in2 = nullptr;
    e->pending_slot = -1;
    return PIV_OK;
}

int piv_queue_images(piv_engine *e, const uint8_t *f1, const uint8_t *f2)
{
    if (!e || !f1 || !f2) return PIV_ERR_ARG;
    if (e->pending_slot >= 0) return set_err(e, PIV_ERR_STATE, "a queued pair has not been run yet");
    cudaSetDevice(e->device);
    const size_t npix = (size_t)e->p.Nx * e->p.Ny;
    if (!e->copy_stream) {
        CK(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
        for (int q = 0; q < 2; ++q) {
            int rc;
            if ((rc = dalloc(e, &e->d_slot[q][0], npix)) || (rc = dalloc(e, &e->d_slot[q][1], npix))) return rc;
            CK(cudaEventCreateWithFlags(&e->ev_up[q], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&e->ev_done[q], cudaEventDisableTiming));
        }
    }
    const int q = e->next_slot;
    // the slot's previous pair must have finished reading it
    if (e->slot_read[q]) CK(cudaStreamWaitEvent(e->copy_stream, e->ev_done[q], 0));
    CK(cudaMemcpyAsync(e->d_slot[q][0], f1, npix, cudaMemcpyHostToDevice, e->copy_stream));
    CK(cudaMemcpyAsync(e->d_slot[q][1], f2, npix, cudaMemcpyHostToDevice, e->copy_stream));
    CK(cudaEventRecord(e->ev_up[q], e->copy_stream));
    e->pending_slot = q;
    e->next_slot = q ^ 1;
    return PIV_OK;
}

int piv_host_alloc(size_t bytes, void **ptr)
{
    if (!ptr || bytes == 0) return PIV_ERR_ARG;
    *ptr = nullptr;
    return cudaHostAlloc(ptr, bytes, cudaHostAllocDefault) == cudaSuccess ? PIV_OK : PIV_ERR_ALLOC;
}

int piv_host_free(void *ptr)
{
    if (!ptr) return PIV_OK;
    return cudaFreeHost(ptr) == cudaSuccess ? PIV_OK : PIV_ERR_CUDA;
}

int piv_set_device_images(piv_engine *e, const uint8_t *d_f1, const uint8_t *d_f2)
{
    if (!e || (!d_f1) != (!d_f2)) return PIV_ERR_ARG;
    e->d_in1 = d_f1;
    e->d_in2 = d_f2;
    e->pending_slot = -1;
    return PIV_OK;
}

int piv_prep(piv_engine *e)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    return do_prep(e);
}

int piv_pass_grid1(piv_engine *e, int idx_pass)
{
    int rc = check_ready(e, true);
    if (rc) return rc;
    if (idx_pass < 0) return set_err(e, PIV_ERR_ARG, "negative pass index");
    if ((rc = ensure_workspace(e, 0))) return rc;
    if (idx_pass > 0 && !e->grid[0].def) {
        // the engine was created for a single grid-1 pass; deformation needs its buffer
        GridState &gs = e->grid[0];
        const size_t nd = (size_t)gs.def_pitch * gs.gg.Ny_aug;
        if ((rc = dalloc(e, &gs.def, nd))) return rc;
    }
    return do_pass(e, 0, idx_pass);
}

int piv_validate_grid1(piv_engine *e, int Npass_median, int minNneigh, float residual_threshold,
                       float insert_threshold, int Npass_smooth)
{
    (void)residual_threshold;  // read but unused by the reference as well
    int rc = check_ready(e, false);
    if (rc) return rc;
    return do_validate(e, 0, Npass_median, minNneigh, insert_threshold, Npass_smooth, 1);
}

int piv_upsample(piv_engine *e)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    return do_upsample(e);
}

int piv_pass_grid2(piv_engine *e)
{
    int rc = check_ready(e, true);
    if (rc) return rc;
    if ((rc = ensure_workspace(e, 1))) return rc;
    if (!e->grid[1].def) {
        GridState &gs = e->grid[1];
        const size_t nd = (size_t)gs.def_pitch * gs.gg.Ny_aug;
        if ((rc = dalloc(e, &gs.def, nd))) return rc;
    }
    return do_pass(e, 1, 1);
}

int piv_validate_grid2(piv_engine *e, int Npass_median, int minNneigh, float residual_threshold,
                       float insert_threshold, int Npass_smooth, int iffill)
{
    (void)residual_threshold;
    int rc = check_ready(e, false);
    if (rc) return rc;
    return do_validate(e, 1, Npass_median, minNneigh, insert_threshold, Npass_smooth, iffill == 1 ? 1 : 0);
}

int piv_run_pair(piv_engine *e)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (e->timing) {
        if ((rc = do_pair(e, true))) return rc;
        e->have_times = true;
        return PIV_OK;
    }
    // a queued upload (piv_queue_images) becomes this pair's input
    if (e->pending_slot >= 0) {
        const int q = e->pending_slot;
        CK(cudaStreamWaitEvent(e->stream, e->ev_up[q], 0));
        e->d_in1 = e->d_slot[q][0];
        e->d_in2 = e->d_slot[q][1];
        e->reading_slot = q;
        e->pending_slot = -1;
    }
    piv_engine::PairGraph *pg = nullptr;
    for (int i = 0; i < e->n_graphs; ++i)
        if (e->graphs[i].in1 == e->d_in1 && e->graphs[i].in2 == e->d_in2) pg = &e->graphs[i];
    if (!pg) {
        if (e->n_graphs == 4) {  // drop the oldest
            cudaGraphExecDestroy(e->graphs[0].exec);
            for (int i = 1; i < 4; ++i) e->graphs[i - 1] = e->graphs[i];
            e->n_graphs = 3;
        }
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        rc = do_pair(e, false);
        cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        cudaGraphExec_t exec = nullptr;
        cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
        pg = &e->graphs[e->n_graphs++];
        pg->exec = exec;
        pg->in1 = e->d_in1;
        pg->in2 = e->d_in2;
    }
    CK(cudaGraphLaunch(pg->exec, e->stream));
    if (e->reading_slot >= 0 && e->d_in1 == e->d_slot[e->reading_slot][0]) {
        CK(cudaEventRecord(e->ev_done[e->reading_slot], e->stream));
        e->slot_read[e->reading_slot] = true;
    }
    e->prepared = true;
    e->grid[0].has_pass = e->p.Npass1 > 0;
    e->grid[0].last_deformed = e->p.Npass1 > 1;
    e->grid[1].has_pass = e->p.Npass2 > 0;
    e->grid[1].last_deformed = true;
    return PIV_OK;
}

int piv_net_features(piv_engine *e, piv_net *n, float *d_out)
{
    int rc = check_ready(e, true);
    if (rc) return rc;
    if (!n || !d_out) return set_err(e, PIV_ERR_ARG, "null net or output");
    if (e->p.ws_x1 < 8 || e->p.ws_y1 < 8) return set_err(e, PIV_ERR_UNSUPPORTED, "grid-1 windows under 8 px");
    if ((rc = learned::net_reserve_features(n, e->p.Nx, e->p.Ny))) return set_err(e, rc, "feature scratch");
    return do_features(e, n, d_out);
}

int piv_run_pair_learned(piv_engine *e, piv_net *n, float max_reject_frac, float max_rms_px, int *fell_back,
                         float *reject_frac, float *rms_px)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (!n) return set_err(e, PIV_ERR_ARG, "null net");
    if (e->p.Npass2 < 1) return set_err(e, PIV_ERR_STATE, "the learned form needs grid-2 passes (Npass2 > 0)");
    if (e->p.ws_x1 < 8 || e->p.ws_y1 < 8) return set_err(e, PIV_ERR_UNSUPPORTED, "grid-1 windows under 8 px");
    if ((rc = ensure_workspace(e, 1))) return rc;
    if (e->pending_slot >= 0) return set_err(e, PIV_ERR_STATE, "a queued pair is pending: use piv_run_pair");
    GridState &g1 = e->grid[0], &g2 = e->grid[1];
    if (!g2.def) {
        const size_t nd = (size_t)g2.def_pitch * g2.gg.Ny_aug;
        if ((rc = dalloc(e, &g2.def, nd))) return rc;
    }
    if (!e->d_pred2) {
        if ((rc = dalloc(e, &e->d_pred2, 2 * (size_t)g2.gg.Nt_vec))) return rc;
        if ((rc = dalloc(e, &e->d_judge, 2))) return rc;
        if (cudaMallocHost(&e->h_judge, 2 * sizeof(float)) != cudaSuccess)
            return set_err(e, PIV_ERR_ALLOC, "pinned judge buffer");
    }
    if ((rc = learned::net_reserve(n, 1, g1.gg.Ny_vec, g1.gg.Nx_vec))) return set_err(e, rc, "network buffers");
    if ((rc = learned::net_reserve_features(n, e->p.Nx, e->p.Ny))) return set_err(e, rc, "feature scratch");
    if (!e->learned_exec || e->learned_in1 != e->d_in1 || e->learned_in2 != e->d_in2 || e->learned_net != n ||
        e->learned_gen != learned::net_generation(n)) {
        if (e->learned_exec) cudaGraphExecDestroy(e->learned_exec);
        e->learned_exec = nullptr;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        rc = do_learned(e, n);
        cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        cudaError_t ie = cudaGraphInstantiate(&e->learned_exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return set_err(e, PIV_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
        e->learned_in1 = e->d_in1;
        e->learned_in2 = e->d_in2;
        e->learned_net = n;
        e->learned_gen = learned::net_generation(n);
    }
    CK(cudaGraphLaunch(e->learned_exec, e->stream));
    CK(cudaMemcpyAsync(e->h_judge, e->d_judge, 2 * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    if ((rc = learned::net_check_status(n))) return set_err(e, rc, "predictor network: tensor-core wait timed out");
    const float rej = e->h_judge[1] / (float)g2.gg.Nt_vec;
    const float rms = std::sqrt(e->h_judge[0] / (float)g2.gg.Nt_vec);
    if (reject_frac) *reject_frac = rej;
    if (rms_px) *rms_px = rms;
    e->prepared = true;
    g1.has_pass = true;
    g1.last_deformed = false;
    g2.has_pass = true;
    g2.last_deformed = true;
    const bool fail = !(rej <= max_reject_frac) || !(rms <= max_rms_px);
    if (fell_back) *fell_back = fail ? 1 : 0;
    if (fail) return piv_run_pair(e);
    return PIV_OK;
}

int piv_synchronize(piv_engine *e)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    CK(cudaMemcpyAsync(e->h_status, e->d_status, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    if (*e->h_status) {
        const int st = *e->h_status;
        CK(cudaMemsetAsync(e->d_status, 0, sizeof(int), e->stream));
        CK(cudaStreamSynchronize(e->stream));
        return set_err(e, PIV_ERR_DEVICE, "device status 0x%x (%s)", st,
                       (st & kStatusMmaWait) ? "tensor-core MMA completion wait timed out"
                                             : "hole-fill iteration cap reached");
    }
    if (e->timing && e->have_times) {
        cudaEventElapsedTime(&e->stage_ms[0], e->ev[0], e->ev[1]);
        cudaEventElapsedTime(&e->stage_ms[1], e->ev[1], e->ev[2]);
        cudaEventElapsedTime(&e->stage_ms[2], e->ev[2], e->ev[3]);
        cudaEventElapsedTime(&e->stage_ms[4], e->ev[0], e->ev[3]);
        e->stage_ms[3] = 0.f;
    }
    return PIV_OK;
}

int piv_stage_times(piv_engine *e, float *ms5)
{
    if (!e || !ms5) return PIV_ERR_ARG;
    if (!e->timing || !e->have_times) return set_err(e, PIV_ERR_STATE, "stage timing is off (PIV_TIMING=1)");
    int rc = piv_synchronize(e);
    if (rc) return rc;
    // [0] prep+MHE, [1] grid-1 loop, [2] upsampling + grid-2 loop, [3] unused, [4] total
    for (int i = 0; i < 5; ++i) ms5[i] = e->stage_ms[i];
    return PIV_OK;
}

int piv_get_field(piv_engine *e, int sel, float *x, float *y, float *dx, float *dy, uint8_t *valid)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (sel < 0 || sel > 3) return set_err(e, PIV_ERR_ARG, "selection must be 0..3");
    if ((rc = piv_synchronize(e))) return rc;
    const int k = sel / 2;
    const bool raw = (sel % 2) == 0;
    const GridState &gs = e->grid[k];
    const size_t Nt = (size_t)gs.gg.Nt_vec, n = raw ? Nt * e->p.Npeak_save : Nt;
    if (dx) CK(cudaMemcpyAsync(dx, raw ? gs.cdx : gs.fx, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    if (dy) CK(cudaMemcpyAsync(dy, raw ? gs.cdy : gs.fy, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    if (valid) CK(cudaMemcpyAsync(valid, raw ? gs.cv : gs.fv, n, cudaMemcpyDeviceToHost, e->stream));
    if (x || y) {
        for (int j = 0; j < gs.gg.Ny_vec; ++j)
            for (int i = 0; i < gs.gg.Nx_vec; ++i) {
                // grid coordinates of X/xcorr2d_multi_grid.cu:1237-1254
                if (x) x[j * gs.gg.Nx_vec + i] = (float)(gs.gg.sp_x / 2 + i * gs.gg.sp_x);
                if (y) y[j * gs.gg.Nx_vec + i] = (float)(gs.gg.sp_y / 2 + j * gs.gg.sp_y);
            }
    }
    CK(cudaStreamSynchronize(e->stream));
    return PIV_OK;
}

int piv_field_async(piv_engine *e, int sel, int *ticket)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (sel < 0 || sel > 3 || !ticket) return set_err(e, PIV_ERR_ARG, "selection must be 0..3 and ticket non-NULL");
    int q = -1;
    for (int i = 0; i < 2 && q < 0; ++i)
        if (!e->results[i].pending) q = i;
    if (q < 0) return set_err(e, PIV_ERR_STATE, "two readbacks are pending: wait for one first");
    piv_engine::ResultSlot &r = e->results[q];
    const int k = sel / 2;
    const bool raw = (sel % 2) == 0;
    const GridState &gs = e->grid[k];
    const size_t Nt = (size_t)gs.gg.Nt_vec, n = raw ? Nt * e->p.Npeak_save : Nt;
    if (r.cap < n) {
        cudaFreeHost(r.dx);
        cudaFreeHost(r.dy);
        cudaFreeHost(r.valid);
        r.dx = r.dy = nullptr;
        r.valid = nullptr;
        r.cap = 0;
        if (cudaHostAlloc((void **)&r.dx, n * sizeof(float), cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc((void **)&r.dy, n * sizeof(float), cudaHostAllocDefault) != cudaSuccess ||
            cudaHostAlloc((void **)&r.valid, n, cudaHostAllocDefault) != cudaSuccess)
            return set_err(e, PIV_ERR_ALLOC, "cudaMallocHost ERROR! (readback slot)");
        r.cap = n;
    }
    if (!r.status && cudaHostAlloc((void **)&r.status, sizeof(int), cudaHostAllocDefault) != cudaSuccess)
        return set_err(e, PIV_ERR_ALLOC, "cudaMallocHost ERROR! (readback status)");
    if (!r.ev) CK(cudaEventCreateWithFlags(&r.ev, cudaEventDisableTiming));
    CK(cudaMemcpyAsync(r.dx, raw ? gs.cdx : gs.fx, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(r.dy, raw ? gs.cdy : gs.fy, n * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(r.valid, raw ? gs.cv : gs.fv, n, cudaMemcpyDeviceToHost, e->stream));
    // the status word of the work behind this readback travels with it, then restarts at 0
    CK(cudaMemcpyAsync(r.status, e->d_status, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemsetAsync(e->d_status, 0, sizeof(int), e->stream));
    CK(cudaEventRecord(r.ev, e->stream));
    r.sel = sel;
    r.seq = ++e->result_seq;
    r.pending = true;
    *ticket = q | (r.seq << 1);
    return PIV_OK;
}

int piv_field_wait(piv_engine *e, int ticket, float *x, float *y, float *dx, float *dy, uint8_t *valid)
{
    if (!e || ticket < 2) return PIV_ERR_ARG;
    piv_engine::ResultSlot &r = e->results[ticket & 1];
    if (!r.pending || r.seq != (ticket >> 1)) return set_err(e, PIV_ERR_STATE, "no pending readback with this ticket");
    cudaSetDevice(e->device);
    CK(cudaEventSynchronize(r.ev));
    r.pending = false;
    if (*r.status)
        return set_err(e, PIV_ERR_DEVICE, "device status 0x%x (%s)", *r.status,
                       (*r.status & kStatusMmaWait) ? "tensor-core MMA completion wait timed out"
                                                    : "hole-fill iteration cap reached");
    const GridState &gs = e->grid[r.sel / 2];
    const size_t Nt = (size_t)gs.gg.Nt_vec, n = (r.sel % 2 == 0) ? Nt * e->p.Npeak_save : Nt;
    if (dx) std::memcpy(dx, r.dx, n * sizeof(float));
    if (dy) std::memcpy(dy, r.dy, n * sizeof(float));
    if (valid) std::memcpy(valid, r.valid, n);
    if (x || y) {
        for (int j = 0; j < gs.gg.Ny_vec; ++j)
            for (int i = 0; i < gs.gg.Nx_vec; ++i) {
                // grid coordinates of X/xcorr2d_multi_grid.cu:1237-1254
                if (x) x[j * gs.gg.Nx_vec + i] = (float)(gs.gg.sp_x / 2 + i * gs.gg.sp_x);
                if (y) y[j * gs.gg.Nx_vec + i] = (float)(gs.gg.sp_y / 2 + j * gs.gg.sp_y);
            }
    }
    return PIV_OK;
}

int piv_get_peaks(piv_engine *e, int grid, int32_t *count, int32_t *pidx, float *pval)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (grid < 0 || grid > 1) return set_err(e, PIV_ERR_ARG, "grid must be 0 or 1");
    const GridState &gs = e->grid[grid];
    const size_t Nt = (size_t)gs.gg.Nt_vec, Nc = Nt * e->p.Npeak_save;
    if (count) CK(cudaMemcpyAsync(count, gs.count, Nt * 4, cudaMemcpyDeviceToHost, e->stream));
    if (pidx) CK(cudaMemcpyAsync(pidx, gs.pidx, Nc * 4, cudaMemcpyDeviceToHost, e->stream));
    if (pval) CK(cudaMemcpyAsync(pval, gs.pval, Nc * 4, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return PIV_OK;
}

int piv_set_field(piv_engine *e, int grid, const float *dx, const float *dy, const uint8_t *valid)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (grid < 0 || grid > 1) return set_err(e, PIV_ERR_ARG, "grid must be 0 or 1");
    GridState &gs = e->grid[grid];
    const size_t Nt = (size_t)gs.gg.Nt_vec;
    if (dx) CK(cudaMemcpyAsync(gs.fx, dx, Nt * 4, cudaMemcpyHostToDevice, e->stream));
    if (dy) CK(cudaMemcpyAsync(gs.fy, dy, Nt * 4, cudaMemcpyHostToDevice, e->stream));
    if (valid) CK(cudaMemcpyAsync(gs.fv, valid, Nt, cudaMemcpyHostToDevice, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return PIV_OK;
}

int piv_set_candidates(piv_engine *e, int grid, const float *dx, const float *dy, const uint8_t *valid)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (grid < 0 || grid > 1) return set_err(e, PIV_ERR_ARG, "grid must be 0 or 1");
    GridState &gs = e->grid[grid];
    const size_t Nc = (size_t)gs.gg.Nt_vec * e->p.Npeak_save;
    if (dx) CK(cudaMemcpyAsync(gs.cdx, dx, Nc * 4, cudaMemcpyHostToDevice, e->stream));
    if (dy) CK(cudaMemcpyAsync(gs.cdy, dy, Nc * 4, cudaMemcpyHostToDevice, e->stream));
    if (valid) CK(cudaMemcpyAsync(gs.cv, valid, Nc, cudaMemcpyHostToDevice, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return PIV_OK;
}

int piv_get_frames(piv_engine *e, uint8_t *f1, uint8_t *f2)
{
    int rc = check_ready(e, true);
    if (rc) return rc;
    const size_t off = (size_t)e->my * e->pitch + e->mx;
    if (f1) CK(cudaMemcpy2DAsync(f1, e->p.Nx, e->d_f1 + off, e->pitch, e->p.Nx, e->p.Ny, cudaMemcpyDeviceToHost, e->stream));
    if (f2) CK(cudaMemcpy2DAsync(f2, e->p.Nx, e->d_f2 + off, e->pitch, e->p.Nx, e->p.Ny, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return PIV_OK;
}

int piv_get_deformed(piv_engine *e, int grid, float *out)
{
    int rc = check_ready(e, false);
    if (rc) return rc;
    if (grid < 0 || grid > 1 || !out) return set_err(e, PIV_ERR_ARG, "bad arguments");
    const GridState &gs = e->grid[grid];
    if (!gs.def) return set_err(e, PIV_ERR_STATE, "no deformed frame for this grid");
    CK(cudaMemcpy2DAsync(out, (size_t)gs.gg.Nx_aug * 4, gs.def, (size_t)gs.def_pitch * 4, (size_t)gs.gg.Nx_aug * 4,
                         gs.gg.Ny_aug, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return PIV_OK;
}

int piv_debug_cc_planes(piv_engine *e, int grid, int first, int n, float *out)
{
    int rc = check_ready(e, true);
    if (rc) return rc;
    if (grid < 0 || grid > 1 || !out || n < 1) return set_err(e, PIV_ERR_ARG, "bad arguments");
    GridState &gs = e->grid[grid];
    if (!gs.has_pass) return set_err(e, PIV_ERR_STATE, "grid has not run a pass");
    if (first < 0 || first + n > gs.gg.Nt_vec) return set_err(e, PIV_ERR_ARG, "window range out of bounds");
    const size_t np = (size_t)n * gs.gg.ws_x * gs.gg.ws_y;
    float *d = nullptr;
    if ((rc = dalloc(e, &d, np))) return rc;
    rc = do_xcorr(e, grid, gs.last_deformed, first, first + n, d);
    if (!rc) {
        cudaError_t c1 = cudaMemcpyAsync(out, d, np * 4, cudaMemcpyDeviceToHost, e->stream);
        cudaError_t c2 = cudaStreamSynchronize(e->stream);
        if (c1 != cudaSuccess || c2 != cudaSuccess) rc = set_err(e, PIV_ERR_CUDA, "cc plane readback failed");
    }
    cudaFree(d);
    return rc;
}

// ---- measurement -----------------------------------------------------------------

int piv_set_xcorr_path(piv_engine *e, int grid, int path)
{
    if (!e || grid < 0 || grid > 1 || path < PIV_XCORR_SIMT || path > PIV_XCORR_TC_F16) return PIV_ERR_ARG;
    GridState &gs = e->grid[grid];
    if (path != PIV_XCORR_SIMT && !xcorr_tc_supported(gs.gg.ws_x, gs.gg.ws_y))
        return set_err(e, PIV_ERR_UNSUPPORTED, "window shape %dx%d has no tensor-core path", gs.gg.ws_x, gs.gg.ws_y);
    if (path != PIV_XCORR_SIMT && gs.generic)
        return set_err(e, PIV_ERR_UNSUPPORTED, "the tensor-core path keeps at most 8 peaks per window");
    if (gs.path != path && (e->n_graphs || e->learned_exec)) {
        cudaStreamSynchronize(e->stream);
        for (int i = 0; i < e->n_graphs; ++i) cudaGraphExecDestroy(e->graphs[i].exec);
        e->n_graphs = 0;
        if (e->learned_exec) cudaGraphExecDestroy(e->learned_exec);
        e->learned_exec = nullptr;
    }
    gs.path = path;
    return PIV_OK;
}

int piv_get_xcorr_path(const piv_engine *e, int grid, int *path)
{
    if (!e || grid < 0 || grid > 1 || !path) return PIV_ERR_ARG;
    *path = e->grid[grid].path;
    return PIV_OK;
}

int piv_xcorr_config(const piv_engine *e, int grid, int *windows_per_cta, int *threads_per_cta, float *tuned_ms)
{
    if (!e || grid < 0 || grid > 1) return PIV_ERR_ARG;
    const GridState &gs = e->grid[grid];
    if (gs.generic) {
        if (windows_per_cta) *windows_per_cta = 1;
        if (threads_per_cta) *threads_per_cta = kGenericThreads;
        if (tuned_ms) *tuned_ms = 0.f;
        return PIV_OK;
    }
    if (!xcorr_variant_shape(gs.gg.ws_x, gs.gg.ws_y, gs.variant, windows_per_cta, threads_per_cta))
        return PIV_ERR_UNSUPPORTED;
    if (tuned_ms) *tuned_ms = gs.n_tuned ? gs.tuned_ms[gs.variant] : 0.f;
    return PIV_OK;
}

int piv_get_stream(const piv_engine *e, void **stream)
{
    if (!e || !stream) return PIV_ERR_ARG;
    *stream = (void *)e->stream;
    return PIV_OK;
}

int piv_kernel_launches_per_pair(const piv_engine *e, int *n)
{
    if (!e || !n) return PIV_ERR_ARG;
    const piv_params &p = e->p;
    auto val = [&](int npm, int nps) { return (npm > 0 ? npm : 1) + 1 /* fill */ + nps; };
    int k = (p.if_mhe == 1) ? 4 : 0;
    for (int j = 0; j < p.Npass1; ++j)
        k += (j > 0 ? 1 : 0) + e->g.Nsec[0] + val(p.Npass1_median, p.Npass1_smooth);
    if (p.Npass2 > 0) k += 1 + p.Npass2 * (1 + e->g.Nsec[1] + val(p.Npass2_median, p.Npass2_smooth));
    *n = k;
    return PIV_OK;
}

int piv_time_stage(piv_engine *e, int which, int reps, float *ms)
{
    int rc = check_ready(e, which != 4);
    if (rc) return rc;
    if (!ms || reps < 1 || which < 0 || which > 4) return set_err(e, PIV_ERR_ARG, "bad arguments");
    if (which == 4 && e->p.if_mhe != 1) return set_err(e, PIV_ERR_STATE, "MHE is off");
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, e->stream));
    for (int r = 0; r < reps && !rc; ++r) {
        switch (which) {
        case 0: rc = do_xcorr(e, 0, e->grid[0].last_deformed, 0, 0, nullptr); break;
        case 1: rc = do_xcorr(e, 1, true, 0, 0, nullptr); break;
        case 2: rc = do_deform(e, 1); break;
        case 3:
            rc = do_validate(e, 1, e->p.Npass2_median, e->p.minNneigh_p2, e->p.insert_threshold_p2,
                             e->p.Npass2_smooth, 1);
            break;
        case 4: {
            const uint8_t *src = e->d_in1 ? e->d_in1 : e->d_stage1;
            cudaError_t c = launch_mhe(e->mg, src, e->p.Nx, e->d_levels, e->d_f1, e->pitch, e->mx, e->my, e->stream);
            if (c != cudaSuccess) rc = set_err(e, PIV_ERR_CUDA, "MHE: %s", cudaGetErrorString(c));
            break;
        }
        }
    }
    CK(cudaEventRecord(b, e->stream));
    CK(cudaEventSynchronize(b));
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = t / reps;
    return rc;
}

}  // extern "C"

namespace {
// 8 independent FMA chains per thread so that the FMA pipes, not latency, bound it.
__global__ void fp32_peak_kernel(float *out, int iters, float s)
{
    float a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fmaf(a0, s, 0.5f);
            a1 = fmaf(a1, s, 0.5f);
            a2 = fmaf(a2, s, 0.5f);
            a3 = fmaf(a3, s, 0.5f);
            a4 = fmaf(a4, s, 0.5f);
            a5 = fmaf(a5, s, 0.5f);
            a6 = fmaf(a6, s, 0.5f);
            a7 = fmaf(a7, s, 0.5f);
        }
    }
    const float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.678f) out[0] = r;  // keeps the chains live
}
}  // namespace

extern "C" {

int piv_probe_fp32_peak(float *tflops)
{
    if (!tflops) return PIV_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PIV_ERR_CUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float *d = nullptr;
    if (cudaMalloc(&d, 4) != cudaSuccess) return PIV_ERR_ALLOC;
    const int threads = 512, blocks = sms * 4, iters = 4096;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fp32_peak_kernel<<<blocks, threads>>>(d, iters / 8, 0.999f);  // warm-up
    cudaEventRecord(a);
    fp32_peak_kernel<<<blocks, threads>>>(d, iters, 0.999f);
    cudaEventRecord(b);
    cudaError_t c = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (c != cudaSuccess || ms <= 0) return PIV_ERR_CUDA;
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    *tflops = (float)(flops / (ms * 1e-3) / 1e12);
    return PIV_OK;
}

// ---- standalone MHE ------------------------------------------------------------

int piv_mhe_create(int Nx, int Ny, int ws, float thresh, piv_mhe **out)
{
    if (!out) return PIV_ERR_ARG;
    *out = nullptr;
    piv_mhe *m = new piv_mhe();
    if (!mhe_geometry(Nx, Ny, ws, thresh, m->mg)) {
        delete m;
        return PIV_ERR_ARG;
    }
    cudaGetDevice(&m->device);
    const size_t nlev = (size_t)(m->mg.maxI + 2) * (m->mg.maxJ + 2) * 256 * sizeof(int);
    if (cudaMalloc((void **)&m->d_levels, nlev) != cudaSuccess) {
        delete m;
        return PIV_ERR_ALLOC;
    }
    if (cudaMemset(m->d_levels, 0, nlev) != cudaSuccess) {
        cudaFree(m->d_levels);
        delete m;
        return PIV_ERR_CUDA;
    }
    *out = m;
    return PIV_OK;
}

int piv_mhe_process(piv_mhe *m, const uint8_t *d_in, uint8_t *d_out, void *stream)
{
    if (!m || !d_in || !d_out) return PIV_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const MheGeom &g = m->mg;
    if (g.width != g.Nx || g.height != g.Ny) {
        if (cudaMemsetAsync(d_out, 0, (size_t)g.Nx * g.Ny, s) != cudaSuccess) return PIV_ERR_CUDA;
    }
    if (launch_mhe(g, d_in, g.Nx, m->d_levels, d_out, g.Nx, 0, 0, s) != cudaSuccess) return PIV_ERR_CUDA;
    return PIV_OK;
}

int piv_mhe_destroy(piv_mhe *m)
{
    if (!m) return PIV_ERR_ARG;
    cudaFree(m->d_levels);
    delete m;
    return PIV_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------
// Batches of pairs of uneven size and window shape (piv_batch_*; no reference
// counterpart).  One engine per pair holds its frames, geometry and fields; the batch
// runs their pass loop together: per pass, the pairs' deformations on parallel graph
// branches, then ONE persistent correlation launch per (grid, window shape, top-K width)
// over all pairs that share it, then the pairs' validations on parallel branches.  The
// whole loop is one captured CUDA graph.  The first run autotunes the tile variant of
// every shape group on the batch's own data.
// ------------------------------------------------------------------------------
struct piv_batch {
    int n = 0, device = 0;
    std::vector<piv_engine *> eng;
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> workers;
    std::vector<cudaEvent_t> ev_join;
    cudaEvent_t ev_fork = nullptr;
    struct Group {
        int k = 0;
        bool deformed = false;
        int wsx = 0, wsy = 0, K = 4;
        std::vector<int> pairs;
        std::vector<XcorrBatch> chunks[2];  // per tile variant: launches of <= kBatchMaxPairs pairs
        int n_variants = 0, variant = 0;
        float tuned_ms[2] = {};
    };
    std::vector<Group> groups;
    std::vector<int> paths;  // each engine's (grid 1, grid 2) correlation path the groups were built for
    bool tuned = false;
    cudaGraphExec_t exec = nullptr;
    std::vector<const uint8_t *> graph_in;
    std::string err;
};

namespace {

int batch_err(piv_batch *b, int code, const char *fmt, ...)
{
    if (b) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        b->err = buf;
    }
    return code;
}

#define BCK(call)                                                                                              \
    do {                                                                                                       \
        cudaError_t _e = (call);                                                                               \
        if (_e != cudaSuccess) return batch_err(b, PIV_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));      \
    } while (0)

void batch_free(piv_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (cudaStream_t s : b->workers) cudaStreamDestroy(s);
    for (cudaEvent_t ev : b->ev_join) cudaEventDestroy(ev);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (piv_engine *e : b->eng)
        if (e) piv_destroy(e);
}

// the groups' argument tables (the engines' buffers are fixed after creation).  Only
// pairs on the FP32 SIMT path join a group; a pair whose engine is set to a tensor-core
// path runs its own tensor-core launch on its branch of the batch graph.
int batch_build_groups(piv_batch *b)
{
    b->groups.clear();
    b->paths.clear();
    for (piv_engine *e : b->eng) {
        b->paths.push_back(e->grid[0].path);
        b->paths.push_back(e->grid[1].path);
    }
    for (int k = 0; k < 2; ++k)
        for (int d = 0; d < 2; ++d) {
            for (int i = 0; i < b->n; ++i) {
                piv_engine *e = b->eng[i];
                const int np = k ? e->p.Npass2 : e->p.Npass1;
                if (np == 0) continue;
                const bool deformed = d == 1;
                if (!deformed && k == 1) continue;   // grid 2 passes are all deformed
                if (deformed && k == 0 && np < 2) continue;
                const GridState &gs = e->grid[k];
                if (gs.path != PIV_XCORR_SIMT || gs.generic) continue;
                const int K = gs.gg.Nps <= 4 ? 4 : 8;
                piv_batch::Group *grp = nullptr;
                for (auto &g : b->groups)
                    if (g.k == k && g.deformed == deformed && g.wsx == gs.gg.ws_x && g.wsy == gs.gg.ws_y && g.K == K)
                        grp = &g;
                if (!grp) {
                    b->groups.emplace_back();
                    grp = &b->groups.back();
                    grp->k = k;
                    grp->deformed = deformed;
                    grp->wsx = gs.gg.ws_x;
                    grp->wsy = gs.gg.ws_y;
                    grp->K = K;
                    grp->n_variants = std::min(2, xcorr_batch_variants(gs.gg.ws_x, gs.gg.ws_y));
                }
                grp->pairs.push_back(i);
            }
        }
    for (auto &g : b->groups) {
        if (g.n_variants < 1) return batch_err(b, PIV_ERR_UNSUPPORTED, "window shape %dx%d has no batch launch", g.wsx, g.wsy);
        for (int v = 0; v < g.n_variants; ++v) {
            const int B = xcorr_batch_windows_per_cta(g.wsx, g.wsy, v);
            for (size_t c0 = 0; c0 < g.pairs.size(); c0 += kBatchMaxPairs) {
                g.chunks[v].emplace_back();
                XcorrBatch &xb = g.chunks[v].back();
                memset(&xb, 0, sizeof(xb));
                xb.n = (int)std::min(g.pairs.size() - c0, (size_t)kBatchMaxPairs);
                xb.first[0] = 0;
                for (int j = 0; j < xb.n; ++j) {
                    xb.pairs[j] = xcorr_args(b->eng[g.pairs[c0 + j]], g.k);
                    const int nw = xb.pairs[j].w_end - (xb.pairs[j].w_first & ~1);
                    xb.first[j + 1] = xb.first[j] + (nw + B - 1) / B;
                }
                xb.items = xb.first[xb.n];
            }
        }
    }
    return PIV_OK;
}

int batch_launch_group(piv_batch *b, const piv_batch::Group &g, int variant)
{
    for (const XcorrBatch &xb : g.chunks[variant]) {
        const char *why = nullptr;
        cudaError_t c = launch_xcorr_batch(g.wsx, g.wsy, variant, xb, g.deformed, g.K, b->stream, &why);
        if (c != cudaSuccess)
            return batch_err(b, PIV_ERR_CUDA, "batch correlation: %s", why ? why : cudaGetErrorString(c));
    }
    return PIV_OK;
}

// The pass loop of every pair, queued on the batch stream with per-pair stages on the
// worker streams (fork / join through events; inside a capture these become parallel
// graph branches).
int batch_enqueue(piv_batch *b)
{
    const int W = (int)b->workers.size();
    std::vector<cudaStream_t> own(b->n);
    for (int i = 0; i < b->n; ++i) {
        own[i] = b->eng[i]->stream;
        b->eng[i]->stream = b->workers[i % W];
    }
    auto restore = [&]() {
        for (int i = 0; i < b->n; ++i) b->eng[i]->stream = own[i];
    };
    auto fork = [&]() -> int {
        BCK(cudaEventRecord(b->ev_fork, b->stream));
        for (cudaStream_t w : b->workers) BCK(cudaStreamWaitEvent(w, b->ev_fork, 0));
        return PIV_OK;
    };
    auto join = [&]() -> int {
        for (int w = 0; w < W; ++w) {
            BCK(cudaEventRecord(b->ev_join[w], b->workers[w]));
            BCK(cudaStreamWaitEvent(b->stream, b->ev_join[w], 0));
        }
        return PIV_OK;
    };
    auto per_pair = [&](auto fn) -> int {
        int rc = fork();
        for (int i = 0; !rc && i < b->n; ++i) {
            rc = fn(b->eng[i]);
            if (rc) b->err = b->eng[i]->err;
        }
        const int rj = join();
        return rc ? rc : rj;
    };
    int rc = per_pair([](piv_engine *e) { return do_prep(e); });
    const piv_params &p0 = b->eng[0]->p;
    for (int k = 0; !rc && k < 2; ++k) {
        const int np = k ? p0.Npass2 : p0.Npass1;
        if (np == 0) continue;
        if (k == 1) rc = per_pair([](piv_engine *e) { return do_upsample(e); });
        for (int j = 0; !rc && j < np; ++j) {
            const bool deformed = !(k == 0 && j == 0);
            rc = per_pair([&](piv_engine *e) -> int {
                GridState &gs = e->grid[k];
                if (!deformed) {
                    CK(cudaMemsetAsync(gs.fx, 0, sizeof(float) * gs.gg.Nt_vec, e->stream));
                    CK(cudaMemsetAsync(gs.fy, 0, sizeof(float) * gs.gg.Nt_vec, e->stream));
                } else {
                    const int r = do_deform(e, k);
                    if (r) return r;
                }
                // a pair on a tensor-core path or the generic-size kernel correlates on its own branch
                return gs.path == PIV_XCORR_SIMT && !gs.generic ? PIV_OK : do_xcorr(e, k, deformed, 0, 0, nullptr);
            });
            for (auto &g : b->groups)
                if (!rc && g.k == k && g.deformed == deformed) rc = batch_launch_group(b, g, g.variant);
            if (rc) break;
            rc = per_pair([&](piv_engine *e) {
                const piv_params &p = e->p;
                return k ? do_validate(e, 1, p.Npass2_median, p.minNneigh_p2, p.insert_threshold_p2, p.Npass2_smooth, 1)
                         : do_validate(e, 0, p.Npass1_median, p.minNneigh_p1, p.insert_threshold_p1, p.Npass1_smooth, 1);
            });
        }
    }
    restore();
    return rc;
}

// each group's tile variant, timed on the batch's own data after one eager run
int batch_tune(piv_batch *b)
{
    int rc = batch_enqueue(b);
    if (rc) return rc;
    BCK(cudaStreamSynchronize(b->stream));
    if (const char *fixed = getenv("PIV_BATCH_VARIANT")) {
        // every group's variant by index (taken modulo the group's count), no timing
        const int v = atoi(fixed);
        if (v < 0) return batch_err(b, PIV_ERR_ARG, "PIV_BATCH_VARIANT wants a non-negative index");
        for (auto &g : b->groups) g.variant = v % g.n_variants;
        return PIV_OK;
    }
    if (!autotune_enabled()) return PIV_OK;
    cudaEvent_t t0, t1;
    BCK(cudaEventCreate(&t0));
    BCK(cudaEventCreate(&t1));
    for (auto &g : b->groups) {
        float best = 0.f;
        for (int v = 0; v < g.n_variants; ++v) {
            if ((rc = batch_launch_group(b, g, v))) break;  // warm-up
            BCK(cudaEventRecord(t0, b->stream));
            for (int r = 0; r < 3 && !rc; ++r) rc = batch_launch_group(b, g, v);
            BCK(cudaEventRecord(t1, b->stream));
            BCK(cudaEventSynchronize(t1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            g.tuned_ms[v] = ms / 3.f;
            if (v == 0 || g.tuned_ms[v] < best) {
                best = g.tuned_ms[v];
                g.variant = v;
            }
        }
        if (rc) break;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return rc;
}

}  // namespace

extern "C" {

int piv_batch_create(const piv_params *params, int n, piv_batch **out)
{
    if (!params || n < 1 || !out) return PIV_ERR_ARG;
    *out = nullptr;
    for (int i = 1; i < n; ++i)
        if (params[i].Npass1 != params[0].Npass1 || params[i].Npass2 != params[0].Npass2) return PIV_ERR_ARG;
    piv_batch *b = new piv_batch;
    b->n = n;
    b->eng.assign(n, nullptr);
    cudaGetDevice(&b->device);
    int rc = PIV_OK;
    for (int i = 0; i < n && !rc; ++i) {
        piv_params p = params[i];
        p.device_id = b->device;
        rc = piv_create(&p, &b->eng[i]);
        if (rc) batch_err(b, rc, "pair %d: engine creation failed", i);
    }
    if (!rc) {
        const int W = std::min(n, 8);
        b->workers.resize(W);
        b->ev_join.resize(W);
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess)
            rc = PIV_ERR_CUDA;
        for (int w = 0; w < W && !rc; ++w)
            if (cudaStreamCreateWithFlags(&b->workers[w], cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&b->ev_join[w], cudaEventDisableTiming) != cudaSuccess)
                rc = PIV_ERR_CUDA;
    }
    if (!rc) {
        // every pass buffer up front (deformed frames of both grids)
        for (int i = 0; i < n && !rc; ++i)
            for (int k = 0; k < 2 && !rc; ++k) {
                GridState &gs = b->eng[i]->grid[k];
                const int np = k ? b->eng[i]->p.Npass2 : b->eng[i]->p.Npass1;
                if (!gs.def && (k == 1 ? np > 0 : np > 1))
                    rc = dalloc(b->eng[i], &gs.def, (size_t)gs.def_pitch * gs.gg.Ny_aug);
            }
    }
    if (!rc) rc = batch_build_groups(b);
    if (rc) {
        batch_free(b);
        delete b;
        return rc;
    }
    *out = b;
    return PIV_OK;
}

int piv_batch_destroy(piv_batch *b)
{
    if (!b) return PIV_ERR_ARG;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_free(b);
    delete b;
    return PIV_OK;
}

const char *piv_batch_last_error(const piv_batch *b) { return b ? b->err.c_str() : "null batch"; }

int piv_batch_engine(piv_batch *b, int i, piv_engine **e)
{
    if (!b || !e || i < 0 || i >= b->n) return PIV_ERR_ARG;
    *e = b->eng[i];
    return PIV_OK;
}

int piv_batch_run(piv_batch *b)
{
    if (!b) return PIV_ERR_ARG;
    cudaSetDevice(b->device);
    for (piv_engine *e : b->eng)
        if (e->pending_slot >= 0) return batch_err(b, PIV_ERR_STATE, "a queued pair is pending on an engine");
    int rc;
    std::vector<int> paths;
    for (piv_engine *e : b->eng) {
        paths.push_back(e->grid[0].path);
        paths.push_back(e->grid[1].path);
    }
    if (paths != b->paths) {
        // a member engine's correlation path changed: regroup, retune, recapture
        if ((rc = batch_build_groups(b))) return rc;
        b->tuned = false;
        if (b->exec) cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (!b->tuned) {
        if ((rc = batch_tune(b))) return rc;
        b->tuned = true;
    }
    std::vector<const uint8_t *> in;
    for (piv_engine *e : b->eng) {
        in.push_back(e->d_in1);
        in.push_back(e->d_in2);
    }
    if (!b->exec || in != b->graph_in) {
        if (b->exec) cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
        cudaGraph_t g = nullptr;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        rc = batch_enqueue(b);
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return batch_err(b, PIV_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        cudaError_t ie = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return batch_err(b, PIV_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
        b->graph_in = in;
    }
    BCK(cudaGraphLaunch(b->exec, b->stream));
    for (piv_engine *e : b->eng) {
        e->prepared = true;
        e->grid[0].has_pass = e->p.Npass1 > 0;
        e->grid[0].last_deformed = e->p.Npass1 > 1;
        e->grid[1].has_pass = e->p.Npass2 > 0;
        e->grid[1].last_deformed = true;
    }
    return PIV_OK;
}

int piv_batch_synchronize(piv_batch *b)
{
    if (!b) return PIV_ERR_ARG;
    cudaSetDevice(b->device);
    BCK(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < b->n; ++i) {
        int rc = piv_synchronize(b->eng[i]);
        if (rc) return batch_err(b, rc, "pair %d: %s", i, b->eng[i]->err.c_str());
    }
    return PIV_OK;
}

int piv_batch_stream(const piv_batch *b, void **stream)
{
    if (!b || !stream) return PIV_ERR_ARG;
    *stream = b->stream;
    return PIV_OK;
}

int piv_batch_groups(const piv_batch *b, int max, int *wsx, int *wsy, int *grid, int *deformed, int *pairs,
                     int *variant, int *windows_per_cta, int *n_groups)
{
    if (!b || !n_groups) return PIV_ERR_ARG;
    *n_groups = (int)b->groups.size();
    for (int i = 0; i < *n_groups && i < max; ++i) {
        const auto &g = b->groups[i];
        if (wsx) wsx[i] = g.wsx;
        if (wsy) wsy[i] = g.wsy;
        if (grid) grid[i] = g.k;
        if (deformed) deformed[i] = g.deformed ? 1 : 0;
        if (pairs) pairs[i] = (int)g.pairs.size();
        if (variant) variant[i] = g.variant;
        if (windows_per_cta) windows_per_cta[i] = xcorr_batch_windows_per_cta(g.wsx, g.wsy, g.variant);
    }
    return PIV_OK;
}

}  // extern "C"
