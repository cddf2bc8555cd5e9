// piv_xcorr2d -- command-line driver, a Linux replacement for X/main.cpp of
// xinzhixue/PIV_xcorr2d_V1.0 (X/ = xcorr2d_V1.0/) on top of the C-ABI.
//
//   piv_xcorr2d [Parameter.dat] [--overlap] [--resume] [--npy] [--shard r/W]
//
// Reads the 50-line parameter file (default ./Parameter.dat), the image-pair index list,
// and for every index NNNN the frames prefix1+NNNN+suffix1 and prefix2+NNNN+suffix2
// (8-bit TIFF).  Runs the grid-1/grid-2 pass loop of X/main.cpp:288-326 on the GPU and
// writes the Tecplot files of X/main.cpp:327-376 (grid-1 raw and filtered, grid-2 raw,
// filtered and median-only) into the result folder, which is created if missing.
// Messages follow the reference's; exit status 0 = "NO ERROR!", 1 = "ERROR!".
//
// --overlap: while the GPU processes the current pair, reads the next pair's frames into
// a second pinned buffer pair and queues their upload (piv_queue_images, overlapping the
// computation), and writes the previous pair's files on a host thread.
// --resume:  skips pairs whose output files all exist already.
// --npy:     also writes every field as a float32 .npy sidecar next to its .dat file
//            ([Ny_vec][Nx_vec][2] filtered, [Ny_vec][Nx_vec][Npeak_save][2] raw).
// --shard r/W: processes pairs r, r+W, r+2W, ... of the list (replicas: run W processes,
//            one per GPU, e.g. with CUDA_VISIBLE_DEVICES=r; pairs are independent).
#include <sys/stat.h>
#include <sys/types.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "piv_b200.h"

namespace {

bool file_exists(const std::string &p)
{
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

bool make_dirs(const std::string &p)
{
    std::string cur;
    for (size_t i = 0; i < p.size(); ++i) {
        cur.push_back(p[i]);
        if ((p[i] == '/' || i + 1 == p.size()) && !cur.empty()) {
            struct stat st;
            if (stat(cur.c_str(), &st) != 0 && mkdir(cur.c_str(), 0775) != 0) return false;
        }
    }
    return true;
}

std::string frame_path(const char *prefix, int idx, const char *suffix)
{
    char num[32];
    snprintf(num, sizeof(num), "%04d", idx);
    return std::string(prefix) + num + suffix;
}

// The five output files of one pair, from host copies of the fields.
struct PairOutput {
    int idx = 0;
    std::vector<float> raw1x, raw1y, f1x, f1y, raw2x, raw2y, f2x, f2y, m2x, m2y;
};

int fetch(piv_engine *e, const piv_params &p, const piv_geometry &g, PairOutput &o)
{
    const size_t n1 = (size_t)g.Nt_vec[0], n2 = (size_t)g.Nt_vec[1], k = (size_t)p.Npeak_save;
    o.raw1x.resize(n1 * k);
    o.raw1y.resize(n1 * k);
    o.f1x.resize(n1);
    o.f1y.resize(n1);
    int rc = piv_get_field(e, 0, nullptr, nullptr, o.raw1x.data(), o.raw1y.data(), nullptr);
    if (!rc) rc = piv_get_field(e, 1, nullptr, nullptr, o.f1x.data(), o.f1y.data(), nullptr);
    if (rc || p.Npass2 <= 0) return rc;
    o.raw2x.resize(n2 * k);
    o.raw2y.resize(n2 * k);
    o.f2x.resize(n2);
    o.f2y.resize(n2);
    o.m2x.resize(n2);
    o.m2y.resize(n2);
    rc = piv_get_field(e, 2, nullptr, nullptr, o.raw2x.data(), o.raw2y.data(), nullptr);
    if (!rc) rc = piv_get_field(e, 3, nullptr, nullptr, o.f2x.data(), o.f2y.data(), nullptr);
    // X/main.cpp:363: median test only, no smoothing, no fill
    if (!rc) rc = piv_validate_grid2(e, p.Npass2_median, p.minNneigh_p2, p.residual_threshold_p2,
                                     p.insert_threshold_p2, 0, 0);
    if (!rc) rc = piv_get_field(e, 3, nullptr, nullptr, o.m2x.data(), o.m2y.data(), nullptr);
    return rc;
}

int n_kinds(const piv_params &p) { return p.Npass2 > 0 ? 5 : 2; }

bool outputs_exist(const piv_params &p, const char *folder, int idx)
{
    char path[4096];
    for (int kind = 0; kind < n_kinds(p); ++kind)
        if (piv_output_name(&p, folder, idx, kind, path, sizeof(path)) || !file_exists(path)) return false;
    return true;
}

int write_outputs(const piv_params &p, const piv_geometry &g, const char *folder, const PairOutput &o, bool npy)
{
    char path[4096];
    int rc = 0;
    auto w = [&](int kind, int grid, bool raw, const std::vector<float> &x, const std::vector<float> &y) {
        if (rc) return;
        if ((rc = piv_output_name(&p, folder, o.idx, kind, path, sizeof(path)))) return;
        const int spx = grid ? p.spacing_x2 : p.spacing_x1, spy = grid ? p.spacing_y2 : p.spacing_y1;
        rc = piv_tecplot_write_arrays(path, g.Nx_vec[grid], g.Ny_vec[grid], spx, spy, raw ? 1 : 0, p.Npeak_save,
                                      x.data(), y.data());
        if (rc || !npy) return;
        std::string np(path);
        if (np.size() > 4 && np.compare(np.size() - 4, 4, ".dat") == 0) np.resize(np.size() - 4);
        np += ".npy";
        std::vector<float> xy(x.size() * 2);
        for (size_t i = 0; i < x.size(); ++i) {
            xy[2 * i] = x[i];
            xy[2 * i + 1] = y[i];
        }
        const int shape_raw[4] = {g.Ny_vec[grid], g.Nx_vec[grid], p.Npeak_save, 2};
        const int shape_f[3] = {g.Ny_vec[grid], g.Nx_vec[grid], 2};
        rc = raw ? piv_npy_write_f32(np.c_str(), xy.data(), 4, shape_raw)
                 : piv_npy_write_f32(np.c_str(), xy.data(), 3, shape_f);
    };
    w(0, 0, true, o.raw1x, o.raw1y);
    w(1, 0, false, o.f1x, o.f1y);
    if (p.Npass2 > 0) {
        w(2, 1, true, o.raw2x, o.raw2y);
        w(3, 1, false, o.f2x, o.f2y);
        w(4, 1, false, o.m2x, o.m2y);
    }
    if (rc) printf("Error occurs while the vector file is being written.\n");
    return rc;
}

}  // namespace

int main(int argc, char **argv)
{
    const char *param_path = "Parameter.dat";
    bool overlap = false, resume = false, npy = false;
    int shard_r = 0, shard_w = 1;
    for (int i = 1; i < argc; ++i) {
        if (!strcmp(argv[i], "--overlap")) overlap = true;
        else if (!strcmp(argv[i], "--resume")) resume = true;
        else if (!strcmp(argv[i], "--npy")) npy = true;
        else if (!strcmp(argv[i], "--shard") && i + 1 < argc) {
            if (sscanf(argv[++i], "%d/%d", &shard_r, &shard_w) != 2 || shard_w < 1 || shard_r < 0 ||
                shard_r >= shard_w) {
                printf("--shard expects r/W with 0 <= r < W\n");
                return 1;
            }
        } else param_path = argv[i];
    }
    piv_params p;
    piv_paths paths;
    int rc = piv_params_read(param_path, &p, &paths);
    if (rc == PIV_ERR_IO) {
        printf("Can't open parameter file!\n");
        return 1;
    }
    if (rc) {
        printf("Parameter missing in Parameter.dat!\n");
        return 1;
    }
    std::vector<int> pairs;
    {
        FILE *f = fopen(paths.dir_index, "rb");
        if (!f) {
            printf("Can't open image pair index file!\n");
            return 1;
        }
        char line[256];
        while (fgets(line, sizeof(line), f)) pairs.push_back(atoi(line));
        fclose(f);
    }
    if (pairs.empty()) {
        printf("No image pair index detected!\n");
        return 1;
    }
    if (shard_w > 1) {
        std::vector<int> mine;
        for (size_t i = (size_t)shard_r; i < pairs.size(); i += (size_t)shard_w) mine.push_back(pairs[i]);
        pairs.swap(mine);
    }
    if (resume) {
        std::vector<int> todo;
        for (int idx : pairs)
            if (!outputs_exist(p, paths.folder_result, idx)) todo.push_back(idx);
        printf("Resuming: %zu of %zu pairs have outputs already\n", pairs.size() - todo.size(), pairs.size());
        pairs.swap(todo);
        if (pairs.empty()) {
            printf("NO ERROR!\n");
            return 0;
        }
    }
    if (pairs.empty()) {
        printf("NO ERROR!\n");
        return 0;
    }
    if (!make_dirs(paths.folder_result)) {
        printf("Folder creation not successful!\n");
        return 1;
    }
    const std::string first = frame_path(paths.prefix_f1, pairs[0], paths.suffix_f1);
    if (!file_exists(first)) {
        printf("An image for crosss-correlation is missing!\n");
        return 1;
    }
    piv_engine *e = nullptr;
    if ((rc = piv_create(&p, &e))) {
        printf("Initialization of xcorr2d_multi class failed! (%s)\n", piv_status_string(rc));
        return 1;
    }
    piv_geometry g;
    piv_get_geometry(e, &g);
    const size_t npx = (size_t)p.Nx * p.Ny;
    // frame buffers: two pinned pairs (the engine's own and one more) so that in --overlap
    // mode the next pair is read while the current one is computed, then its upload is
    // queued (piv_queue_images) while the GPU still works
    uint8_t *hb[2][2] = {};
    piv_host_images(e, &hb[0][0], &hb[0][1]);
    void *extra1 = nullptr, *extra2 = nullptr;
    if (overlap && (piv_host_alloc(npx, &extra1) || piv_host_alloc(npx, &extra2))) {
        printf("cudaMallocHost ERROR!\n");
        piv_host_free(extra1);
        piv_destroy(e);
        return 1;
    }
    hb[1][0] = static_cast<uint8_t *>(extra1);
    hb[1][1] = static_cast<uint8_t *>(extra2);
    std::vector<uint8_t> next1(overlap ? 0 : npx), next2(overlap ? 0 : npx);
    bool status = true;
    std::thread writer;
    int writer_rc = 0;
    PairOutput pending;

    auto read_pair = [&](int idx, uint8_t *a, uint8_t *b) -> int {
        const std::string p1 = frame_path(paths.prefix_f1, idx, paths.suffix_f1);
        const std::string p2 = frame_path(paths.prefix_f2, idx, paths.suffix_f2);
        if (!file_exists(p1) || !file_exists(p2)) return PIV_ERR_IO;
        int r = piv_tiff_read8(p1.c_str(), a, p.Nx, p.Ny);
        return r ? r : piv_tiff_read8(p2.c_str(), b, p.Nx, p.Ny);
    };

    int have_next;
    if (overlap) {
        have_next = read_pair(pairs[0], hb[0][0], hb[0][1]) == PIV_OK ? 1 : -1;
        if (have_next > 0 && (rc = piv_queue_images(e, hb[0][0], hb[0][1]))) have_next = -1;
    } else {
        have_next = read_pair(pairs[0], next1.data(), next2.data()) == PIV_OK ? 1 : -1;
    }
    for (size_t i = 0; i < pairs.size(); ++i) {
        auto begin = std::chrono::steady_clock::now();
        printf("Processing pair %d: %zu out of %zu\n", pairs[i], i + 1, pairs.size());
        if (have_next < 0) {
            printf("An image for crosss-correlation is missing!\n");
            status = false;
            break;
        }
        if ((!overlap && (rc = piv_set_images(e, next1.data(), next2.data(), 0))) || (rc = piv_run_pair(e))) {
            printf("xcor pair processing failed: %s\n", piv_last_error(e));
            status = false;
            break;
        }
        // while the GPU works: read the next pair's frames and queue their upload
        int next_rc = 0;
        if (i + 1 < pairs.size() && overlap) {
            // the other buffer pair fed pair i-1, whose upload finished before it ran
            uint8_t *a = hb[(i + 1) & 1][0], *b = hb[(i + 1) & 1][1];
            next_rc = read_pair(pairs[i + 1], a, b);
            if (next_rc == PIV_OK) next_rc = piv_queue_images(e, a, b);
        }
        PairOutput out;
        out.idx = pairs[i];
        rc = fetch(e, p, g, out);
        if (i + 1 < pairs.size() && !overlap) next_rc = read_pair(pairs[i + 1], next1.data(), next2.data());
        have_next = next_rc == PIV_OK ? 1 : -1;
        if (rc) {
            printf("xcor pair processing failed: %s\n", piv_last_error(e));
            status = false;
            break;
        }
        if (writer.joinable()) {
            writer.join();
            if (writer_rc) {
                status = false;
                break;
            }
        }
        if (overlap) {
            pending = std::move(out);
            writer = std::thread([&] { writer_rc = write_outputs(p, g, paths.folder_result, pending, npy); });
        } else if (write_outputs(p, g, paths.folder_result, out, npy)) {
            status = false;
            break;
        }
        const double secs =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
        printf("Done! %g seconds\n", secs);
    }
    if (writer.joinable()) {
        writer.join();
        if (writer_rc) status = false;
    }
    piv_destroy(e);
    piv_host_free(extra1);
    piv_host_free(extra2);
    printf(status ? "NO ERROR!\n" : "ERROR!\n");
    return status ? 0 : 1;
}
