// io.cpp -- parameter file, output naming and the Tecplot writer (host only).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "piv_b200.h"

namespace {

// One line of a CStdioFile::ReadString loop: false at end of file, trailing CR/LF removed.
bool read_line(FILE *f, std::string &out)
{
    out.clear();
    int c;
    bool any = false;
    while ((c = fgetc(f)) != EOF) {
        any = true;
        if (c == '\n') break;
        out.push_back((char)c);
    }
    if (!any) return false;
    while (!out.empty() && (out.back() == '\r' || out.back() == '\n')) out.pop_back();
    return true;
}

void copy_str(char *dst, size_t cap, const std::string &s)
{
    size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
    std::memcpy(dst, s.data(), n);
    dst[n] = 0;
}

}  // namespace

extern "C" {

// X/main.cpp:93-158: 6 path lines then 44 numeric lines, parsed like _wtoi/_wtof.
int piv_params_read(const char *path, piv_params *out, piv_paths *paths)
{
    if (!path || !out) return PIV_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return PIV_ERR_IO;  // "Can't open parameter file!"
    std::vector<std::string> L;
    std::string s;
    while (L.size() < 50 && read_line(f, s)) L.push_back(s);
    fclose(f);
    if (L.size() < 50) return PIV_ERR_ARG;  // "Parameter missing in Parameter.dat!"
    if (paths) {
        copy_str(paths->prefix_f1, sizeof(paths->prefix_f1), L[0]);
        copy_str(paths->suffix_f1, sizeof(paths->suffix_f1), L[1]);
        copy_str(paths->prefix_f2, sizeof(paths->prefix_f2), L[2]);
        copy_str(paths->suffix_f2, sizeof(paths->suffix_f2), L[3]);
        copy_str(paths->dir_index, sizeof(paths->dir_index), L[4]);
        copy_str(paths->folder_result, sizeof(paths->folder_result), L[5]);
    }
    auto I = [&](int line) { return atoi(L[line - 1].c_str()); };
    auto F = [&](int line) { return (float)atof(L[line - 1].c_str()); };
    piv_params &p = *out;
    p.device_id = I(7);
    p.if_mhe = I(8);
    p.mhe_ws = I(9);
    p.mhe_thresh = F(10);
    p.Nx = I(11);
    p.Ny = I(12);
    p.ws_x1 = I(13);
    p.ws_y1 = I(14);
    p.spacing_x1 = I(15);
    p.spacing_y1 = I(16);
    p.Npass1 = I(17);
    p.ws_x2 = I(18);
    p.ws_y2 = I(19);
    p.spacing_x2 = I(20);
    p.spacing_y2 = I(21);
    p.Npass2 = I(22);
    p.Nsec_cc = I(23);
    p.wx1_median = I(24);
    p.wy1_median = I(25);
    p.Npass1_median = I(26);
    p.minNneigh_p1 = I(27);
    p.residual_threshold_p1 = F(28);
    p.insert_threshold_p1 = F(29);
    p.wx1_smooth = I(30);
    p.wy1_smooth = I(31);
    p.Npass1_smooth = I(32);
    p.wx2_median = I(33);
    p.wy2_median = I(34);
    p.Npass2_median = I(35);
    p.minNneigh_p2 = I(36);
    p.residual_threshold_p2 = F(37);
    p.insert_threshold_p2 = F(38);
    p.wx2_smooth = I(39);
    p.wy2_smooth = I(40);
    p.Npass2_smooth = I(41);
    p.max_dispx_win_percent1 = F(42);
    p.max_dispy_win_percent1 = F(43);
    p.max_dispx_win_percent2 = F(44);
    p.max_dispy_win_percent2 = F(45);
    p.Npeak_save = I(46);
    p.dispx_lim1 = F(47);
    p.dispx_lim2 = F(48);
    p.dispy_lim1 = F(49);
    p.dispy_lim2 = F(50);
    return PIV_OK;
}

// File names of X/main.cpp:327-369 (folder + %04d index + suffix).
int piv_output_name(const piv_params *p, const char *folder, int idx, int kind, char *out, size_t cap)
{
    if (!p || !out || cap == 0) return PIV_ERR_ARG;
    char name[512];
    switch (kind) {
    case 0:
        snprintf(name, sizeof(name), "_vector_GPU_Grid1_%d-peak-candidate_3DCC-%d-%d-%dpass_4peaks_raw.dat",
                 p->Npeak_save, p->ws_x1, p->ws_y1, p->Npass1);
        break;
    case 1:
        snprintf(name, sizeof(name),
                 "_vector_GPU_Grid1_%d-peak-candidate_3DCC-%d-%d-%dpass_median-%d-%d-%.1f-%dpass_smooth-%d-%d-%dpass.dat",
                 p->Npeak_save, p->ws_x1, p->ws_y1, p->Npass1, p->wx1_median, p->wy1_median,
                 (double)p->insert_threshold_p1, p->Npass1_median, p->wx1_smooth, p->wy1_smooth, p->Npass1_smooth);
        break;
    case 2:
        snprintf(name, sizeof(name), "_vector_GPU_Grid2_%d-peak-candidate_3DCC-%d-%d-%dpass_4peaks_raw.dat",
                 p->Npeak_save, p->ws_x2, p->ws_y2, p->Npass2);
        break;
    case 3:
        snprintf(name, sizeof(name),
                 "_vector_GPU_Grid2_%d-peak-candidate_3DCC-%d-%d-%dpass_median-%d-%d-%.1f-%dpass_smooth-%d-%d-%dpass.dat",
                 p->Npeak_save, p->ws_x2, p->ws_y2, p->Npass2, p->wx2_median, p->wy2_median,
                 (double)p->insert_threshold_p2, p->Npass2_median, p->wx2_smooth, p->wy2_smooth, p->Npass2_smooth);
        break;
    case 4:
        snprintf(name, sizeof(name), "_vector_GPU_Grid2_%d-peak-candidate_3DCC-%d-%d-%dpass_median-%d-%d-%.1f-%dpass.dat",
                 p->Npeak_save, p->ws_x2, p->ws_y2, p->Npass2, p->wx2_median, p->wy2_median,
                 (double)p->insert_threshold_p2, p->Npass2_median);
        break;
    default:
        return PIV_ERR_ARG;
    }
    int n = snprintf(out, cap, "%s%04d%s", folder ? folder : "", idx, name);
    return (n < 0 || (size_t)n >= cap) ? PIV_ERR_ARG : PIV_OK;
}

// Tecplot ASCII body of write_vec_data_general (X/xcorr2d_multi_grid.cu:1875-1886,
// :1902-1911): setprecision(2) fixed == "%.2f", tab separated, '\n' line ends.
int piv_tecplot_write_arrays(const char *path, int Nx_vec, int Ny_vec, int sp_x, int sp_y, int raw, int Npeak_save,
                             const float *dx, const float *dy)
{
    if (!path || !dx || !dy || Nx_vec < 1 || Ny_vec < 1) return PIV_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return PIV_ERR_IO;  // "Error occurs while the vector file is being written."
    std::vector<char> buf(1 << 20);
    setvbuf(f, buf.data(), _IOFBF, buf.size());
    fputs("TITLE = \"B00001\"\n", f);
    if (raw)
        fputs("VARIABLES = \"x\", \"y\", \"dx1\", \"dy1\", \"dx2\", \"dy2\", \"dx3\", \"dy3\", \"dx4\", \"dy4\"\n", f);
    else
        fputs("VARIABLES = \"x\", \"y\", \"displacement-x\", \"displacement-y\"\n", f);
    fprintf(f, "ZONE T=\"Frame 0\", I=%d, J=%d\n", Nx_vec, Ny_vec);
    const long Nt = (long)Nx_vec * Ny_vec, n = Nt * (raw ? Npeak_save : 1);
    for (long i = 0; i < Nt; ++i) {
        const long j = i / Nx_vec, k = i - j * Nx_vec;
        fprintf(f, "%.2f\t%.2f", (double)(float)(sp_x / 2 + k * sp_x), (double)(float)(sp_y / 2 + j * sp_y));
        if (raw) {
            // the reference always prints four candidate columns at i*Npeak_save + c
            for (int c = 0; c < 4; ++c) {
                const long q = i * Npeak_save + c;
                fprintf(f, "\t%.2f\t%.2f", q < n ? (double)dx[q] : 0.0, q < n ? (double)dy[q] : 0.0);
            }
        } else {
            fprintf(f, "\t%.2f\t%.2f", (double)dx[i], (double)dy[i]);
        }
        fputc('\n', f);
    }
    int bad = ferror(f);
    fclose(f);
    return bad ? PIV_ERR_IO : PIV_OK;
}

int piv_write_tecplot(piv_engine *e, const char *path, int selection)
{
    if (!e || !path || selection < 0 || selection > 3) return PIV_ERR_ARG;
    piv_geometry g;
    piv_params p;
    piv_get_geometry(e, &g);
    piv_get_params(e, &p);
    const int k = selection / 2;
    const int spx = k ? p.spacing_x2 : p.spacing_x1, spy = k ? p.spacing_y2 : p.spacing_y1, nps = p.Npeak_save;
    const bool raw = (selection % 2) == 0;
    const size_t Nt = (size_t)g.Nt_vec[k], n = raw ? Nt * nps : Nt;
    std::vector<float> dx(n), dy(n);
    int rc = piv_get_field(e, selection, nullptr, nullptr, dx.data(), dy.data(), nullptr);
    if (rc) return rc;
    return piv_tecplot_write_arrays(path, g.Nx_vec[k], g.Ny_vec[k], spx, spy, raw ? 1 : 0, nps, dx.data(), dy.data());
}

}  // extern "C"
