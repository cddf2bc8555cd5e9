// io.cpp -- parameter file, output naming and the Tecplot writer (host only).
#include <cmath>
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

namespace {

// "%.2f" of a float without printf: f*100 is exact in double (24 + 7 significant
// bits), rint() rounds it half-to-even in the default rounding mode exactly as printf
// rounds the exact decimal value, and the sign of negative values that round to zero is
// kept ("-0.00").  Non-finite values fall back to snprintf.
char *fmt2(char *p, float f)
{
    if (!std::isfinite(f)) return p + std::sprintf(p, "%.2f", (double)f);
    double t = std::rint((double)f * 100.0);
    if (std::signbit(f)) *p++ = '-';
    unsigned long long v = (unsigned long long)std::fabs(t);
    char tmp[32];
    int n = 0;
    unsigned long long ip = v / 100;
    unsigned fr = (unsigned)(v % 100);
    do {
        tmp[n++] = (char)('0' + ip % 10);
        ip /= 10;
    } while (ip);
    while (n) *p++ = tmp[--n];
    *p++ = '.';
    *p++ = (char)('0' + fr / 10);
    *p++ = (char)('0' + fr % 10);
    return p;
}

}  // namespace

// Tecplot ASCII body of write_vec_data_general (X/xcorr2d_multi_grid.cu:1875-1886,
// :1902-1911): setprecision(2) fixed == "%.2f", tab separated, '\n' line ends.
int piv_tecplot_write_arrays(const char *path, int Nx_vec, int Ny_vec, int sp_x, int sp_y, int raw, int Npeak_save,
                             const float *dx, const float *dy)
{
    if (!path || !dx || !dy || Nx_vec < 1 || Ny_vec < 1 || Npeak_save < 1) return PIV_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return PIV_ERR_IO;  // "Error occurs while the vector file is being written."
    std::string out;
    const long Nt = (long)Nx_vec * Ny_vec, n = Nt * (raw ? Npeak_save : 1);
    out.reserve((size_t)Nt * (raw ? 80 : 36) + 256);
    out += "TITLE = \"B00001\"\n";
    if (raw)
        out += "VARIABLES = \"x\", \"y\", \"dx1\", \"dy1\", \"dx2\", \"dy2\", \"dx3\", \"dy3\", \"dx4\", \"dy4\"\n";
    else
        out += "VARIABLES = \"x\", \"y\", \"displacement-x\", \"displacement-y\"\n";
    char line[512];
    std::snprintf(line, sizeof(line), "ZONE T=\"Frame 0\", I=%d, J=%d\n", Nx_vec, Ny_vec);
    out += line;
    for (long i = 0; i < Nt; ++i) {
        const long j = i / Nx_vec, k = i - j * Nx_vec;
        char *p = line;
        p = fmt2(p, (float)(sp_x / 2 + k * sp_x));
        *p++ = '\t';
        p = fmt2(p, (float)(sp_y / 2 + j * sp_y));
        if (raw) {
            // the reference always prints four candidate columns at i*Npeak_save + c
            for (int c = 0; c < 4; ++c) {
                const long q = i * Npeak_save + c;
                *p++ = '\t';
                p = fmt2(p, q < n ? dx[q] : 0.f);
                *p++ = '\t';
                p = fmt2(p, q < n ? dy[q] : 0.f);
            }
        } else {
            *p++ = '\t';
            p = fmt2(p, dx[i]);
            *p++ = '\t';
            p = fmt2(p, dy[i]);
        }
        *p++ = '\n';
        out.append(line, (size_t)(p - line));
    }
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    const bool closed = std::fclose(f) == 0;
    return (ok && closed) ? PIV_OK : PIV_ERR_IO;
}

// ---- binary sidecar: NPY v1.0, little-endian float32, C order ----
int piv_npy_write_f32(const char *path, const float *data, int ndim, const int *shape)
{
    if (!path || !data || !shape || ndim < 1 || ndim > 8) return PIV_ERR_ARG;
    size_t n = 1;
    std::string sh = "(";
    for (int d = 0; d < ndim; ++d) {
        if (shape[d] < 0) return PIV_ERR_ARG;
        n *= (size_t)shape[d];
        sh += std::to_string(shape[d]) + (ndim == 1 ? "," : (d + 1 < ndim ? ", " : ""));
    }
    sh += ")";
    std::string hdr = "{'descr': '<f4', 'fortran_order': False, 'shape': " + sh + ", }";
    const size_t pre = 10;  // magic(6) + version(2) + header length(2)
    size_t total = pre + hdr.size() + 1;
    hdr.append((64 - total % 64) % 64, ' ');
    hdr.push_back('\n');
    FILE *f = fopen(path, "wb");
    if (!f) return PIV_ERR_IO;
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    const uint16_t hl = (uint16_t)hdr.size();
    const unsigned char hlb[2] = {(unsigned char)(hl & 0xff), (unsigned char)(hl >> 8)};
    bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(hlb, 1, 2, f) == 2 &&
              fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size() && fwrite(data, sizeof(float), n, f) == n;
    return (fclose(f) == 0 && ok) ? PIV_OK : PIV_ERR_IO;
}

// ---- minimal baseline TIFF (uncompressed, 8-bit grey, strips; both byte orders) ----

namespace {

struct TiffReader {
    std::vector<uint8_t> d;
    bool le = true;
    uint32_t u16(size_t o) const
    {
        return le ? (uint32_t)d[o] | ((uint32_t)d[o + 1] << 8) : ((uint32_t)d[o] << 8) | d[o + 1];
    }
    uint32_t u32(size_t o) const
    {
        return le ? (uint32_t)d[o] | ((uint32_t)d[o + 1] << 8) | ((uint32_t)d[o + 2] << 16) | ((uint32_t)d[o + 3] << 24)
                  : ((uint32_t)d[o] << 24) | ((uint32_t)d[o + 1] << 16) | ((uint32_t)d[o + 2] << 8) | d[o + 3];
    }
    bool ok(size_t o, size_t n) const { return o + n <= d.size(); }
};

struct TiffInfo {
    uint32_t width = 0, height = 0, bits = 8, spp = 1, compression = 1, rows_per_strip = 0;
    std::vector<uint32_t> offsets, counts;
};

int tiff_parse(const char *path, TiffReader &r, TiffInfo &t)
{
    FILE *f = fopen(path, "rb");
    if (!f) return PIV_ERR_IO;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (sz < 8) {
        fclose(f);
        return PIV_ERR_IO;
    }
    r.d.resize((size_t)sz);
    size_t got = fread(r.d.data(), 1, (size_t)sz, f);
    fclose(f);
    if (got != (size_t)sz) return PIV_ERR_IO;
    if (r.d[0] == 'I' && r.d[1] == 'I') r.le = true;
    else if (r.d[0] == 'M' && r.d[1] == 'M') r.le = false;
    else return PIV_ERR_IO;
    if (r.u16(2) != 42) return PIV_ERR_IO;
    size_t ifd = r.u32(4);
    if (!r.ok(ifd, 2)) return PIV_ERR_IO;
    const uint32_t ne = r.u16(ifd);
    for (uint32_t i = 0; i < ne; ++i) {
        const size_t e = ifd + 2 + 12 * i;
        if (!r.ok(e, 12)) return PIV_ERR_IO;
        const uint32_t tag = r.u16(e), type = r.u16(e + 2), cnt = r.u32(e + 4);
        const uint32_t esz = type == 3 ? 2 : (type == 4 ? 4 : (type == 1 ? 1 : 0));
        if (esz == 0) continue;
        const size_t base = (size_t)cnt * esz <= 4 ? e + 8 : r.u32(e + 8);
        if (!r.ok(base, (size_t)cnt * esz)) return PIV_ERR_IO;
        auto val = [&](uint32_t k) -> uint32_t {
            return esz == 2 ? r.u16(base + 2 * k) : (esz == 4 ? r.u32(base + 4 * k) : r.d[base + k]);
        };
        switch (tag) {
        case 256: t.width = val(0); break;
        case 257: t.height = val(0); break;
        case 258: t.bits = val(0); break;
        case 259: t.compression = val(0); break;
        case 277: t.spp = val(0); break;
        case 278: t.rows_per_strip = val(0); break;
        case 273:
            t.offsets.resize(cnt);
            for (uint32_t k = 0; k < cnt; ++k) t.offsets[k] = val(k);
            break;
        case 279:
            t.counts.resize(cnt);
            for (uint32_t k = 0; k < cnt; ++k) t.counts[k] = val(k);
            break;
        default: break;
        }
    }
    return PIV_OK;
}

void put16(std::vector<uint8_t> &b, uint32_t v)
{
    b.push_back((uint8_t)v);
    b.push_back((uint8_t)(v >> 8));
}

void put32(std::vector<uint8_t> &b, uint32_t v)
{
    put16(b, v & 0xffff);
    put16(b, v >> 16);
}

}  // namespace

int piv_tiff_info(const char *path, int *Nx, int *Ny, int *bits)
{
    if (!path) return PIV_ERR_ARG;
    TiffReader r;
    TiffInfo t;
    int rc = tiff_parse(path, r, t);
    if (rc) return rc;
    if (Nx) *Nx = (int)t.width;
    if (Ny) *Ny = (int)t.height;
    if (bits) *bits = (int)t.bits;
    return PIV_OK;
}

// CImageIO::getImHeadTiff + ImReadTiff8 (X/ImageIOPkg.cpp:124, :280): an 8-bit grey,
// uncompressed, strip-organised TIFF of exactly Nx x Ny pixels into out (row-major).
int piv_tiff_read8(const char *path, uint8_t *out, int Nx, int Ny)
{
    if (!path || !out || Nx < 1 || Ny < 1) return PIV_ERR_ARG;
    TiffReader r;
    TiffInfo t;
    int rc = tiff_parse(path, r, t);
    if (rc) return rc;
    if (t.width != (uint32_t)Nx || t.height != (uint32_t)Ny) return PIV_ERR_ARG;
    if (t.bits != 8 || t.spp != 1 || t.compression != 1) return PIV_ERR_UNSUPPORTED;
    if (t.offsets.empty()) return PIV_ERR_IO;
    if (t.counts.size() != t.offsets.size()) {
        // StripByteCounts missing: strips of rows_per_strip rows
        const uint32_t rps = t.rows_per_strip ? t.rows_per_strip : (uint32_t)Ny;
        t.counts.assign(t.offsets.size(), rps * (uint32_t)Nx);
    }
    const size_t need = (size_t)Nx * Ny;
    size_t pos = 0;
    for (size_t s = 0; s < t.offsets.size() && pos < need; ++s) {
        size_t n = t.counts[s];
        if (n > need - pos) n = need - pos;
        if (!r.ok(t.offsets[s], n)) return PIV_ERR_IO;
        std::memcpy(out + pos, r.d.data() + t.offsets[s], n);
        pos += n;
    }
    return pos == need ? PIV_OK : PIV_ERR_IO;
}

// ImWriteTiff8 (X/ImageIOPkg.cpp:641): little-endian, one strip, 8-bit grey.
int piv_tiff_write8(const char *path, const uint8_t *img, int Nx, int Ny)
{
    if (!path || !img || Nx < 1 || Ny < 1) return PIV_ERR_ARG;
    std::vector<uint8_t> b;
    const uint32_t n = (uint32_t)Nx * (uint32_t)Ny, ntag = 9, ifd = 8, data = ifd + 2 + ntag * 12 + 4;
    b.push_back('I');
    b.push_back('I');
    put16(b, 42);
    put32(b, ifd);
    put16(b, ntag);
    auto tag = [&](uint32_t id, uint32_t type, uint32_t v) {
        put16(b, id);
        put16(b, type);
        put32(b, 1);
        if (type == 3) {
            put16(b, v);
            put16(b, 0);
        } else {
            put32(b, v);
        }
    };
    tag(256, 4, (uint32_t)Nx);
    tag(257, 4, (uint32_t)Ny);
    tag(258, 3, 8);
    tag(259, 3, 1);
    tag(262, 3, 1);
    tag(273, 4, data);
    tag(277, 3, 1);
    tag(278, 4, (uint32_t)Ny);
    tag(279, 4, n);
    put32(b, 0);
    b.insert(b.end(), img, img + n);
    FILE *f = fopen(path, "wb");
    if (!f) return PIV_ERR_IO;
    const bool ok = fwrite(b.data(), 1, b.size(), f) == b.size();
    return (fclose(f) == 0 && ok) ? PIV_OK : PIV_ERR_IO;
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
