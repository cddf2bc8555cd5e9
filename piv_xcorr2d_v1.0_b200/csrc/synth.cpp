// synth.cpp -- seeded synthetic PIV image pairs (no counterpart in the reference; it
// stands in for the missing sample TIFFs and for the public benchmark data the
// reference never shipped).
//
// Particles: uniform positions over the image plus a 32 px margin at density ppp,
// peak intensity U(i_min, i_max), pixel-integrated Gaussian spots
//   I(px) = I0 * gx(px) * gy(py),
//   gx(px) = [erf((px+0.5-xp)/(sqrt2 s)) - erf((px-0.5-xp)/(sqrt2 s))] / (2 erf(0.5/(sqrt2 s))),
// so a particle centred on a pixel gives I0 there.  Frame 2 moves every particle by
// the field evaluated at its frame-1 position (x2 = x1 + u(x1)).  Background and
// Gaussian noise are added per pixel, then clipped to [0, 255] and rounded.
// Random numbers: Philox4x32-10 (Salmon et al., SC'11), counter = (item, stream),
// key = seed, so every value is reproducible and independent of evaluation order.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "piv_b200.h"

namespace {

struct U4 {
    uint32_t v[4];
};

U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * x0, p1 = (uint64_t)M1 * x2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ x1 ^ k0, n1 = lo1, n2 = hi0 ^ x3 ^ k1, n3 = lo0;
        x0 = n0;
        x1 = n1;
        x2 = n2;
        x3 = n3;
        k0 += W0;
        k1 += W1;
    }
    return U4{{x0, x1, x2, x3}};
}

// (0, 1): never 0, so log() in Box-Muller is finite
double u01(uint32_t a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); }

enum : uint32_t { kStreamParticle = 1, kStreamNoise = 2, kStreamField = 3 };

struct Field {
    const piv_synth_params *s;
    double vortex_k = 0;  // Lamb-Oseen scale: v(r) = k * (1 - exp(-(r/rc)^2)) / (r/rc)
    double fk[8][6];      // Fourier modes: kx, ky, phase_u, phase_v, amp_u, amp_v

    explicit Field(const piv_synth_params *sp) : s(sp)
    {
        if (s->field == PIV_FIELD_VORTEX) {
            // peak of (1 - exp(-x^2))/x by golden-section search on [0.5, 2]
            double a = 0.5, b = 2.0;
            const double gr = 0.6180339887498949;
            for (int i = 0; i < 200; ++i) {
                double c = b - gr * (b - a), d = a + gr * (b - a);
                double fc = (1 - std::exp(-c * c)) / c, fd = (1 - std::exp(-d * d)) / d;
                if (fc > fd) b = d; else a = c;
            }
            double xm = 0.5 * (a + b), fmax = (1 - std::exp(-xm * xm)) / xm;
            vortex_k = s->a / fmax;
        } else if (s->field == PIV_FIELD_FOURIER) {
            double norm_u = 0, norm_v = 0;
            for (int m = 0; m < 8; ++m) {
                U4 r = philox((uint32_t)m, kStreamField, 0, 0, s->seed);
                U4 q = philox((uint32_t)m, kStreamField, 1, 0, s->seed);
                double lam = s->a + (s->b - s->a) * u01(r.v[0]);
                double th = 2 * M_PI * u01(r.v[1]);
                fk[m][0] = 2 * M_PI * std::cos(th) / lam;
                fk[m][1] = 2 * M_PI * std::sin(th) / lam;
                fk[m][2] = 2 * M_PI * u01(r.v[2]);
                fk[m][3] = 2 * M_PI * u01(r.v[3]);
                fk[m][4] = 0.5 + u01(q.v[0]);
                fk[m][5] = 0.5 + u01(q.v[1]);
                norm_u += fk[m][4];
                norm_v += fk[m][5];
            }
            for (int m = 0; m < 8; ++m) {
                fk[m][4] *= s->c / norm_u;
                fk[m][5] *= s->c / norm_v;
            }
        }
    }

    void eval(double x, double y, double &u, double &v) const
    {
        switch (s->field) {
        case PIV_FIELD_UNIFORM:
            u = s->a;
            v = s->b;
            return;
        case PIV_FIELD_VORTEX: {
            double xc = 0.5 * s->Nx, yc = 0.5 * s->Ny;
            double dx = x - xc, dy = y - yc, r = std::sqrt(dx * dx + dy * dy);
            double vt = 0;
            if (r > 1e-12) {
                double q = r / s->b;
                vt = vortex_k * (1 - std::exp(-q * q)) / q;
                u = -vt * dy / r;
                v = vt * dx / r;
            } else {
                u = v = 0;
            }
            u += s->c * (y - yc);
            return;
        }
        case PIV_FIELD_FOURIER: {
            u = v = 0;
            for (int m = 0; m < 8; ++m) {
                double ph = fk[m][0] * x + fk[m][1] * y;
                u += fk[m][4] * std::cos(ph + fk[m][2]);
                v += fk[m][5] * std::cos(ph + fk[m][3]);
            }
            return;
        }
        default:
            u = v = 0;
        }
    }
};

void render(std::vector<float> &acc, int Nx, int Ny, double xp, double yp, double I0, double sigma, double norm)
{
    const double rad = 3.0 * sigma + 1.0, k = 1.0 / (std::sqrt(2.0) * sigma);
    int x0 = (int)std::floor(xp - rad), x1 = (int)std::ceil(xp + rad);
    int y0 = (int)std::floor(yp - rad), y1 = (int)std::ceil(yp + rad);
    if (x1 < 0 || y1 < 0 || x0 >= Nx || y0 >= Ny) return;
    if (x0 < 0) x0 = 0;
    if (y0 < 0) y0 = 0;
    if (x1 > Nx - 1) x1 = Nx - 1;
    if (y1 > Ny - 1) y1 = Ny - 1;
    double gx[16], gy[16];
    const int nx = x1 - x0 + 1, ny = y1 - y0 + 1;
    if (nx > 16 || ny > 16) return;
    for (int i = 0; i < nx; ++i) {
        double px = x0 + i;
        gx[i] = (std::erf((px + 0.5 - xp) * k) - std::erf((px - 0.5 - xp) * k)) * norm;
    }
    for (int j = 0; j < ny; ++j) {
        double py = y0 + j;
        gy[j] = (std::erf((py + 0.5 - yp) * k) - std::erf((py - 0.5 - yp) * k)) * norm;
    }
    for (int j = 0; j < ny; ++j) {
        float *row = acc.data() + (size_t)(y0 + j) * Nx + x0;
        const double a = I0 * gy[j];
        for (int i = 0; i < nx; ++i) row[i] += (float)(a * gx[i]);
    }
}

void finish(const std::vector<float> &acc, const piv_synth_params *s, uint32_t frame, uint8_t *out)
{
    const size_t n = (size_t)s->Nx * s->Ny;
    for (size_t i = 0; i < n; i += 2) {
        // Box-Muller: two normals per Philox draw
        U4 r = philox((uint32_t)i, (uint32_t)(i >> 32), kStreamNoise, frame, s->seed);
        double rr = std::sqrt(-2.0 * std::log(u01(r.v[0]))), th = 2 * M_PI * u01(r.v[1]);
        double z[2] = {rr * std::cos(th), rr * std::sin(th)};
        for (int q = 0; q < 2 && i + q < n; ++q) {
            double v = s->background + acc[i + q] + s->noise_sigma * z[q];
            v = v < 0 ? 0 : (v > 255 ? 255 : v);
            out[i + q] = (uint8_t)std::floor(v + 0.5);
        }
    }
}

}  // namespace

extern "C" {

int piv_synth_field(const piv_synth_params *s, const float *x, const float *y, int n, float *u, float *v)
{
    if (!s || !x || !y || !u || !v || n < 0) return PIV_ERR_ARG;
    Field f(s);
    for (int i = 0; i < n; ++i) {
        double uu, vv;
        f.eval(x[i], y[i], uu, vv);
        u[i] = (float)uu;
        v[i] = (float)vv;
    }
    return PIV_OK;
}

int piv_synth_pair(const piv_synth_params *s, uint8_t *f1, uint8_t *f2)
{
    if (!s || !f1 || !f2 || s->Nx < 1 || s->Ny < 1 || s->ppp < 0 || s->sigma <= 0) return PIV_ERR_ARG;
    const int m = 32;
    const double W = s->Nx + 2.0 * m, H = s->Ny + 2.0 * m;
    const long np = std::lround(s->ppp * W * H);
    Field fld(s);
    const double norm = 1.0 / (2.0 * std::erf(0.5 / (std::sqrt(2.0) * s->sigma)));
    std::vector<float> a1((size_t)s->Nx * s->Ny, 0.f), a2((size_t)s->Nx * s->Ny, 0.f);
    for (long p = 0; p < np; ++p) {
        U4 r = philox((uint32_t)p, (uint32_t)(p >> 32), kStreamParticle, 0, s->seed);
        const double xp = u01(r.v[0]) * W - m, yp = u01(r.v[1]) * H - m;
        const double I0 = s->i_min + (s->i_max - s->i_min) * u01(r.v[2]);
        double u, v;
        fld.eval(xp, yp, u, v);
        render(a1, s->Nx, s->Ny, xp, yp, I0, s->sigma, norm);
        render(a2, s->Nx, s->Ny, xp + u, yp + v, I0, s->sigma, norm);
    }
    finish(a1, s, 0, f1);
    finish(a2, s, 1, f2);
    return PIV_OK;
}

}  // extern "C"
