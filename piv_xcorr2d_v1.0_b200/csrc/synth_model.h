// synth_model.h -- the random streams and displacement-field models of the synthetic
// particle-image generator, shared by the host generator (synth.cpp) and the device one
// (synth_device.cu) so that both draw the same particles and fields from a seed.
//
// Random numbers: Philox4x32-10 (Salmon et al., "Parallel random numbers: as easy as
// 1, 2, 3", SC'11), counter = (item, stream), key = seed.
#pragma once
#include <cmath>
#include <cstdint>

#include "piv_b200.h"

#ifdef __CUDACC__
#define PIV_HD __host__ __device__
#else
#define PIV_HD
#endif

namespace piv {

struct U4 {
    uint32_t v[4];
};

PIV_HD inline U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed)
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
PIV_HD inline double u01(uint32_t a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); }

enum : uint32_t { kStreamParticle = 1, kStreamNoise = 2, kStreamField = 3 };

constexpr double kSynthPi = 3.14159265358979323846;

// The field model with its derived constants.
struct SynthModel {
    int field = PIV_FIELD_UNIFORM;
    int Nx = 0, Ny = 0;
    double a = 0, b = 0, c = 0;
    double vortex_k = 0;  // Lamb-Oseen scale: v(r) = k * (1 - exp(-(r/rc)^2)) / (r/rc)
    double fk[8][6] = {}; // Fourier modes: kx, ky, phase_u, phase_v, amp_u, amp_v
};

inline SynthModel synth_model(const piv_synth_params *s)
{
    SynthModel m;
    m.field = s->field;
    m.Nx = s->Nx;
    m.Ny = s->Ny;
    m.a = s->a;
    m.b = s->b;
    m.c = s->c;
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
        m.vortex_k = s->a / fmax;
    } else if (s->field == PIV_FIELD_FOURIER) {
        double norm_u = 0, norm_v = 0;
        for (int q = 0; q < 8; ++q) {
            U4 r = philox((uint32_t)q, kStreamField, 0, 0, s->seed);
            U4 t = philox((uint32_t)q, kStreamField, 1, 0, s->seed);
            double lam = s->a + (s->b - s->a) * u01(r.v[0]);
            double th = 2 * kSynthPi * u01(r.v[1]);
            m.fk[q][0] = 2 * kSynthPi * std::cos(th) / lam;
            m.fk[q][1] = 2 * kSynthPi * std::sin(th) / lam;
            m.fk[q][2] = 2 * kSynthPi * u01(r.v[2]);
            m.fk[q][3] = 2 * kSynthPi * u01(r.v[3]);
            m.fk[q][4] = 0.5 + u01(t.v[0]);
            m.fk[q][5] = 0.5 + u01(t.v[1]);
            norm_u += m.fk[q][4];
            norm_v += m.fk[q][5];
        }
        for (int q = 0; q < 8; ++q) {
            m.fk[q][4] *= s->c / norm_u;
            m.fk[q][5] *= s->c / norm_v;
        }
    }
    return m;
}

PIV_HD inline void synth_eval(const SynthModel &m, double x, double y, double &u, double &v)
{
    switch (m.field) {
    case PIV_FIELD_UNIFORM:
        u = m.a;
        v = m.b;
        return;
    case PIV_FIELD_VORTEX: {
        double xc = 0.5 * m.Nx, yc = 0.5 * m.Ny;
        double dx = x - xc, dy = y - yc, r = sqrt(dx * dx + dy * dy);
        if (r > 1e-12) {
            double q = r / m.b;
            double vt = m.vortex_k * (1 - exp(-q * q)) / q;
            u = -vt * dy / r;
            v = vt * dx / r;
        } else {
            u = v = 0;
        }
        u += m.c * (y - yc);
        return;
    }
    case PIV_FIELD_FOURIER: {
        u = v = 0;
        for (int q = 0; q < 8; ++q) {
            double ph = m.fk[q][0] * x + m.fk[q][1] * y;
            u += m.fk[q][4] * cos(ph + m.fk[q][2]);
            v += m.fk[q][5] * cos(ph + m.fk[q][3]);
        }
        return;
    }
    default:
        u = v = 0;
    }
}

}  // namespace piv
