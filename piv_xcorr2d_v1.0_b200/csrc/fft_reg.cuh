// fft_reg.cuh -- register-resident, fully unrolled mixed-radix FFT for one thread.
//
// fft<N, INV>(x) transforms N complex values held in registers in place (natural
// order in, natural order out), unnormalised: INV=false uses exp(-2*pi*i*k*n/N)
// (cuFFT FORWARD), INV=true exp(+2*pi*i*k*n/N) (cuFFT INVERSE).  Decimation in time,
// radix 4 where possible, then 2, 3, 5, 7, 11, 13 (every multiple of 4 up to 64 is
// covered).  All twiddles are compile-time immediates (piv_common.cuh).
#pragma once

#include "piv_common.cuh"

namespace piv {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward quarter turn) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot_quarter(float2 a)
{
    if constexpr (INV) return make_float2(-a.y, a.x);
    else return make_float2(a.y, -a.x);
}

// v * exp(-/+ 2*pi*i*E/N)
template <int N, bool INV, int E>
__device__ __forceinline__ float2 twiddle(float2 v)
{
    constexpr int e = ((E % N) + N) % N;
    if constexpr (e == 0) {
        return v;
    } else if constexpr (2 * e == N) {
        return make_float2(-v.x, -v.y);
    } else if constexpr (4 * e == N) {
        return rot_quarter<INV>(v);
    } else if constexpr (4 * e == 3 * N) {
        return rot_quarter<!INV>(v);
    } else {
        constexpr CosSin cs = cossin_2pi(e, N);
        constexpr float c = (float)cs.c;
        constexpr float s = INV ? (float)cs.s : (float)(-cs.s);
        return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
    }
}

constexpr int smallest_factor(int n)
{
    for (int f = 2; f * f <= n; ++f)
        if (n % f == 0) return f;
    return n;
}

constexpr int pick_radix(int n)
{
    if (n % 4 == 0) return 4;
    return smallest_factor(n);
}

// Direct DFT of a small prime length (or 4), out of place into y.
template <int P, bool INV>
__device__ __forceinline__ void dft_small(float2 (&x)[P])
{
    if constexpr (P == 1) {
    } else if constexpr (P == 2) {
        float2 a = x[0], b = x[1];
        x[0] = cadd(a, b);
        x[1] = csub(a, b);
    } else if constexpr (P == 3) {
        // X1 = a - (b+c)/2 -/+ i*sqrt(3)/2*(b-c), X2 = conjugate rotation
        constexpr float h = 0.86602540378443864676f;  // sqrt(3)/2
        float2 a = x[0], b = x[1], c = x[2];
        float2 t1 = cadd(b, c), t2 = csub(b, c);
        float2 m = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
        float2 r = rot_quarter<INV>(make_float2(h * t2.x, h * t2.y));  // -/+ i*h*t2
        x[0] = cadd(a, t1);
        x[1] = cadd(m, r);
        x[2] = csub(m, r);
    } else if constexpr (P == 4) {
        float2 a = x[0], b = x[1], c = x[2], d = x[3];
        float2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = rot_quarter<INV>(csub(b, d));
        x[0] = cadd(t0, t2);
        x[1] = cadd(t1, t3);
        x[2] = csub(t0, t2);
        x[3] = csub(t1, t3);
    } else {
        float2 in[P];
#pragma unroll
        for (int r = 0; r < P; ++r) in[r] = x[r];
        static_for<0, P>([&](auto sc) {
            constexpr int s = decltype(sc)::value;
            float2 acc = in[0];
            static_for<1, P>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                acc = cadd(acc, twiddle<P, INV, r * s>(in[r]));
            });
            x[s] = acc;
        });
    }
}

template <int N, bool INV>
__device__ __forceinline__ void fft(float2 (&x)[N])
{
    constexpr int R = pick_radix(N);
    if constexpr (R == N) {
        dft_small<N, INV>(x);
    } else {
        constexpr int M = N / R;
        float2 sub[R][M];
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int m = 0; m < M; ++m) sub[r][m] = x[r + R * m];
#pragma unroll
        for (int r = 0; r < R; ++r) fft<M, INV>(sub[r]);
        static_for<0, M>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            float2 t[R];
            t[0] = sub[0][k];
            static_for<1, R>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                t[r] = twiddle<N, INV, r * k>(sub[r][k]);
            });
            dft_small<R, INV>(t);
#pragma unroll
            for (int s = 0; s < R; ++s) x[k + M * s] = t[s];
        });
    }
}

// Two-thread transform of length N (N % 4 == 0) by a lane pair (lanes l and l ^ 16, both
// in `mask`; the halves sit in different half-warps, so the pair's 8-byte shared-memory
// accesses do not share banks).  Decimation in time by 2: half 0 holds x[2j], half 1 holds x[2j + 1]
// (j < N/2) in y, each transforms its half (E, O), and after an exchange of N/4 values
// each finishes half of the radix-2 step  X[k] = E[k] + W^k O[k],  X[k + N/2] =
// E[k] - W^k O[k], for k = half*N/4 + j, j < N/4  (W^(N/4 + j) = W^(N/4) W^j).
// Output: y[m] = X[fft2t_index<N>(m, half)].
template <int N>
__device__ __forceinline__ int fft2t_index(int m, int half)
{
    return m < N / 4 ? half * (N / 4) + m : N / 2 + half * (N / 4) + (m - N / 4);
}

template <int N, bool INV>
__device__ __forceinline__ void fft2t(float2 (&y)[N / 2], int half, unsigned mask)
{
    static_assert(N % 4 == 0, "two-thread transform of a length divisible by 4");
    constexpr int Q = N / 4;
    fft<N / 2, INV>(y);
    // half 0 keeps E[0, Q) and needs O[0, Q); half 1 keeps O[Q, 2Q) and needs E[Q, 2Q)
    float2 e[Q], o[Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) {
        const float2 send = half ? y[j] : y[j + Q];
        float2 recv;
        recv.x = __shfl_xor_sync(mask, send.x, 16);
        recv.y = __shfl_xor_sync(mask, send.y, 16);
        e[j] = half ? recv : y[j];
        o[j] = half ? y[j + Q] : recv;
    }
    static_for<0, Q>([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        const float2 t0 = twiddle<N, INV, j>(o[j]);
        const float2 t = half ? rot_quarter<INV>(t0) : t0;
        y[j] = cadd(e[j], t);
        y[j + Q] = csub(e[j], t);
    });
}

// One-thread transform with exactly the arithmetic of fft2t: the even and odd halves by
// fft<N/2>, then X[k] = E[k] + t, X[k + N/2] = E[k] - t with t = W^j O[k] for k = j < N/4
// and t = (W^(N/4)) (W^j O[k]) for k = N/4 + j.  A CTA shape that runs a transform on one
// thread therefore produces the same bits as one that runs it on a lane pair, so the
// tile variant the autotuner picks never changes a result.
template <int N, bool INV>
__device__ __forceinline__ void fft_r2(float2 (&x)[N])
{
    static_assert(N % 4 == 0, "radix-2-first transform of a length divisible by 4");
    constexpr int H = N / 2, Q = N / 4;
    float2 e[H], o[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        e[j] = x[2 * j];
        o[j] = x[2 * j + 1];
    }
    fft<H, INV>(e);
    fft<H, INV>(o);
    static_for<0, Q>([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        const float2 t0 = twiddle<N, INV, j>(o[j]);
        x[j] = cadd(e[j], t0);
        x[j + H] = csub(e[j], t0);
        const float2 t1 = rot_quarter<INV>(twiddle<N, INV, j>(o[j + Q]));
        x[j + Q] = cadd(e[j + Q], t1);
        x[j + Q + H] = csub(e[j + Q], t1);
    });
}

// The inverse transform of the correlation kernels' P3/P4 phases: lengths of 32 and more
// (divisible by 4) always split radix-2 first, whether one thread or a lane pair runs it.
template <int N>
constexpr bool inverse_radix2_first() { return N % 4 == 0 && N >= 32; }

}  // namespace piv
