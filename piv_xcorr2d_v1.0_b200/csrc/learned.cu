// learned.cu -- the learned grid-1 predictor: features (cost volume), U-Net forward and
// backward, loss and Adam, all as hand-written kernels; the net object and its C-ABI.
// No counterpart in the reference: the plain method's grid-1 passes
// (X/xcorr2d_multi_grid.cu:1287-1447 driven by X/main.cpp:290-300) are what it replaces.
//
// Tensors are [N][C][H][W] FP32.  Weights live as FP32 master copies (Adam state beside
// them) and as the BF16 copies every convolution reads; biases are FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "learned.cuh"
#include "tc_common.cuh"
#include "piv_b200.h"
#include "synth_model.h"

namespace piv {
namespace learned {

constexpr float kSlope = 0.1f;  // LeakyReLU negative slope
constexpr int kLayers = 13;
constexpr int kTensors = kLayers + 1;

// Layer i reads tensor `a` (optionally nearest-upsampled x2) concatenated with tensor
// `b` and writes tensor i + 1.  Tensor 0 is the cost volume.
struct LayerSpec {
    int a, ca, b, cb, up, cout, stride, act;
};
constexpr LayerSpec kSpec[kLayers] = {
    {0, 81, -1, 0, 0, 32, 1, 1},    // t1  level 0
    {1, 32, -1, 0, 0, 32, 1, 1},    // t2  level 0 (skip)
    {2, 32, -1, 0, 0, 64, 2, 1},    // t3  level 1
    {3, 64, -1, 0, 0, 64, 1, 1},    // t4  level 1 (skip)
    {4, 64, -1, 0, 0, 96, 2, 1},    // t5  level 2
    {5, 96, -1, 0, 0, 96, 1, 1},    // t6  level 2 (skip)
    {6, 96, -1, 0, 0, 128, 2, 1},   // t7  level 3
    {7, 128, -1, 0, 0, 128, 1, 1},  // t8  level 3
    {8, 128, 6, 96, 1, 96, 1, 1},   // t9  level 2: up(t8) ++ t6
    {9, 96, -1, 0, 0, 96, 1, 1},    // t10 level 2
    {10, 96, 4, 64, 1, 64, 1, 1},   // t11 level 1: up(t10) ++ t4
    {11, 64, 2, 32, 1, 32, 1, 1},   // t12 level 0: up(t11) ++ t2
    {12, 32, -1, 0, 0, 2, 1, 0},    // t13 level 0: head (downsampled px)
};
constexpr int kLevel[kTensors] = {0, 0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 0, 0};
constexpr int kChan[kTensors] = {81, 32, 32, 64, 64, 96, 96, 128, 128, 96, 96, 64, 32, 2};

// ------------------------------------------------------------------------------
// Features: 4x4 box average and the normalised cost volume.
// ------------------------------------------------------------------------------

__device__ __forceinline__ float block_sum128(float v, float *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    float s = 0.f;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    return s;
}

// down[f][y][x] = mean of the 4x4 image block / 255; sums[f] += its total.  A fixed
// grid strides over the outputs so that the frame sums take one atomic add per block.
__global__ void __launch_bounds__(128) down4_kernel(const uint8_t *f1, const uint8_t *f2, int pitch, int W4, int H4,
                                                    float *down, double *sums)
{
    __shared__ float red[4];
    const int f = blockIdx.y;
    const uint8_t *src = f ? f2 : f1;
    const bool al4 = ((reinterpret_cast<uintptr_t>(src) | (uintptr_t)pitch) & 3) == 0;
    float part = 0.f;
    for (int q = blockIdx.x * 128 + threadIdx.x; q < W4 * H4; q += gridDim.x * 128) {
        const int y = q / W4, x = q - y * W4;
        const uint8_t *p = src + (size_t)(4 * y) * pitch + 4 * x;
        int s = 0;
        if (al4) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const uint32_t w = __ldg(reinterpret_cast<const uint32_t *>(p + (size_t)r * pitch));
                s += (int)(w & 0xff) + (int)((w >> 8) & 0xff) + (int)((w >> 16) & 0xff) + (int)(w >> 24);
            }
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) s += p[(size_t)r * pitch + c];
        }
        const float v = (float)s * (1.0f / (16.0f * 255.0f));
        down[(size_t)f * W4 * H4 + q] = v;
        part += v;
    }
    const float t = block_sum128(part, red);
    if (threadIdx.x == 0) atomicAdd(sums + f, (double)t);
}

// Cost volume.  A CTA takes kCvVec consecutive vectors of kCvRows rows of the grid;
// frame 1's windows and frame 2's region (the windows grown by R) are staged once in
// shared memory, mean-free and zero outside the image (neighbouring windows overlap, so
// the CTA's rows share most of it).  Thread (row, v, dy) computes the 9 shifts
// (dy, 0..8) of its vector, sliding along each window row with the 9 frame-2 values in
// registers; the dy = R thread also sums both windows' energies.
constexpr int kCvVec = 16, kCvRows = 2;

__host__ __device__ __forceinline__ int cv_centre(int i, int sp, int left, int ws) { return (i * sp - left + ws / 2 + kDown / 2) >> 2; }

template <int WD>
__global__ void __launch_bounds__(kCvVec *kShifts *kCvRows) cv_kernel(const float *down, const double *sums, int W4,
                                                                      int H4, GridGeom g, int LW, int LHt, float *out)
{
    extern __shared__ float sh[];
    __shared__ float energy[kCvRows][kCvVec][2];
    const int Wd = WD ? WD : g.ws_x / kDown, Hd = g.ws_y / kDown;
    const int ix0 = blockIdx.x * kCvVec, iy0 = blockIdx.y * kCvRows;
    const int nv = min(kCvVec, g.Nx_vec - ix0), nr = min(kCvRows, g.Ny_vec - iy0);
    const int c0 = cv_centre(ix0, g.sp_x, g.Nx_left, g.ws_x), r0 = cv_centre(iy0, g.sp_y, g.Ny_left, g.ws_y);
    const int xl = c0 - Wd / 2 - kRadius, yl = r0 - Hd / 2 - kRadius;
    const int L1W = LW - 2 * kRadius, L1H = LHt - 2 * kRadius;
    float *s2 = sh, *s1 = sh + LHt * LW;
    const float m1 = (float)(sums[0] / ((double)W4 * H4)), m2 = (float)(sums[1] / ((double)W4 * H4));
    const float *d1 = down, *d2 = down + (size_t)W4 * H4;
    for (int e = threadIdx.x; e < LHt * LW; e += blockDim.x) {
        const int r = e / LW, c = e - r * LW;
        const int y = yl + r, x = xl + c;
        s2[e] = (x >= 0 && x < W4 && y >= 0 && y < H4) ? __ldg(d2 + (size_t)y * W4 + x) - m2 : 0.f;
    }
    for (int e = threadIdx.x; e < L1H * L1W; e += blockDim.x) {
        const int r = e / L1W, c = e - r * L1W;
        const int y = yl + kRadius + r, x = xl + kRadius + c;
        s1[e] = (x >= 0 && x < W4 && y >= 0 && y < H4) ? __ldg(d1 + (size_t)y * W4 + x) - m1 : 0.f;
    }
    __syncthreads();
    const int row = threadIdx.x / (kCvVec * kShifts);
    const int rem = threadIdx.x - row * (kCvVec * kShifts);
    const int v = rem / kShifts, dy = rem - v * kShifts;
    const bool live = v < nv && row < nr;
    float acc[kShifts];
#pragma unroll
    for (int k = 0; k < kShifts; ++k) acc[k] = 0.f;
    float e1 = 0.f, e2 = 0.f;
    if (live) {
        const int offx = cv_centre(ix0 + v, g.sp_x, g.Nx_left, g.ws_x) - c0;
        const int offy = cv_centre(iy0 + row, g.sp_y, g.Ny_left, g.ws_y) - r0;
        for (int r = 0; r < Hd; ++r) {
            const float *a = s1 + (offy + r) * L1W + offx, *b = s2 + (offy + r + dy) * LW + offx;
            float win[kShifts];
#pragma unroll
            for (int q = 0; q < kShifts - 1; ++q) win[q] = b[q];
#pragma unroll(WD ? WD : 1)
            for (int c = 0; c < Wd; ++c) {
                win[kShifts - 1] = b[c + kShifts - 1];
                const float av = a[c];
#pragma unroll
                for (int k = 0; k < kShifts; ++k) acc[k] = fmaf(av, win[k], acc[k]);
                e1 = fmaf(av, av, e1);
                e2 = fmaf(win[kRadius], win[kRadius], e2);
#pragma unroll
                for (int q = 0; q < kShifts - 1; ++q) win[q] = win[q + 1];
            }
        }
        if (dy == kRadius) {
            energy[row][v][0] = e1;
            energy[row][v][1] = e2;
        }
    }
    __syncthreads();
    if (!live) return;
    const float den = energy[row][v][0] * energy[row][v][1];
    const float sc = den > 0.f ? rsqrtf(den) : 0.f;
    const size_t plane = (size_t)g.Ny_vec * g.Nx_vec, o = (size_t)(iy0 + row) * g.Nx_vec + ix0 + v;
#pragma unroll
    for (int k = 0; k < kShifts; ++k) out[(size_t)(dy * kShifts + k) * plane + o] = acc[k] * sc;
}

size_t feature_scratch_floats(int Nx, int Ny) { return (size_t)2 * (Nx / kDown) * (Ny / kDown); }

cudaError_t launch_features(const FeatArgs &a, cudaStream_t s)
{
    const int W4 = a.Nx / kDown, H4 = a.Ny / kDown;
    if (W4 < 1 || H4 < 1 || a.g.ws_x < 2 * kDown || a.g.ws_y < 2 * kDown) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(a.sums, 0, 2 * sizeof(double), s);
    if (e != cudaSuccess) return e;
    const int blocks = std::min((W4 * H4 + 127) / 128, 4 * 148);
    down4_kernel<<<dim3(blocks, 2), 128, 0, s>>>(a.f1, a.f2, a.pitch, W4, H4, a.down, a.sums);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int Wd = a.g.ws_x / kDown, Hd = a.g.ws_y / kDown;
    // widest frame-2 region of a CTA: the spread of its vector centres plus a window and 2R
    int spread = 0;
    for (int ix0 = 0; ix0 < a.g.Nx_vec; ix0 += kCvVec) {
        const int last = std::min(ix0 + kCvVec, a.g.Nx_vec) - 1;
        spread = std::max(spread, cv_centre(last, a.g.sp_x, a.g.Nx_left, a.g.ws_x) -
                                      cv_centre(ix0, a.g.sp_x, a.g.Nx_left, a.g.ws_x));
    }
    int spread_y = 0;
    for (int iy0 = 0; iy0 < a.g.Ny_vec; iy0 += kCvRows) {
        const int last = std::min(iy0 + kCvRows, a.g.Ny_vec) - 1;
        spread_y = std::max(spread_y, cv_centre(last, a.g.sp_y, a.g.Ny_left, a.g.ws_y) -
                                          cv_centre(iy0, a.g.sp_y, a.g.Ny_left, a.g.ws_y));
    }
    // the region's row stride made odd: the threads of a warp read 9 shift rows of 4 vectors,
    // which an even stride (144 floats at 64 px windows) put on 4 banks
    const int LW = (spread + Wd + 2 * kRadius) | 1, LHt = spread_y + Hd + 2 * kRadius;
    const size_t smem = sizeof(float) * ((size_t)LHt * LW + (size_t)(LHt - 2 * kRadius) * (LW - 2 * kRadius));
    if (smem > 48 * 1024) return cudaErrorInvalidValue;
    const dim3 grid((a.g.Nx_vec + kCvVec - 1) / kCvVec, (a.g.Ny_vec + kCvRows - 1) / kCvRows);
    const int nt = kCvVec * kShifts * kCvRows;
    if (Wd == 16) cv_kernel<16><<<grid, nt, smem, s>>>(a.down, a.sums, W4, H4, a.g, LW, LHt, a.out);
    else cv_kernel<0><<<grid, nt, smem, s>>>(a.down, a.sums, W4, H4, a.g, LW, LHt, a.out);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------
// Convolutions (3x3, padding 1, stride 1 or 2).  The input is tensor a (optionally read
// through a nearest x2 upsampling) concatenated with tensor b along channels.
// ------------------------------------------------------------------------------

struct ConvIn {
    const float *a, *b;
    int ca, cb, up;
    int Hin, Win;  // resolution of the (upsampled) input
    int Ha, Wa;    // resolution of a as stored
};

struct ConvFwd {
    ConvIn in;
    int N, Ho, Wo, stride;
    const __nv_bfloat16 *w;  // [ci][tap][co] (the forward's layout; 16-byte aligned)
    const float *bias;
    int cout;
    float *out;
    int act;
    int splits;   // input-channel splits across CTAs (blockIdx.z = n * splits + split)
    float *part;  // splits > 1: partial sums [N * splits][cout][Ho * Wo], finished by conv_finish_kernel
};

// tap offsets of output pixel (oy, ox): into a (upsampled or not) and into b
__device__ __forceinline__ void conv_taps(const ConvIn &c, int oy, int ox, int stride, bool live, int (&oa)[9],
                                          int (&ob)[9])
{
#pragma unroll
    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
            const int y = oy * stride + ky - 1, x = ox * stride + kx - 1;
            const bool ok = live && y >= 0 && y < c.Hin && x >= 0 && x < c.Win;
            ob[ky * 3 + kx] = ok ? y * c.Win + x : -1;
            oa[ky * 3 + kx] = ok ? (c.up ? (y >> 1) * c.Wa + (x >> 1) : y * c.Win + x) : -1;
        }
}

__device__ __forceinline__ void conv_gather(const ConvIn &c, int n, int ci, const int (&oa)[9], const int (&ob)[9],
                                            float (&x)[9])
{
    if (ci < c.ca) {
        const float *src = c.a + ((size_t)n * c.ca + ci) * c.Ha * c.Wa;
#pragma unroll
        for (int t = 0; t < 9; ++t) x[t] = oa[t] >= 0 ? __ldg(src + oa[t]) : 0.f;
    } else {
        const float *src = c.b + ((size_t)n * c.cb + (ci - c.ca)) * c.Hin * c.Win;
#pragma unroll
        for (int t = 0; t < 9; ++t) x[t] = ob[t] >= 0 ? __ldg(src + ob[t]) : 0.f;
    }
}

// Forward convolution as a split-K implicit GEMM: a CTA computes 32 output pixels
// (lane = pixel) x COT output channels; its 8 warps take the input channels in turn, two
// per iteration (both channels' loads in flight before their FMAs), each staging those
// channels' COT x 9 weights in its own shared slice (FMAs read broadcasts); the partial
// sums are reduced through shared memory, which the weight slices alias.  The small
// vector grids of the coarse levels still fill the GPU this way.
constexpr int kConvWarps = 8;

template <int COT>
constexpr size_t conv_fwd_smem()
{
    const size_t w = (size_t)kConvWarps * 2 * 9 * COT, r = (size_t)kConvWarps * COT * 33;
    return (w > r ? w : r) * sizeof(float);
}

template <int COT>
__global__ void __launch_bounds__(256, 2) conv_fwd_kernel(const ConvFwd c)
{
    constexpr int NW = kConvWarps;
    extern __shared__ __align__(16) float csm[];
    float(*wsm)[2][9][COT] = reinterpret_cast<float(*)[2][9][COT]>(csm);  // [warp][buffer][tap][co]
    float(*red)[COT][33] = reinterpret_cast<float(*)[COT][33]>(csm);      // [warp][co][pixel]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = blockIdx.z / c.splits, split = blockIdx.z - n * c.splits, co0 = blockIdx.y * COT;
    const int HWo = c.Ho * c.Wo;
    const int p = blockIdx.x * 32 + lane;
    const bool live = p < HWo;
    const int oy = live ? p / c.Wo : 0, ox = live ? p - oy * c.Wo : 0;
    const int cin = c.in.ca + c.in.cb;
    int oa[9], ob[9];
    conv_taps(c.in, oy, ox, c.stride, live, oa, ob);
    float acc[COT];
#pragma unroll
    for (int k = 0; k < COT; ++k) acc[k] = 0.f;
    const int step = 2 * NW * c.splits;
    if constexpr (COT % 8 == 0) {
        // Each iteration's weights (raw BF16 chunks) and input taps are loaded into registers
        // one iteration ahead, so that their global latency overlaps the FMAs before them.
        constexpr int Q = COT / 8;                         // 16-byte chunks per tap run
        constexpr int WPL = (2 * 9 * Q + 31) / 32;         // chunks per lane
        uint4 wn[WPL];
        float xn0[9], xn1[9];
        auto prefetch = [&](int ci) {
            const int cj = ci + NW;
            const bool two = cj < cin;
#pragma unroll
            for (int i = 0; i < WPL; ++i) {
                const int e = lane + 32 * i;
                wn[i] = make_uint4(0u, 0u, 0u, 0u);
                if (e < 2 * 9 * Q) {
                    const int ch = e / (9 * Q), r = e - ch * (9 * Q), tap = r / Q, q = r - tap * Q;
                    if (ch == 0 || two)
                        wn[i] = __ldg(reinterpret_cast<const uint4 *>(c.w + ((size_t)(ch ? cj : ci) * 9 + tap) * c.cout + co0) + q);
                }
            }
            conv_gather(c.in, n, ci, oa, ob, xn0);
            if (two) {
                conv_gather(c.in, n, cj, oa, ob, xn1);
            } else {
#pragma unroll
                for (int t = 0; t < 9; ++t) xn1[t] = 0.f;
            }
        };
        int ci = split * 2 * NW + warp;
        if (ci < cin) prefetch(ci);
#pragma unroll 1
        for (; ci < cin; ci += step) {
            // this iteration's weights into the warp's slices (FMAs read broadcasts)
#pragma unroll
            for (int i = 0; i < WPL; ++i) {
                const int e = lane + 32 * i;
                if (e < 2 * 9 * Q) {
                    const int ch = e / (9 * Q), r = e - ch * (9 * Q), tap = r / Q, q = r - tap * Q;
                    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&wn[i]);
                    const float2 f0 = __bfloat1622float2(h[0]), f1 = __bfloat1622float2(h[1]);
                    const float2 f2 = __bfloat1622float2(h[2]), f3 = __bfloat1622float2(h[3]);
                    float4 *dst = reinterpret_cast<float4 *>(&wsm[warp][ch][tap][8 * q]);  // 16-byte stores
                    dst[0] = make_float4(f0.x, f0.y, f1.x, f1.y);
                    dst[1] = make_float4(f2.x, f2.y, f3.x, f3.y);
                }
            }
            float x0[9], x1[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                x0[t] = xn0[t];
                x1[t] = xn1[t];
            }
            __syncwarp();
            if (ci + step < cin) prefetch(ci + step);
#pragma unroll
            for (int t = 0; t < 9; ++t)
#pragma unroll
                for (int k = 0; k < COT; ++k) acc[k] = fmaf(wsm[warp][0][t][k], x0[t], acc[k]);
#pragma unroll
            for (int t = 0; t < 9; ++t)
#pragma unroll
                for (int k = 0; k < COT; ++k) acc[k] = fmaf(wsm[warp][1][t][k], x1[t], acc[k]);
            __syncwarp();
        }
    } else {
#pragma unroll 1
        for (int ci = split * 2 * NW + warp; ci < cin; ci += step) {
            const int cj = ci + NW;
            const bool two = cj < cin;
            for (int e = lane; e < 2 * 9 * COT; e += 32) {
                const int ch = e / (9 * COT), r = e - ch * (9 * COT), tap = r / COT, co = r - tap * COT;
                const int cc = ch ? cj : ci;
                const bool ok = co0 + co < c.cout && (ch == 0 || two);
                wsm[warp][ch][tap][co] = ok ? __bfloat162float(c.w[((size_t)cc * 9 + tap) * c.cout + co0 + co]) : 0.f;
            }
            __syncwarp();
            float x0[9], x1[9];
            conv_gather(c.in, n, ci, oa, ob, x0);
            if (two) conv_gather(c.in, n, cj, oa, ob, x1);
            else {
#pragma unroll
                for (int t = 0; t < 9; ++t) x1[t] = 0.f;
            }
#pragma unroll
            for (int t = 0; t < 9; ++t)
#pragma unroll
                for (int k = 0; k < COT; ++k) acc[k] = fmaf(wsm[warp][0][t][k], x0[t], acc[k]);
#pragma unroll
            for (int t = 0; t < 9; ++t)
#pragma unroll
                for (int k = 0; k < COT; ++k) acc[k] = fmaf(wsm[warp][1][t][k], x1[t], acc[k]);
            __syncwarp();
        }
    }
    __syncthreads();  // every warp is done with its weight slices: the reduction reuses them
#pragma unroll
    for (int k = 0; k < COT; ++k) red[warp][k][lane] = acc[k];
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * COT; e += 256) {
        const int k = e >> 5, l = e & 31;
        const int pp = blockIdx.x * 32 + l, co = co0 + k;
        if (pp >= HWo || co >= c.cout) continue;
        float v = 0.f;
#pragma unroll
        for (int w = 0; w < NW; ++w) v += red[w][k][l];
        if (c.splits > 1) {
            c.part[((size_t)blockIdx.z * c.cout + co) * HWo + pp] = v;
            continue;
        }
        v += c.bias[co];
        if (c.act) v = v > 0.f ? v : kSlope * v;
        c.out[((size_t)n * c.cout + co) * HWo + pp] = v;
    }
}

// bias + the splits' partial sums in split order + activation
__global__ void conv_finish_kernel(const float *part, int splits, const float *bias, int N, int cout, int HWo, int act,
                                   float *out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)N * cout * HWo) return;
    const int p = (int)(i % HWo);
    const size_t r = i / HWo;
    const int co = (int)(r % cout), n = (int)(r / cout);
    float v = 0.f;
    for (int sp = 0; sp < splits; ++sp) v += part[(((size_t)n * splits + sp) * cout + co) * HWo + p];
    v += bias[co];
    if (act) v = v > 0.f ? v : kSlope * v;
    out[i] = v;
}

// Forward convolution on the tensor cores, for stride-1 layers with 32 or 64 output
// channels over enough pixels: an implicit GEMM D[pixel][co] = sum_k A[pixel][k] W[co][k],
// k = (input channel, tap), on tcgen05 (kind::f16, FP32 accumulation in tensor memory).
//   - A CTA takes an 8 x 16 tile of output pixels (M = 128) with 512 threads, four per
//     pixel (a CTA holding tensor memory is resident once per SM, and 4 warps per SM left
//     every dependent instruction exposed).  Per block of 16 input channels it stages the
//     10 x 18 input patch (FP32, zero padded, through the upsampling / concatenation of the
//     layer's input) in shared memory and builds all 9 taps' operands from it: each thread
//     writes 4 of its pixel's 16 channel values as BF16 hi + lo pairs (x ~= hi + lo, about
//     16 significant bits) into the K-major A operand of each tap, and the threads copy
//     each tap's 16 x N weights ([ci][tap][co], BF16, exact) as the MN-major B operand.  After one barrier thread 0 issues the
//     block's 18 MMAs (D += A_hi W + A_lo W per tap) and one commit.
//   - Blocks alternate between two operand buffers: the tensor core works on block b while
//     the threads stage block b + 1.  The commit of block b - 2 on the buffer's mbarrier
//     frees it; every wait is bounded (kMaxTries probes), and a timeout sets bit 0 of
//     *status, skips the epilogue and still releases the tensor memory.
//   - Epilogue: warp w reads the accumulators of pixels 32 (w % 4) .. + 31 (its lane
//     quarter of tensor memory), 16 output channels per warpgroup (tcgen05.ld), adds the
//     bias, applies LeakyReLU and stores.
constexpr int kTcTY = 8, kTcTX = 16, kTcPY = kTcTY + 2, kTcPX = kTcTX + 2, kTcCB = 16;

template <int N>
struct ConvTcSmem {
    float patch[2][kTcCB][kTcPY][kTcPX];
    alignas(128) uint8_t a_hi[2][9][128 * kTcCB * 2];
    alignas(128) uint8_t a_lo[2][9][128 * kTcCB * 2];
    alignas(128) uint8_t b[2][9][N * kTcCB * 2];
    alignas(8) uint64_t mbar[3];
    uint32_t tmem_base;
};

// cp.async of one float into shared memory; zero-filled (nothing read) when !valid
__device__ __forceinline__ void cp_async_f32(uint32_t dst, const float *src, bool valid)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory"); }

// the input patch of channel block `blk` into `patch` by cp.async (one group per call):
// threads 0..359 each own one of the 180 patch positions for 8 of the 16 channels, so the
// position's bounds and offsets are worked out once (the channels are a plane apart)
__device__ __forceinline__ void conv_tc_patch(const ConvFwd &c, int n, int x0, int y0, int blk, int tid,
                                              float (*patch)[kTcPY][kTcPX])
{
    constexpr int NPOS = kTcPY * kTcPX;
    if (tid < 2 * NPOS) {
        const int pos = tid < NPOS ? tid : tid - NPOS, ch0 = tid < NPOS ? 0 : kTcCB / 2;
        const int py = pos / kTcPX, px = pos - py * kTcPX;
        const int y = y0 - 1 + py, x = x0 - 1 + px;
        const bool inside = y >= 0 && y < c.in.Hin && x >= 0 && x < c.in.Win;
        const int cin = c.in.ca + c.in.cb, cb0 = blk * kTcCB + ch0;
        const size_t plane_a = (size_t)c.in.Ha * c.in.Wa, plane_b = (size_t)c.in.Hin * c.in.Win;
        const int off_a = inside ? (c.in.up ? (y >> 1) * c.in.Wa + (x >> 1) : y * c.in.Win + x) : 0;
        const int off_b = inside ? y * c.in.Win + x : 0;
        const uint32_t dst = tc::smem_u32(&patch[ch0][py][px]);
#pragma unroll
        for (int q = 0; q < kTcCB / 2; ++q) {
            const int cc = cb0 + q;
            const bool ok = inside && cc < cin;
            const float *src = c.in.a;  // any valid address where nothing is read
            if (ok)
                src = cc < c.in.ca ? c.in.a + ((size_t)n * c.in.ca + cc) * plane_a + off_a
                                   : c.in.b + ((size_t)n * c.in.cb + (cc - c.in.ca)) * plane_b + off_b;
            cp_async_f32(dst + (uint32_t)(q * NPOS * 4), src, ok);
        }
    }
    cp_async_commit();
}

template <int N>
__global__ void __launch_bounds__(512, 1) conv_tc_kernel(const ConvFwd c, int *status)
{
    extern __shared__ __align__(128) uint8_t tc_raw[];
    ConvTcSmem<N> &S = *reinterpret_cast<ConvTcSmem<N> *>(tc_raw);
    constexpr uint32_t TCOLS = N < 32 ? 32 : N;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int n = blockIdx.z, x0 = blockIdx.x * kTcTX, y0 = blockIdx.y * kTcTY;
    const int px_id = tid >> 2, quarter = tid & 3;  // the pixel (A row) and the 4 channels this thread builds
    const int ty = px_id >> 4, tx = px_id & 15;
    const int cin = c.in.ca + c.in.cb, nblk = (cin + kTcCB - 1) / kTcCB;
    if (tid == 0) {
        for (int i = 0; i < 3; ++i) tc::mbar_init(tc::smem_u32(&S.mbar[i]), 1);
        tc::fence_mbar_init();
    }
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tmem_base), TCOLS);
    conv_tc_patch(c, n, x0, y0, 0, tid, S.patch[0]);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = S.tmem_base;
    constexpr uint32_t idesc = tc::idesc_f16(N, false, true, true);
    // K-major A: byte (k/8)*2048 + m*16 + (k%8)*2 with m = px_id; this thread's channels
    // k = 4*quarter .. + 3 are 8 bytes at (quarter/2)*2048 + m*16 + (quarter%2)*8
    const uint32_t a_off = (uint32_t)(quarter >> 1) * 2048u + (uint32_t)px_id * 16u + (uint32_t)(quarter & 1) * 8u;
    // the 9 taps' weights of a channel block, (tap, g = co/8, k) at byte (co/8)*256 + k*16 of
    // the tap's B operand: loaded into registers one block ahead (their global latency
    // overlaps the operand build of the block before), stored once the buffer is free
    constexpr int WPT = (9 * 2 * N + 511) / 512;  // 16-byte chunks per thread
    uint4 wreg[WPT];
    auto load_w = [&](int b) {
#pragma unroll
        for (int i = 0; i < WPT; ++i) {
            const int e = tid + 512 * i;
            wreg[i] = make_uint4(0u, 0u, 0u, 0u);
            if (e < 9 * 2 * N) {
                const int tap = e / (2 * N), r = e - tap * (2 * N), g = r / kTcCB, k = r - g * kTcCB;
                const int cc = b * kTcCB + k;
                if (cc < cin) wreg[i] = __ldg(reinterpret_cast<const uint4 *>(c.w + ((size_t)cc * 9 + tap) * c.cout) + g);
            }
        }
    };
    auto store_w = [&](int bb) {
#pragma unroll
        for (int i = 0; i < WPT; ++i) {
            const int e = tid + 512 * i;
            if (e < 9 * 2 * N) {
                const int tap = e / (2 * N), r = e - tap * (2 * N), g = r / kTcCB, k = r - g * kTcCB;
                reinterpret_cast<uint4 *>(S.b[bb][tap])[g * kTcCB + k] = wreg[i];
            }
        }
    };
    load_w(0);
    bool ok = true;
    int blk = 0;
    for (; blk < nblk; ++blk) {
        const int bb = blk & 1;
        // the next block's patch streams in while this one is built (its buffer was last
        // read by block blk - 1's operand build, finished before that block's MMA barrier)
        if (blk + 1 < nblk) {
            conv_tc_patch(c, n, x0, y0, blk + 1, tid, S.patch[bb ^ 1]);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        if (blk >= 2) {
            // the MMAs of block blk - 2 read this block's operand buffers: wait for their commit
            const bool done = tc::mbar_wait(tc::smem_u32(&S.mbar[bb]), ((blk >> 1) - 1) & 1);
            if (!__syncthreads_and(done)) {
                ok = false;
                break;
            }
            tc::fence_after_sync();
        } else {
            __syncthreads();  // every thread's patch copies have landed
        }
        float(*patch)[kTcPY][kTcPX] = S.patch[bb];
        store_w(bb);
        if (blk + 1 < nblk) load_w(blk + 1);
#pragma unroll 1
        for (int tap = 0; tap < 9; ++tap) {
            const int ky = tap / 3, kx = tap - ky * 3;
            uint32_t hi[2], lo[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int k = 4 * quarter + 2 * j;
                tc::split_bf16x2(patch[k][ty + ky][tx + kx], patch[k + 1][ty + ky][tx + kx], hi[j], lo[j]);
            }
            *reinterpret_cast<uint2 *>(S.a_hi[bb][tap] + a_off) = make_uint2(hi[0], hi[1]);
            *reinterpret_cast<uint2 *>(S.a_lo[bb][tap] + a_off) = make_uint2(lo[0], lo[1]);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            for (int tap = 0; tap < 9; ++tap) {
                const uint64_t bd = tc::smem_desc(tc::smem_u32(S.b[bb][tap]), 128, 256);
                tc::mma_f16(tmem, tc::smem_desc(tc::smem_u32(S.a_hi[bb][tap]), 2048, 128), bd, idesc,
                            (blk > 0 || tap > 0) ? 1u : 0u);
                tc::mma_f16(tmem, tc::smem_desc(tc::smem_u32(S.a_lo[bb][tap]), 2048, 128), bd, idesc, 1u);
            }
            tc::mma_commit(tc::smem_u32(&S.mbar[bb]));
        }
    }
    cp_async_wait<0>();  // no copy outlives the CTA (the early exit leaves one in flight)
    if (tid == 0 && ok) tc::mma_commit(tc::smem_u32(&S.mbar[2]));
    const bool fin = ok && __syncthreads_and(tc::mbar_wait(tc::smem_u32(&S.mbar[2]), 0));
    if (!fin) {
        if (tid == 0 && status) atomicOr(status, 1);
        // the block in flight gets one more bounded wait before the tensor memory is released
        if (blk > 0) tc::mbar_wait(tc::smem_u32(&S.mbar[(blk - 1) & 1]), ((blk - 1) >> 1) & 1);
    } else if (warp / 4 < N / 16) {
        tc::fence_after_sync();
        const int lq = warp & 3, c0 = (warp >> 2) * 16;   // lane quarter, 16 output channels
        const int pe = lq * 32 + (tid & 31);              // this thread's pixel in the epilogue
        const int y = y0 + (pe >> 4), x = x0 + (pe & 15);
        const bool live = y < c.Ho && x < c.Wo;
        const int HWo = c.Ho * c.Wo;
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(lq * 32) << 16) + c0, v);
        tc::tmem_wait_ld();
        if (live) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                float o = v[k] + c.bias[c0 + k];
                if (c.act) o = o > 0.f ? o : kSlope * o;
                c.out[((size_t)n * c.cout + c0 + k) * HWo + y * c.Wo + x] = o;
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, TCOLS);
}

template <int N>
cudaError_t launch_conv_tc(const ConvFwd &c, int *status, cudaStream_t s)
{
    const size_t smem = sizeof(ConvTcSmem<N>);
    cudaError_t e = cudaFuncSetAttribute(conv_tc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((c.Wo + kTcTX - 1) / kTcTX, (c.Ho + kTcTY - 1) / kTcTY, c.N);
    conv_tc_kernel<N><<<grid, 512, smem, s>>>(c, status);
    return cudaGetLastError();
}

// dIn of the concatenated (upsampled) input, [N][ca+cb][Hin][Win], overwritten.
struct ConvBwdData {
    int N, cin, Hin, Win, Ho, Wo, stride, cout;
    const __nv_bfloat16 *w;
    const float *g;  // [N][cout][Ho][Wo], activation gradient already applied
    float *din;
};

template <int CIB>
__global__ void __launch_bounds__(128) conv_bwd_data_kernel(const ConvBwdData c)
{
    constexpr int COC = 8;
    __shared__ __align__(16) float ws[COC][9][CIB];
    const int n = blockIdx.z, ci0 = blockIdx.y * CIB;
    const int p = blockIdx.x * 128 + threadIdx.x;
    const bool live = p < c.Hin * c.Win;
    const int y = live ? p / c.Win : 0, x = live ? p - y * c.Win : 0;
    // output pixel fed by each tap: y = oy*s + ky - 1  =>  oy = (y + 1 - ky) / s
    int og[9];
#pragma unroll
    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
            const int ny = y + 1 - ky, nx = x + 1 - kx;
            int oy = -1, ox = -1;
            if (c.stride == 1) {
                oy = ny;
                ox = nx;
            } else if (ny >= 0 && nx >= 0 && !(ny & 1) && !(nx & 1)) {
                oy = ny >> 1;
                ox = nx >> 1;
            }
            const bool ok = live && oy >= 0 && oy < c.Ho && ox >= 0 && ox < c.Wo;
            og[ky * 3 + kx] = ok ? oy * c.Wo + ox : -1;
        }
    float acc[CIB];
#pragma unroll
    for (int k = 0; k < CIB; ++k) acc[k] = 0.f;
    for (int co0 = 0; co0 < c.cout; co0 += COC) {
        __syncthreads();
        for (int e = threadIdx.x; e < COC * 9 * CIB; e += 128) {
            const int ci = e % CIB, r = e / CIB, tap = r % 9, co = r / 9;
            float wv = 0.f;
            if (co0 + co < c.cout && ci0 + ci < c.cin)
                wv = __bfloat162float(c.w[((size_t)(co0 + co) * c.cin + ci0 + ci) * 9 + tap]);
            ws[co][tap][ci] = wv;
        }
        __syncthreads();
        const int nco = min(COC, c.cout - co0);
#pragma unroll 1
        for (int co = 0; co < nco; ++co) {
            const float *src = c.g + ((size_t)n * c.cout + co0 + co) * c.Ho * c.Wo;
            float gv[9];
#pragma unroll
            for (int t = 0; t < 9; ++t) gv[t] = og[t] >= 0 ? __ldg(src + og[t]) : 0.f;
#pragma unroll
            for (int t = 0; t < 9; ++t)
#pragma unroll
                for (int k = 0; k < CIB; ++k) acc[k] = fmaf(ws[co][t][k], gv[t], acc[k]);
        }
    }
    if (!live) return;
#pragma unroll
    for (int k = 0; k < CIB; ++k) {
        const int ci = ci0 + k;
        if (ci >= c.cin) break;
        c.din[((size_t)n * c.cin + ci) * c.Hin * c.Win + p] = acc[k];
    }
}

// dW[co][ci][tap] and db[co]: one CTA per (input channel, COC output channels), threads
// over the N*Ho*Wo output pixels, then a block reduction.  Overwrites its outputs.
struct ConvBwdW {
    ConvIn in;
    int N, Ho, Wo, stride, cout;
    const float *g;
    float *dw, *db;
};

template <int COC>
__global__ void __launch_bounds__(256) conv_bwd_w_kernel(const ConvBwdW c)
{
    constexpr int NV = COC * 10;  // 9 taps + bias per output channel
    __shared__ float red[8][NV];
    const int ci = blockIdx.x, co0 = blockIdx.y * COC;
    const int cin = c.in.ca + c.in.cb;
    const int HW = c.Ho * c.Wo, npix = c.N * HW;
    float acc[COC][10];
#pragma unroll
    for (int k = 0; k < COC; ++k)
#pragma unroll
        for (int t = 0; t < 10; ++t) acc[k][t] = 0.f;
    for (int q = threadIdx.x; q < npix; q += 256) {
        const int n = q / HW, p = q - n * HW;
        const int oy = p / c.Wo, ox = p - oy * c.Wo;
        int oa[9], ob[9];
        conv_taps(c.in, oy, ox, c.stride, true, oa, ob);
        float x[9];
        conv_gather(c.in, n, ci, oa, ob, x);
#pragma unroll
        for (int k = 0; k < COC; ++k) {
            const int co = co0 + k;
            const float gv = co < c.cout ? __ldg(c.g + ((size_t)n * c.cout + co) * HW + p) : 0.f;
#pragma unroll
            for (int t = 0; t < 9; ++t) acc[k][t] = fmaf(gv, x[t], acc[k][t]);
            acc[k][9] += gv;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < COC; ++k)
#pragma unroll
        for (int t = 0; t < 10; ++t) {
            float v = acc[k][t];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][k * 10 + t] = v;
        }
    __syncthreads();
    for (int e = threadIdx.x; e < NV; e += 256) {
        float s = 0.f;
#pragma unroll
        for (int w = 0; w < 8; ++w) s += red[w][e];
        const int k = e / 10, t = e - k * 10, co = co0 + k;
        if (co >= c.cout) continue;
        if (t < 9) c.dw[((size_t)co * cin + ci) * 9 + t] = s;
        else if (ci == 0) c.db[co] = s;
    }
}

// g *= LeakyReLU'(pre-activation), read from the layer output's sign
__global__ void act_bwd_kernel(float *g, const float *out, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(out[i] > 0.f)) g[i] *= kSlope;
}

// Route dIn of a concatenated input back: ga (+=, summing the 2x2 fine pixels of each
// coarse pixel when a was upsampled) and gb (+=).
__global__ void split_grad_kernel(const float *din, int N, int ca, int cb, int up, int Hin, int Win, int Ha, int Wa,
                                  float *ga, float *gb)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t na = ga ? (size_t)N * ca * Ha * Wa : 0, nb = gb ? (size_t)N * cb * Hin * Win : 0;
    const int cin = ca + cb;
    if (i < na) {
        const int X = (int)(i % Wa);
        size_t r = i / Wa;
        const int Y = (int)(r % Ha);
        r /= Ha;
        const int ch = (int)(r % ca), n = (int)(r / ca);
        const float *src = din + ((size_t)n * cin + ch) * Hin * Win;
        float s;
        if (up) {
            s = 0.f;
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const int y = 2 * Y + dy, x = 2 * X + dx;
                    if (y < Hin && x < Win) s += src[y * Win + x];
                }
        } else {
            s = src[Y * Win + X];
        }
        ga[i] += s;
    } else if (i < na + nb) {
        const size_t j = i - na;
        const int x = (int)(j % Win);
        size_t r = j / Win;
        const int y = (int)(r % Hin);
        r /= Hin;
        const int ch = (int)(r % cb), n = (int)(r / cb);
        gb[j] += din[((size_t)n * cin + ca + ch) * Hin * Win + y * Win + x];
    }
}

// Charbonnier loss on the head (downsampled px): sum over masked vectors of
// sqrt(e^2 + eps^2) - eps per component, times inv_count; its gradient into gpred.
__global__ void loss_kernel(const float *pred, const float *label, const float *mask, int N, int HW, float inv_count,
                            float *gpred, float *loss)
{
    constexpr float eps = 0.01f;
    __shared__ float red[8];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (i < N * HW) {
        const int n = i / HW, p = i - n * HW;
        const float m = mask[i] * inv_count;
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            const size_t o = ((size_t)n * 2 + ch) * HW + p;
            const float e = pred[o] - label[o];
            const float r = sqrtf(e * e + eps * eps);
            l += m * (r - eps);
            gpred[o] = m * e / r;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        atomicAdd(loss, s);
    }
}

// Adam (Kingma & Ba, 2015) with bias correction; refreshes the BF16 copies.
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, __nv_bfloat16 *pb, size_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    p[i] = pi;
    pb[i] = __float2bfloat16_rn(pi);
}

__global__ void to_bf16_kernel(const float *p, __nv_bfloat16 *pb, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pb[i] = __float2bfloat16_rn(p[i]);
}

// One layer's weights [co][ci][tap] (FP32 masters) -> the forward's BF16 [ci][tap][co]
__global__ void transpose_weights_kernel(const float *w, int cout, int cin, __nv_bfloat16 *wt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // index in the source layout
    if (i >= cout * cin * 9) return;
    const int co = i / (cin * 9), r = i - co * (cin * 9), ci = r / 9, tap = r - ci * 9;
    wt[((size_t)ci * 9 + tap) * cout + co] = __float2bfloat16_rn(w[i]);
}

__global__ void field_from_net_kernel(const float *out, int Nt, float *fx, float *fy, uint8_t *fv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nt) return;
    fx[i] = kOutScale * out[i];
    fy[i] = kOutScale * out[Nt + i];
    fv[i] = 1;
}

cudaError_t launch_field_from_net(const float *out, int Nt, float *fx, float *fy, uint8_t *fv, cudaStream_t s)
{
    field_from_net_kernel<<<(Nt + 255) / 256, 256, 0, s>>>(out, Nt, fx, fy, fv);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256) judge_kernel(const float *px, const float *py, const float *fx,
                                                    const float *fy, int Nt, const int *list_n, float *judge)
{
    __shared__ float red[8];
    float s = 0.f;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < Nt; i += gridDim.x * 256) {
        const float dx = px[i] - fx[i], dy = py[i] - fy[i];
        s = fmaf(dx, dx, fmaf(dy, dy, s));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int w = 0; w < 8; ++w) v += red[w];
        atomicAdd(judge, v);
        if (blockIdx.x == 0) judge[1] = (float)*list_n;
    }
}

cudaError_t launch_judge(const float *px, const float *py, const float *fx, const float *fy, int Nt,
                         const int *list_n, float *judge, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(judge, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
    const int blocks = std::max(1, std::min((Nt + 255) / 256, 148));
    judge_kernel<<<blocks, 256, 0, s>>>(px, py, fx, fy, Nt, list_n, judge);
    return cudaGetLastError();
}

}  // namespace learned
}  // namespace piv

using namespace piv;
using namespace piv::learned;

struct piv_net {
    int device = 0;
    size_t n_params = 0;
    size_t w_off[kLayers] = {}, b_off[kLayers] = {};
    float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    __nv_bfloat16 *wbf = nullptr;
    // the forward's copy of the BF16 weights, [ci][tap][co] per layer (16-byte aligned
    // layers): an input channel's weights for all output channels are contiguous
    __nv_bfloat16 *wt = nullptr;
    size_t wt_off[kLayers] = {};
    size_t wt_total = 0;
    int step = 0;
    // activations for (aN, aH, aW)
    int aN = 0, aH = 0, aW = 0;
    int lh[4] = {}, lw[4] = {};
    size_t t_off[kTensors] = {};
    size_t act_floats = 0, din_floats = 0, part_floats = 0;
    float *act = nullptr, *gact = nullptr, *din = nullptr, *part = nullptr;
    int splits[kLayers] = {};
    float *d_loss = nullptr, *h_loss = nullptr;
    // features scratch
    float *fdown = nullptr;
    double *fsums = nullptr;
    size_t fcap = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int *d_status = nullptr;  // bit 0: a tensor-core convolution's MMA wait timed out
    bool use_tc = true;       // tensor-core forward for the wide stride-1 layers (PIV_NET_TC=0: off)
    // drawn from a process-wide counter at creation and whenever a buffer a captured graph
    // may hold is reallocated or re-laid-out, so (net, generation) never repeats
    unsigned generation = 0;
};

namespace {

unsigned next_generation()
{
    static std::atomic<unsigned> g{0};
    return ++g;
}

int net_err(piv_net *n, int code, const char *msg)
{
    if (n) n->err = msg;
    return code;
}

#define NCK(call)                                                                   \
    do {                                                                            \
        cudaError_t _e = (call);                                                    \
        if (_e != cudaSuccess) return net_err(n, PIV_ERR_CUDA, cudaGetErrorString(_e)); \
    } while (0)

void layout(piv_net *n, int N, int H, int W)
{
    n->lh[0] = H;
    n->lw[0] = W;
    for (int l = 1; l < 4; ++l) {
        n->lh[l] = (n->lh[l - 1] + 1) / 2;
        n->lw[l] = (n->lw[l - 1] + 1) / 2;
    }
    size_t off = 0;
    for (int t = 0; t < kTensors; ++t) {
        n->t_off[t] = off;
        const size_t sz = (size_t)N * kChan[t] * n->lh[kLevel[t]] * n->lw[kLevel[t]];
        off += (sz + 31) & ~(size_t)31;
    }
    n->act_floats = off;
    size_t dmax = 0;
    for (int i = 0; i < kLayers; ++i) {
        const LayerSpec &s = kSpec[i];
        const int lin = s.up ? kLevel[s.b] : kLevel[s.a];
        dmax = std::max(dmax, (size_t)N * (s.ca + s.cb) * n->lh[lin] * n->lw[lin]);
    }
    n->din_floats = dmax;
    // input-channel splits of the forward convolutions: enough CTAs for two per SM, at
    // least 16 input channels (two per warp) per split
    size_t pmax = 0;
    for (int i = 0; i < kLayers; ++i) {
        const LayerSpec &s = kSpec[i];
        const int lo = kLevel[i + 1], cin = s.ca + s.cb;
        const int px = n->lh[lo] * n->lw[lo];
        const long ctas = (long)((px + 31) / 32) * ((s.cout + 31) / 32) * N;
        const int smax = std::max(1, cin / 16);
        int sp = (int)std::min<long>(smax, std::max<long>(1, (2 * 148 + ctas - 1) / ctas));
        if (s.cout % 32) sp = 1;
        n->splits[i] = sp;
        if (sp > 1) pmax = std::max(pmax, (size_t)N * sp * s.cout * px);
    }
    n->part_floats = pmax;
}

ConvIn conv_in(piv_net *n, const float *base, int i, int N)
{
    (void)N;
    const LayerSpec &s = kSpec[i];
    ConvIn c;
    c.a = base + n->t_off[s.a];
    c.b = s.b >= 0 ? base + n->t_off[s.b] : nullptr;
    c.ca = s.ca;
    c.cb = s.cb;
    c.up = s.up;
    const int la = kLevel[s.a];
    const int lin = s.up ? kLevel[s.b] : la;
    c.Hin = n->lh[lin];
    c.Win = n->lw[lin];
    c.Ha = n->lh[la];
    c.Wa = n->lw[la];
    return c;
}

// the forward's weight copy from the FP32 masters (after every change of the weights)
cudaError_t refresh_forward_weights(piv_net *n, cudaStream_t s)
{
    for (int i = 0; i < kLayers; ++i) {
        const int cin = kSpec[i].ca + kSpec[i].cb, cout = kSpec[i].cout, nw = cout * cin * 9;
        transpose_weights_kernel<<<(nw + 255) / 256, 256, 0, s>>>(n->params + n->w_off[i], cout, cin,
                                                                  n->wt + n->wt_off[i]);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t forward_layers(piv_net *n, float *act, int N, cudaStream_t s)
{
    for (int i = 0; i < kLayers; ++i) {
        const LayerSpec &sp = kSpec[i];
        ConvFwd c;
        c.in = conv_in(n, act, i, N);
        const int lo = kLevel[i + 1];
        c.N = N;
        c.Ho = n->lh[lo];
        c.Wo = n->lw[lo];
        c.stride = sp.stride;
        c.w = n->wt + n->wt_off[i];
        c.bias = n->params + n->b_off[i];
        c.cout = sp.cout;
        c.out = act + n->t_off[i + 1];
        c.act = sp.act;
        c.splits = n->splits[i];
        c.part = n->part;
        const int px = c.Ho * c.Wo;
        if (n->use_tc && sp.stride == 1 && (sp.cout == 32 || sp.cout == 64) && (long)N * px >= 4096) {
            cudaError_t e = sp.cout == 32 ? launch_conv_tc<32>(c, n->d_status, s) : launch_conv_tc<64>(c, n->d_status, s);
            if (e != cudaSuccess) return e;
            continue;
        }
        if (sp.cout % 32 == 0) {
            conv_fwd_kernel<32><<<dim3((px + 31) / 32, sp.cout / 32, N * c.splits), 256, conv_fwd_smem<32>(), s>>>(c);
        } else {
            conv_fwd_kernel<2><<<dim3((px + 31) / 32, (sp.cout + 1) / 2, N * c.splits), 256, conv_fwd_smem<2>(), s>>>(c);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (c.splits > 1) {
            const size_t tot = (size_t)N * sp.cout * px;
            conv_finish_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n->part, c.splits, c.bias, N, sp.cout, px,
                                                                            sp.act, c.out);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace

namespace piv {
namespace learned {

int net_reserve(piv_net *n, int N, int H, int W)
{
    if (!n || N < 1 || H < 1 || W < 1) return PIV_ERR_ARG;
    if (n->act && n->aN == N && n->aH == H && n->aW == W) return PIV_OK;
    cudaSetDevice(n->device);
    n->generation = next_generation();
    const size_t old_act = n->act ? n->act_floats : 0, old_din = n->act ? n->din_floats : 0;
    const size_t old_part = n->act ? n->part_floats : 0;
    layout(n, N, H, W);
    if (n->act_floats > old_act || n->din_floats > old_din || n->part_floats > old_part || !n->act) {
        cudaFree(n->act);
        cudaFree(n->gact);
        cudaFree(n->din);
        cudaFree(n->part);
        n->act = n->gact = n->din = n->part = nullptr;
        NCK(cudaMalloc(&n->act, n->act_floats * sizeof(float)));
        NCK(cudaMalloc(&n->gact, n->act_floats * sizeof(float)));
        NCK(cudaMalloc(&n->din, n->din_floats * sizeof(float)));
        NCK(cudaMalloc(&n->part, std::max<size_t>(n->part_floats, 1) * sizeof(float)));
    } else {
        n->act_floats = std::max(n->act_floats, old_act);
        n->din_floats = std::max(n->din_floats, old_din);
        n->part_floats = std::max(n->part_floats, old_part);
    }
    n->aN = N;
    n->aH = H;
    n->aW = W;
    return PIV_OK;
}

float *net_input(piv_net *n) { return n->act + n->t_off[0]; }
const float *net_output(piv_net *n) { return n->act + n->t_off[kTensors - 1]; }

cudaError_t net_forward(piv_net *n, const float *in, int N, int H, int W, float *out, cudaStream_t s)
{
    if (!n->act || n->aN != N || n->aH != H || n->aW != W) return cudaErrorInvalidValue;
    float *t0 = n->act + n->t_off[0];
    const size_t nin = (size_t)N * kInChannels * H * W;
    cudaError_t e;
    if (in != t0 && (e = cudaMemcpyAsync(t0, in, nin * sizeof(float), cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
        return e;
    if ((e = forward_layers(n, n->act, N, s)) != cudaSuccess) return e;
    const float *t13 = n->act + n->t_off[kTensors - 1];
    if (out && out != t13)
        return cudaMemcpyAsync(out, t13, (size_t)N * 2 * H * W * sizeof(float), cudaMemcpyDeviceToDevice, s);
    return cudaSuccess;
}

int net_reserve_features(piv_net *n, int Nx, int Ny)
{
    const size_t need = feature_scratch_floats(Nx, Ny);
    if (n->fdown && n->fcap >= need) return PIV_OK;
    cudaSetDevice(n->device);
    n->generation = next_generation();
    cudaFree(n->fdown);
    n->fdown = nullptr;
    NCK(cudaMalloc(&n->fdown, need * sizeof(float)));
    if (!n->fsums) NCK(cudaMalloc(&n->fsums, 2 * sizeof(double)));
    n->fcap = need;
    return PIV_OK;
}

unsigned net_generation(const piv_net *n) { return n->generation; }

int net_check_status(piv_net *n)
{
    int st = 0;
    if (cudaMemcpy(&st, n->d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return PIV_ERR_CUDA;
    if (!st) return PIV_OK;
    cudaMemset(n->d_status, 0, sizeof(int));
    n->err = "a tensor-core convolution's MMA completion wait timed out";
    return PIV_ERR_DEVICE;
}
float *net_feature_down(piv_net *n) { return n->fdown; }
double *net_feature_sums(piv_net *n) { return n->fsums; }

}  // namespace learned
}  // namespace piv

// ------------------------------------------------------------------------------
// C-ABI
// ------------------------------------------------------------------------------
extern "C" {

int piv_net_create(uint64_t seed, piv_net **out)
{
    if (!out) return PIV_ERR_ARG;
    *out = nullptr;
    piv_net *n = new piv_net;
    n->generation = next_generation();
    cudaGetDevice(&n->device);
    size_t off = 0;
    for (int i = 0; i < kLayers; ++i) {
        n->w_off[i] = off;
        off += (size_t)kSpec[i].cout * (kSpec[i].ca + kSpec[i].cb) * 9;
        n->b_off[i] = off;
        off += kSpec[i].cout;
    }
    n->n_params = off;
    size_t woff = 0;
    for (int i = 0; i < kLayers; ++i) {
        n->wt_off[i] = woff;
        woff += ((size_t)kSpec[i].cout * (kSpec[i].ca + kSpec[i].cb) * 9 + 7) & ~(size_t)7;  // 16-byte layers
    }
    n->wt_total = woff;
    // He-uniform weights for LeakyReLU (bound sqrt(6 / ((1 + slope^2) fan_in))), a head
    // scaled by 0.1, zero biases; Philox stream 4 of the seed
    std::vector<float> h(off, 0.f);
    for (int i = 0; i < kLayers; ++i) {
        const int fan_in = (kSpec[i].ca + kSpec[i].cb) * 9;
        double bound = std::sqrt(6.0 / ((1.0 + kSlope * kSlope) * fan_in));
        if (!kSpec[i].act) bound *= 0.1;
        const size_t nw = (size_t)kSpec[i].cout * fan_in;
        for (size_t k = 0; k < nw; ++k) {
            const U4 r = philox((uint32_t)k, (uint32_t)i, 4, 0, seed);
            h[n->w_off[i] + k] = (float)((2.0 * u01(r.v[0]) - 1.0) * bound);
        }
    }
    int rc = PIV_OK;
    auto fail = [&](int code) {
        rc = code;
        cudaFree(n->params);
        cudaFree(n->grads);
        cudaFree(n->adam_m);
        cudaFree(n->adam_v);
        cudaFree(n->wbf);
        cudaFree(n->wt);
        cudaFree(n->d_loss);
        cudaFree(n->d_status);
        if (n->h_loss) cudaFreeHost(n->h_loss);
        if (n->stream) cudaStreamDestroy(n->stream);
        delete n;
        return rc;
    };
    if (cudaMalloc(&n->params, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&n->grads, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&n->adam_m, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&n->adam_v, off * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&n->wbf, off * sizeof(__nv_bfloat16)) != cudaSuccess ||
        cudaMalloc(&n->wt, n->wt_total * sizeof(__nv_bfloat16)) != cudaSuccess ||
        cudaMalloc(&n->d_loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&n->d_status, sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&n->h_loss, sizeof(float)) != cudaSuccess ||
        cudaStreamCreate(&n->stream) != cudaSuccess)  // blocking: ordered after default-stream work
        return fail(PIV_ERR_CUDA);
    if (cudaMemcpy(n->params, h.data(), off * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(n->adam_m, 0, off * sizeof(float)) != cudaSuccess ||
        cudaMemset(n->adam_v, 0, off * sizeof(float)) != cudaSuccess ||
        cudaMemset(n->grads, 0, off * sizeof(float)) != cudaSuccess ||
        cudaMemset(n->d_status, 0, sizeof(int)) != cudaSuccess)
        return fail(PIV_ERR_CUDA);
    if (const char *tc = getenv("PIV_NET_TC")) n->use_tc = tc[0] != '0';
    to_bf16_kernel<<<(unsigned)((off + 255) / 256), 256, 0, n->stream>>>(n->params, n->wbf, off);
    if (refresh_forward_weights(n, n->stream) != cudaSuccess || cudaStreamSynchronize(n->stream) != cudaSuccess)
        return fail(PIV_ERR_CUDA);
    *out = n;
    return PIV_OK;
}

int piv_net_destroy(piv_net *n)
{
    if (!n) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    cudaFree(n->params);
    cudaFree(n->grads);
    cudaFree(n->adam_m);
    cudaFree(n->adam_v);
    cudaFree(n->wbf);
    cudaFree(n->wt);
    cudaFree(n->act);
    cudaFree(n->gact);
    cudaFree(n->din);
    cudaFree(n->part);
    cudaFree(n->d_loss);
    cudaFree(n->d_status);
    cudaFree(n->fdown);
    cudaFree(n->fsums);
    if (n->h_loss) cudaFreeHost(n->h_loss);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
    return PIV_OK;
}

const char *piv_net_last_error(const piv_net *n) { return n ? n->err.c_str() : "null net"; }

int piv_net_num_params(const piv_net *n, int64_t *count)
{
    if (!n || !count) return PIV_ERR_ARG;
    *count = (int64_t)n->n_params;
    return PIV_OK;
}

int piv_net_layout(int layer, int *cin, int *cout, int *stride, int *weight_offset, int *bias_offset)
{
    if (layer < 0 || layer >= kLayers) return PIV_ERR_ARG;
    size_t off = 0;
    for (int i = 0; i < layer; ++i) off += (size_t)kSpec[i].cout * ((kSpec[i].ca + kSpec[i].cb) * 9 + 1);
    const LayerSpec &s = kSpec[layer];
    if (cin) *cin = s.ca + s.cb;
    if (cout) *cout = s.cout;
    if (stride) *stride = s.stride;
    if (weight_offset) *weight_offset = (int)off;
    if (bias_offset) *bias_offset = (int)(off + (size_t)s.cout * (s.ca + s.cb) * 9);
    return PIV_OK;
}

int piv_net_get_params(piv_net *n, float *host, int64_t count)
{
    if (!n || !host || count != (int64_t)n->n_params) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    NCK(cudaStreamSynchronize(n->stream));
    NCK(cudaMemcpy(host, n->params, n->n_params * sizeof(float), cudaMemcpyDeviceToHost));
    return PIV_OK;
}

int piv_net_set_params(piv_net *n, const float *host, int64_t count)
{
    if (!n || !host || count != (int64_t)n->n_params) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    NCK(cudaStreamSynchronize(n->stream));
    NCK(cudaMemcpy(n->params, host, n->n_params * sizeof(float), cudaMemcpyHostToDevice));
    NCK(cudaMemset(n->adam_m, 0, n->n_params * sizeof(float)));
    NCK(cudaMemset(n->adam_v, 0, n->n_params * sizeof(float)));
    n->step = 0;
    to_bf16_kernel<<<(unsigned)((n->n_params + 255) / 256), 256, 0, n->stream>>>(n->params, n->wbf, n->n_params);
    NCK(cudaGetLastError());
    NCK(refresh_forward_weights(n, n->stream));
    NCK(cudaStreamSynchronize(n->stream));
    return PIV_OK;
}

int piv_net_get_grads(piv_net *n, float *host, int64_t count)
{
    if (!n || !host || count != (int64_t)n->n_params) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    NCK(cudaStreamSynchronize(n->stream));
    NCK(cudaMemcpy(host, n->grads, n->n_params * sizeof(float), cudaMemcpyDeviceToHost));
    return PIV_OK;
}

// weights file: "PIVNET01", uint64 count, count float32 (little-endian)
int piv_net_save(piv_net *n, const char *path)
{
    if (!n || !path) return PIV_ERR_ARG;
    std::vector<float> h(n->n_params);
    int rc = piv_net_get_params(n, h.data(), (int64_t)h.size());
    if (rc) return rc;
    FILE *f = fopen(path, "wb");
    if (!f) return net_err(n, PIV_ERR_IO, "cannot open the weights file for writing");
    const uint64_t cnt = h.size();
    bool ok = fwrite("PIVNET01", 1, 8, f) == 8 && fwrite(&cnt, 8, 1, f) == 1 &&
              fwrite(h.data(), sizeof(float), h.size(), f) == h.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? PIV_OK : net_err(n, PIV_ERR_IO, "short write of the weights file");
}

int piv_net_load(piv_net *n, const char *path)
{
    if (!n || !path) return PIV_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return net_err(n, PIV_ERR_IO, "cannot open the weights file");
    char magic[8];
    uint64_t cnt = 0;
    std::vector<float> h;
    bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "PIVNET01", 8) == 0 && fread(&cnt, 8, 1, f) == 1 &&
              cnt == n->n_params;
    if (ok) {
        h.resize(cnt);
        ok = fread(h.data(), sizeof(float), cnt, f) == cnt;
    }
    fclose(f);
    if (!ok) return net_err(n, PIV_ERR_IO, "not a weights file of this network");
    return piv_net_set_params(n, h.data(), (int64_t)cnt);
}

int piv_net_forward(piv_net *n, const float *d_in, int N, int H, int W, float *d_out, void *stream)
{
    if (!n || !d_in || !d_out) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    int rc = net_reserve(n, N, H, W);
    if (rc) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : n->stream;
    NCK(net_forward(n, d_in, N, H, W, d_out, s));
    return PIV_OK;
}

int piv_net_loss_grad(piv_net *n, const float *d_in, const float *d_label, const float *d_mask, int N, int H, int W,
                      float *loss)
{
    if (!n || !d_in || !d_label || !d_mask) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    int rc = net_reserve(n, N, H, W);
    if (rc) return rc;
    cudaStream_t s = n->stream;
    NCK(net_forward(n, d_in, N, H, W, nullptr, s));
    // mask count on the device would need a reduction first; the host counts instead
    std::vector<float> hm((size_t)N * H * W);
    NCK(cudaMemcpyAsync(hm.data(), d_mask, hm.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
    double cnt = 0;
    for (float v : hm) cnt += v;
    const float inv = cnt > 0 ? (float)(1.0 / cnt) : 0.f;
    NCK(cudaMemsetAsync(n->gact, 0, n->act_floats * sizeof(float), s));
    NCK(cudaMemsetAsync(n->d_loss, 0, sizeof(float), s));
    const int HW = H * W;
    float *pred = n->act + n->t_off[kTensors - 1], *gpred = n->gact + n->t_off[kTensors - 1];
    loss_kernel<<<(N * HW + 255) / 256, 256, 0, s>>>(pred, d_label, d_mask, N, HW, inv, gpred, n->d_loss);
    NCK(cudaGetLastError());
    for (int i = kLayers - 1; i >= 0; --i) {
        const LayerSpec &sp = kSpec[i];
        const int lo = kLevel[i + 1];
        const int Ho = n->lh[lo], Wo = n->lw[lo];
        float *g = n->gact + n->t_off[i + 1];
        const float *o = n->act + n->t_off[i + 1];
        const size_t no = (size_t)N * sp.cout * Ho * Wo;
        if (sp.act) {
            act_bwd_kernel<<<(unsigned)((no + 255) / 256), 256, 0, s>>>(g, o, no);
            NCK(cudaGetLastError());
        }
        ConvBwdW bw;
        bw.in = conv_in(n, n->act, i, N);
        bw.N = N;
        bw.Ho = Ho;
        bw.Wo = Wo;
        bw.stride = sp.stride;
        bw.cout = sp.cout;
        bw.g = g;
        bw.dw = n->grads + n->w_off[i];
        bw.db = n->grads + n->b_off[i];
        const int cin = sp.ca + sp.cb;
        if (sp.cout % 8 == 0) conv_bwd_w_kernel<8><<<dim3(cin, sp.cout / 8), 256, 0, s>>>(bw);
        else conv_bwd_w_kernel<2><<<dim3(cin, (sp.cout + 1) / 2), 256, 0, s>>>(bw);
        NCK(cudaGetLastError());
        if (sp.a == 0 && sp.b < 0) continue;  // the cost volume needs no gradient
        ConvBwdData bd;
        bd.N = N;
        bd.cin = cin;
        bd.Hin = bw.in.Hin;
        bd.Win = bw.in.Win;
        bd.Ho = Ho;
        bd.Wo = Wo;
        bd.stride = sp.stride;
        bd.cout = sp.cout;
        bd.w = n->wbf + n->w_off[i];
        bd.g = g;
        bd.din = n->din;
        const int px = bd.Hin * bd.Win;
        conv_bwd_data_kernel<32><<<dim3((px + 127) / 128, (cin + 31) / 32, N), 128, 0, s>>>(bd);
        NCK(cudaGetLastError());
        float *ga = sp.a > 0 ? n->gact + n->t_off[sp.a] : nullptr;
        float *gb = sp.b >= 0 ? n->gact + n->t_off[sp.b] : nullptr;
        const size_t tot = (ga ? (size_t)N * sp.ca * bw.in.Ha * bw.in.Wa : 0) + (gb ? (size_t)N * sp.cb * px : 0);
        split_grad_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n->din, N, sp.ca, sp.cb, sp.up, bd.Hin,
                                                                         bd.Win, bw.in.Ha, bw.in.Wa, ga, gb);
        NCK(cudaGetLastError());
    }
    NCK(cudaMemcpyAsync(n->h_loss, n->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    NCK(cudaStreamSynchronize(s));
    if (loss) *loss = *n->h_loss;
    return PIV_OK;
}

int piv_net_adam_step(piv_net *n, float lr)
{
    if (!n || !(lr >= 0.f)) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    n->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, n->step)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, n->step)));
    adam_kernel<<<(unsigned)((n->n_params + 255) / 256), 256, 0, n->stream>>>(
        n->params, n->grads, n->adam_m, n->adam_v, n->wbf, n->n_params, lr, b1, b2, 1e-8f, c1, c2);
    NCK(cudaGetLastError());
    NCK(refresh_forward_weights(n, n->stream));
    return PIV_OK;
}

int piv_net_synchronize(piv_net *n)
{
    if (!n) return PIV_ERR_ARG;
    cudaSetDevice(n->device);
    NCK(cudaStreamSynchronize(n->stream));
    return net_check_status(n);
}

}  // extern "C"
