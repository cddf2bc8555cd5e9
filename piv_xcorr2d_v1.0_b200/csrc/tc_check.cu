// tc_check.cu -- piv_tc_gemm_check: one 128 x N x K product on the tcgen05 path with
// either operand in either shared-memory layout, checked by the tests against a host
// product.  It exercises exactly the descriptor, instruction-descriptor, TMEM and
// split-BF16 code the tensor-core correlation kernel is built from.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "piv_b200.h"
#include "tc_common.cuh"

namespace piv {

namespace {

constexpr int kM = 128;
constexpr int kGuard = 64 * 1024;  // slack after the operands

__global__ void __launch_bounds__(128) tc_gemm_check_kernel(const float *A, const float *B, float *D, int N,
                                                            int K, int a_mn, int b_mn, int nprod, int *status)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x;
    uint8_t *a_hi = smem, *a_lo = a_hi + kM * K * 2;
    uint8_t *b_hi = a_lo + kM * K * 2, *b_lo = b_hi + N * K * 2;

    // operands -> bf16 hi/lo in the requested layouts
    for (int t = tid; t < kM * K; t += blockDim.x) {
        const int m = t / K, k = t - m * K;
        uint16_t h, l;
        tc::split_bf16(A[t], h, l);
        const uint32_t o = a_mn ? tc::off_mnmajor(m, k, K) : tc::off_kmajor(m, k, kM);
        *reinterpret_cast<uint16_t *>(a_hi + o) = h;
        *reinterpret_cast<uint16_t *>(a_lo + o) = l;
    }
    for (int t = tid; t < N * K; t += blockDim.x) {
        const int n = t / K, k = t - n * K;
        uint16_t h, l;
        tc::split_bf16(B[t], h, l);
        const uint32_t o = b_mn ? tc::off_mnmajor(n, k, K) : tc::off_kmajor(n, k, N);
        *reinterpret_cast<uint16_t *>(b_hi + o) = h;
        *reinterpret_cast<uint16_t *>(b_lo + o) = l;
    }
    const uint32_t mb = tc::smem_u32(&mbar);
    if (tid == 0) tc::mbar_init(mb, 1);
    if (tid < 32) tc::tmem_alloc(tc::smem_u32(&tmem_base), 128);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;

    if (tid == 0) {
        const uint32_t idesc = tc::idesc_f16(N, a_mn != 0, b_mn != 0, true);
        // per K step (16): K-major advances two 8-element chunks (2 * LBO), MN-major
        // advances 16 K rows of 16 bytes
        const uint32_t a_lbo = a_mn ? 128u : kM * 16u, a_sbo = a_mn ? (uint32_t)K * 16u : 128u;
        const uint32_t b_lbo = b_mn ? 128u : (uint32_t)N * 16u, b_sbo = b_mn ? (uint32_t)K * 16u : 128u;
        const uint32_t a_step = a_mn ? 256u : 2u * a_lbo, b_step = b_mn ? 256u : 2u * b_lbo;
        uint32_t acc = 0;
        for (int s = 0; s < K / 16; ++s) {
            const uint32_t ah = tc::smem_u32(a_hi) + s * a_step, al = tc::smem_u32(a_lo) + s * a_step;
            const uint32_t bh = tc::smem_u32(b_hi) + s * b_step, bl = tc::smem_u32(b_lo) + s * b_step;
            tc::mma_f16(tmem, tc::smem_desc(ah, a_lbo, a_sbo), tc::smem_desc(bh, b_lbo, b_sbo), idesc, acc);
            acc = 1;
            if (nprod >= 3) {
                tc::mma_f16(tmem, tc::smem_desc(ah, a_lbo, a_sbo), tc::smem_desc(bl, b_lbo, b_sbo), idesc, 1);
                tc::mma_f16(tmem, tc::smem_desc(al, a_lbo, a_sbo), tc::smem_desc(bh, b_lbo, b_sbo), idesc, 1);
            }
        }
        tc::mma_commit(mb);
    }
    const bool ok = tc::mbar_wait(mb, 0);
    tc::fence_after_sync();
    if (!ok) {
        if (tid == 0) atomicOr(status, 1);
    } else {
        const uint32_t lane_base = (uint32_t)(tid & ~31) << 16;
        for (int c = 0; c < N; c += 16) {
            float v[16];
            tc::tmem_ld16(tmem + lane_base + c, v);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) D[tid * N + c + i] = v[i];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid < 32) tc::tmem_dealloc(tmem, 128);
}

}  // namespace

}  // namespace piv

extern "C" int piv_tc_gemm_check(const float *A, const float *B, float *D, int N, int K, int a_mn, int b_mn,
                                 int nprod)
{
    using namespace piv;
    if (!A || !B || !D || N < 16 || N > 128 || N % 16 || K < 16 || K > 128 || K % 16 || (nprod != 1 && nprod != 3))
        return PIV_ERR_ARG;
    int dev = 0, cc = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&cc, cudaDevAttrComputeCapabilityMajor, dev) !=
                                                  cudaSuccess)
        return PIV_ERR_CUDA;
    if (cc != 10) return PIV_ERR_UNSUPPORTED;
    float *dA = nullptr, *dB = nullptr, *dD = nullptr;
    int *dS = nullptr;
    int rc = PIV_OK;
    const size_t smem = (size_t)2 * kM * K * 2 + (size_t)2 * N * K * 2 + kGuard;
    do {
        if (cudaMalloc(&dA, sizeof(float) * kM * K) || cudaMalloc(&dB, sizeof(float) * N * K) ||
            cudaMalloc(&dD, sizeof(float) * kM * N) || cudaMalloc(&dS, sizeof(int))) {
            rc = PIV_ERR_CUDA;
            break;
        }
        cudaMemcpy(dA, A, sizeof(float) * kM * K, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, B, sizeof(float) * N * K, cudaMemcpyHostToDevice);
        cudaMemset(dS, 0, sizeof(int));
        if (cudaFuncSetAttribute(tc_gemm_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) {
            rc = PIV_ERR_CUDA;
            break;
        }
        tc_gemm_check_kernel<<<1, 128, smem>>>(dA, dB, dD, N, K, a_mn, b_mn, nprod, dS);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
            rc = PIV_ERR_CUDA;
            break;
        }
        int st = 0;
        cudaMemcpy(&st, dS, sizeof(int), cudaMemcpyDeviceToHost);
        if (st) {
            fprintf(stderr, "piv_tc_gemm_check: MMA completion wait timed out\n");
            rc = PIV_ERR_DEVICE;
            break;
        }
        cudaMemcpy(D, dD, sizeof(float) * kM * N, cudaMemcpyDeviceToHost);
    } while (0);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dS);
    return rc;
}
