/*
 * tc_probe.cu -- diagnostic: one tcgen05 BF16 MMA chain on caller data, to test the tensor-core
 * arithmetic the mixed form is designed around.
 *
 * D[128 x 16] = sum over K-steps s < nsteps of A[:, 16s:16s+16] * B[:, 16s:16s+16]^T, BF16 A and
 * B, FP32 accumulator in TMEM (the first step starts the sum, the others accumulate).  B is read
 * from shared memory (K-major, no swizzle, as the sweeps lay it out); A from shared memory, or,
 * with a_in_tmem, from TMEM written by tcgen05.st (two BF16 per 32-bit column, the even element
 * in the low half, 8 columns per K-step).  What the mixed form relies on, and the GPU test checks:
 * BF16 products are exact; the FP32 sums truncate toward zero (so a long sum in TMEM drifts low,
 * hence the per-chunk diagonal and the block drains); both A sources give the same result.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/admix.h"
#include "tc05.cuh"

namespace {

constexpr int TP_KMAX = 64;                            /* 4 K-steps */
constexpr uint32_t TP_A_LBO = 2048, TP_B_LBO = 256, TP_SBO = 128;

__device__ __forceinline__ uint32_t tp_off(int r, int k, uint32_t lbo)
{
    return (uint32_t)(k >> 3) * lbo + (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

__device__ __forceinline__ void tc_mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n"
                 :: "r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&v)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
                 :: "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
                    "r"(v[7]) : "memory");
}

/* one CTA of 128 threads: thread = row of A and D = TMEM lane */
__global__ void __launch_bounds__(128)
k_tc_probe(const uint16_t *__restrict__ A, const uint16_t *__restrict__ B, float *__restrict__ D, int nsteps,
           int a_in_tmem, int *__restrict__ err)
{
    __shared__ __align__(1024) uint8_t sa[128 * TP_KMAX * 2];
    __shared__ __align__(1024) uint8_t sb[16 * TP_KMAX * 2];
    __shared__ uint64_t bar;
    __shared__ uint32_t holder;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int k = 0; k < TP_KMAX; ++k) *(uint16_t *)(sa + tp_off(tid, k, TP_A_LBO)) = A[tid * TP_KMAX + k];
    if (tid < 16)
        for (int k = 0; k < TP_KMAX; ++k) *(uint16_t *)(sb + tp_off(tid, k, TP_B_LBO)) = B[tid * TP_KMAX + k];
    if (warp == 0) tmem_alloc_warp(&holder, 64);       /* D: columns 0-15, A: columns 32-63 */
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    fence_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = holder, lane = (uint32_t)(warp * 32) << 16;
    if (a_in_tmem) {
        for (int s = 0; s < TP_KMAX / 16; ++s) {
            uint32_t v[8];
            for (int c = 0; c < 8; ++c)
                v[c] = (uint32_t)A[tid * TP_KMAX + 16 * s + 2 * c] | ((uint32_t)A[tid * TP_KMAX + 16 * s + 2 * c + 1] << 16);
            tmem_st8(tmem + lane + 32u + 8u * (uint32_t)s, v);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    if (tid == 0) {
        constexpr uint32_t id = idesc_bf16_f32(128, 16);
        for (int s = 0; s < nsteps; ++s) {
            const uint64_t bd = umma_desc_kmajor(smem_u32(sb) + (uint32_t)s * 2 * TP_B_LBO, TP_B_LBO, TP_SBO);
            if (a_in_tmem)
                tc_mma_bf16_ts(tmem, tmem + 32u + 8u * (uint32_t)s, bd, id, s > 0 ? 1u : 0u);
            else
                tc_mma_bf16(tmem, umma_desc_kmajor(smem_u32(sa) + (uint32_t)s * 2 * TP_A_LBO, TP_A_LBO, TP_SBO), bd, id,
                            s > 0 ? 1u : 0u);
        }
        tc_commit(&bar);
    }
    __syncwarp();
    const bool ok = mbar_wait_bounded(&bar, 0u, 1u << 22);
    if (!ok) atomicOr(err, 1);
    tc_fence_after_sync();
    float v[16];
    tmem_ld16(tmem + lane, v);
    for (int n = 0; n < 16; ++n) D[tid * 16 + n] = ok ? v[n] : __int_as_float(0x7fc00000);
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc_warp(tmem, 64);
}

}  // namespace

extern "C" int admix_tc_probe(const uint16_t *a, const uint16_t *b, float *d, int32_t nsteps, int32_t a_in_tmem)
{
    if (!a || !b || !d || nsteps < 1 || nsteps > TP_KMAX / 16 || (a_in_tmem != 0 && a_in_tmem != 1)) return ADMIX_ERR_ARG;
    uint16_t *dA = nullptr, *dB = nullptr;
    float *dD = nullptr;
    int *dErr = nullptr, hErr = 0;
    cudaError_t e = cudaMalloc(&dA, 128 * TP_KMAX * 2);
    if (e == cudaSuccess) e = cudaMalloc(&dB, 16 * TP_KMAX * 2);
    if (e == cudaSuccess) e = cudaMalloc(&dD, 128 * 16 * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dErr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(dA, a, 128 * TP_KMAX * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dB, b, 16 * TP_KMAX * 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dErr, 0, sizeof(int));
    if (e == cudaSuccess) {
        k_tc_probe<<<1, 128>>>(dA, dB, dD, nsteps, a_in_tmem, dErr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(d, dD, 128 * 16 * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&hErr, dErr, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dErr);
    return (e != cudaSuccess || hErr) ? ADMIX_ERR_CUDA : ADMIX_OK;
}
