/*
 * common.cuh -- shared device helpers for libadmix (sm_100a).
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define ADMIX_KMAX 16

/* Device-side scalars of one handle: the log-likelihood bookkeeping of admixture_qn!
 * (algorithms_outer.jl:98-159) kept on the GPU so an iteration needs no host round trip. */
struct DevScalars {
    double ll_new, ll_prev, ll_basic, ll_qn, reldiff;
    double ll_tmp;                 /* result slot of a stand-alone loglik */
    double qn_cf[8];               /* ZAL: inv(U'(U-V)) U'(x0 - x1); LBQN: the alpha_i of update_QN_LBQN! */
    double qn_gamma;               /* LBQN: gamma_t = u'v / v'v */
    int32_t iter;                  /* iteration number i of the current QN step */
    int32_t accepted;
    int32_t fail_q, fail_p;
    int32_t qn_singular;
    int32_t tc_err;                /* set by a tensor-core kernel whose bounded wait ran out */
    int32_t pad[2];
};

/* 2-bit code -> genotype value (loops.jl:2-5): 00->0, 01->0 (missing), 10->1, 11->2 */
__device__ __forceinline__ double gval(int c) { return c >= 2 ? (double)(c - 1) : 0.0; }

/* Packed upper-triangle index of a K x K symmetric block: t(k, k2) for k <= k2, column
 * major over k2 (t = k2 (k2 + 1) / 2 + k). */
__host__ __device__ __forceinline__ int tri_index(int k, int k2) { return k2 * (k2 + 1) / 2 + k; }

/* inverse map of tri_index on the device */
__device__ __forceinline__ void tri_pair(int t, int &k, int &k2)
{
    int c = 0;
    while ((c + 1) * (c + 2) / 2 <= t) ++c;
    k2 = c;
    k = t - c * (c + 1) / 2;
}

/* Deterministic block sum of one double (blockDim.x a multiple of 32, <= 1024). */
__device__ __forceinline__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int k = 0; k < nw; ++k) s += red[k];
    }
    return s;   /* valid in thread 0 */
}

/* project_q! (projections.jl:27-59) on K values in registers: subtract the pseudocount,
 * sort descending, find the threshold, clamp at zero, add the pseudocount back.  Only the
 * sorted values enter the arithmetic, so any descending sort reproduces the reference. */
template <int K>
__device__ __forceinline__ void project_simplex_local(double (&b)[K])
{
    const double pc = 1e-5;
    const double tau = 1.0 - __dmul_rn((double)K, pc);
    double s[K];
#pragma unroll
    for (int i = 0; i < K; ++i) b[i] -= pc;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const double v = b[i];
        int k = i;
        while (k > 0 && s[k - 1] < v) { s[k] = s[k - 1]; --k; }
        s[k] = v;
    }
    double tsum = 0.0, tmax = 0.0;
    bool bget = false;
    for (int i = 0; i < K - 1; ++i) {
        tsum += s[i];
        tmax = (tsum - tau) / (double)(i + 1);
        if (tmax >= s[i + 1]) { bget = true; break; }
    }
    if (!bget) tmax = (tsum + s[K - 1] - tau) / (double)K;
#pragma unroll
    for (int i = 0; i < K; ++i) b[i] = fmax(b[i] - tmax, 0.0) + pc;
}

/* sub-split of the per-problem accumulator list over NS threads, chosen by K so the
 * FP64 accumulators of one thread stay in registers. */
__host__ __device__ constexpr int ns_for_k(int K) { return K <= 8 ? 1 : (K <= 12 ? 2 : 4); }

#define ADMIX_DISPATCH_K(KV, CALL)                                              \
    switch (KV) {                                                               \
    case 1: { constexpr int KK = 1; CALL; } break;                              \
    case 2: { constexpr int KK = 2; CALL; } break;                              \
    case 3: { constexpr int KK = 3; CALL; } break;                              \
    case 4: { constexpr int KK = 4; CALL; } break;                              \
    case 5: { constexpr int KK = 5; CALL; } break;                              \
    case 6: { constexpr int KK = 6; CALL; } break;                              \
    case 7: { constexpr int KK = 7; CALL; } break;                              \
    case 8: { constexpr int KK = 8; CALL; } break;                              \
    case 9: { constexpr int KK = 9; CALL; } break;                              \
    case 10: { constexpr int KK = 10; CALL; } break;                            \
    case 11: { constexpr int KK = 11; CALL; } break;                            \
    case 12: { constexpr int KK = 12; CALL; } break;                            \
    case 13: { constexpr int KK = 13; CALL; } break;                            \
    case 14: { constexpr int KK = 14; CALL; } break;                            \
    case 15: { constexpr int KK = 15; CALL; } break;                            \
    case 16: { constexpr int KK = 16; CALL; } break;                            \
    default: break;                                                             \
    }
