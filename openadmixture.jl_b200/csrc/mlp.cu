/*
 * mlp.cu -- the learned warm start: genotype sketch, a small MLP encoder (forward, backward,
 * Adam) and the closed-form P step that turns a predicted Q into a starting P.
 *
 * This part has no counterpart in the reference.  Its hook is run_admixture's init_q / init_p
 * (driver.jl:52-53,161-166,183-188): the predicted Q and the derived P replace the random start
 * and the EM priming.
 *
 * Features of individual i: the dosages of S fixed sketch SNPs (int8; 3 = missing) and R
 * projections of the frequency-standardised dosages onto fixed +-1 directions,
 *   proj_ir = S^-1/2 sum_s (d_is - 2 f_s) / sqrt(2 f_s (1 - f_s)) * sign_rs     (missing -> 0).
 * Network: x = [d - 2f | proj] (S + R) -> ReLU(W1 x + b1) (H) -> ReLU(W2 . + b2) (H) ->
 * softmax(W3 . + b3) (K).  Loss: cross-entropy against soft targets (aligned converged Q).
 * All matrices are row-major FP32 (W1: (S+R) x H, W2: H x H, W3: H x K).
 *
 * Every product of the forward and backward passes is one tensor-core GEMM (k_gemm_tc): a CTA
 * owns a 128 x 64 tile of the output in TMEM; each 32-deep slice of the reduction is loaded by
 * the CTA's threads through an operand functor (dense, transposed, or the network input built
 * on the fly from the dosages), split into BF16 high and low parts, and multiplied as
 * hi*hi + lo*hi + hi*lo by tcgen05 (about 2^-17 relative per product, FP32 accumulation).  The
 * accumulator restarts every 128 of the reduction and the threads add it into FP32 registers,
 * so no FP32 partial sees more than 24 of the tensor core's accumulations.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include "../../include/admix.h"
#include "common.cuh"
#include "synth.h"
#include "tc05.cuh"

namespace {

__device__ __forceinline__ int code_of(const uint8_t *bed, int64_t pitch, int64_t i, int64_t j)
{
    return (bed[(size_t)j * pitch + (i >> 2)] >> ((i & 3) << 1)) & 3;
}

/* 2-bit code -> dosage: 00 -> 0, 10 -> 1, 11 -> 2, 01 (missing) -> 3 */
__device__ __forceinline__ int8_t dosage_of(int c) { return c == 1 ? (int8_t)3 : (int8_t)(c == 0 ? 0 : c - 1); }

/* allele frequency of each sketch SNP: one block per SNP */
__global__ void k_sketch_freq(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I,
                              const int32_t *__restrict__ snps, float *__restrict__ freq)
{
    __shared__ double red[8];
    const int64_t j = snps[blockIdx.x];
    double a = 0.0, n = 0.0;
    for (int64_t i = threadIdx.x; i < I; i += blockDim.x) {
        const int c = code_of(bed, pitch, i, j);
        if (c != 1) { a += (c == 0) ? 0.0 : (double)(c - 1); n += 2.0; }
    }
    const double sa = block_sum(a, red);
    const double sn = block_sum(n, red);
    if (threadIdx.x == 0) freq[blockIdx.x] = sn > 0.0 ? (float)(sa / sn) : 0.5f;
}

/* dosage sketch (I x S int8) and the R standardised projections (I x R) */
__global__ void k_sketch(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I, const int32_t *__restrict__ snps,
                         int S, const float *__restrict__ freq, int R, uint64_t seed, int8_t *__restrict__ dos,
                         float *__restrict__ proj)
{
    extern __shared__ float sh[];                     /* [R] partial projections per warp */
    const int64_t i = blockIdx.x;
    float acc[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) acc[r] = 0.f;
    for (int s = threadIdx.x; s < S; s += blockDim.x) {
        const int c = code_of(bed, pitch, i, snps[s]);
        const int8_t d = dosage_of(c);
        dos[(size_t)i * S + s] = d;
        if (d != 3) {
            const float f = freq[s];
            const float z = ((float)d - 2.f * f) * rsqrtf(fmaxf(2.f * f * (1.f - f), 1e-6f));
            const uint64_t h = syn_hash3(seed, (uint64_t)s, 0);
#pragma unroll
            for (int r = 0; r < 32; ++r)
                if (r < R) acc[r] += ((h >> r) & 1u) ? z : -z;
        }
    }
    const float scale = rsqrtf((float)S);
    for (int r = 0; r < R; ++r) {
        float v = acc[r];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sh[(threadIdx.x >> 5) * R + r] = v;
    }
    __syncthreads();
    if (threadIdx.x < R) {
        float v = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sh[w * R + threadIdx.x];
        proj[(size_t)i * R + threadIdx.x] = v * scale;
    }
}

} // namespace

extern "C" int admix_sketch(const uint8_t *d_bed, int64_t pitch, int64_t I, const int32_t *d_snps, int32_t S,
                            int32_t R, uint64_t seed, float *d_freq, int8_t *d_dos, float *d_proj, void *stream)
{
    if (!d_bed || !d_snps || !d_freq || !d_dos || !d_proj || I < 1 || S < 1 || R < 0 || R > 32 || pitch < (I + 3) / 4)
        return ADMIX_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    k_sketch_freq<<<S, 256, 0, st>>>(d_bed, pitch, I, d_snps, d_freq);
    k_sketch<<<(unsigned)I, 256, sizeof(float) * 8 * (R > 0 ? R : 1), st>>>(d_bed, pitch, I, d_snps, S, d_freq, R,
                                                                            seed, d_dos, d_proj);
    return cudaGetLastError() == cudaSuccess ? ADMIX_OK : ADMIX_ERR_CUDA;
}

namespace {

/* ---- operand loaders: element (r, c) of a logical row-major matrix ---- */
struct LoadF {                     /* dense FP32 with arbitrary strides (transposes are strides) */
    const float *p; int64_t sr, sc;
    __device__ float operator()(int64_t r, int64_t c) const { return p[r * sr + c * sc]; }
};
struct LoadX {                     /* network input: [dosage - 2f (0 if missing) | projections] */
    const int8_t *dos; const float *center; const float *proj; int S, R;
    __device__ float operator()(int64_t m, int64_t k) const
    {
        if (k < S) {
            const int8_t d = dos[m * S + k];
            return d == 3 ? 0.f : (float)d - center[k];
        }
        return proj[m * R + (k - S)];
    }
};
struct LoadXT {                    /* the input transposed: (k, m) */
    LoadX x;
    __device__ float operator()(int64_t k, int64_t m) const { return x(m, k); }
};

constexpr int GT_M = 128, GT_N = 64, GT_K = 32;   /* output tile rows x columns, reduction slice */
constexpr int GT_D = 4;                             /* slices per fresh accumulation */
constexpr uint32_t GT_WAIT = 1u << 22;              /* polls of a bounded wait */
/* one stage: A hi, A lo (128 x 32 BF16, K-major core matrices), B hi, B lo (64 x 32) */
constexpr uint32_t GT_A = GT_M * GT_K * 2, GT_B = GT_N * GT_K * 2;
constexpr uint32_t GT_STAGE = 2 * GT_A + 2 * GT_B;
constexpr uint32_t GT_SMEM = 2 * GT_STAGE + 1024;
constexpr uint32_t GT_A_LBO = GT_M * 16, GT_B_LBO = GT_N * 16;

/* v = hi + lo, both BF16 (hi rounded to nearest, lo the BF16 of the remainder) */
__device__ __forceinline__ void split_bf16(float v, uint32_t &hi, uint32_t &lo)
{
    hi = pack_bf16x2(v, 0.f) & 0xFFFFu;
    lo = pack_bf16x2(v - __uint_as_float(hi << 16), 0.f) & 0xFFFFu;
}

/* C[m, n] = alpha * sum_k A(m, k) B(k, n) (+ bias[n]); relu if act; times [mask(m, n) > 0] if mask.
 * 128 threads, one 128 x 64 output tile per CTA (thread = output row = TMEM lane).  Two smem
 * stages: the threads load slice c+1 while the tensor core multiplies slice c.  Every wait is
 * bounded; a CTA whose wait runs out writes NaN into its tile (the failure shows in the loss). */
template <class LA, class LB>
__global__ void __launch_bounds__(128)
k_gemm_tc(LA A, LB B, int64_t M, int64_t N, int64_t Kd, float alpha, const float *__restrict__ bias, int act,
          const float *__restrict__ mask, float *__restrict__ C, int64_t ldc)
{
    extern __shared__ __align__(1024) uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    __shared__ uint64_t bar[2];          /* MMAs of the slice in stage s done */
    __shared__ uint32_t tmem_holder;
    __shared__ volatile int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int64_t m0 = (int64_t)blockIdx.y * GT_M, n0 = (int64_t)blockIdx.x * GT_N;
    if (warp == 0) tmem_alloc_warp(&tmem_holder, GT_N);
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        abort_flag = 0;
        mbar_fence_init();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_holder;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    bool ok = true;
    auto wait = [&](uint64_t *b, uint32_t parity) {
        if (!ok) return;
        for (uint32_t n = 0; n < GT_WAIT; ++n) {
            if (mbar_try_wait(b, parity)) return;
            if ((n & 255u) == 255u && abort_flag) break;
        }
        ok = false;
        abort_flag = 1;
    };
    float acc[GT_N];
#pragma unroll
    for (int n = 0; n < GT_N; ++n) acc[n] = 0.f;
    auto drain = [&]() {   /* the finished accumulation block into the FP32 registers */
        tc_fence_after_sync();
#pragma unroll
        for (int c0 = 0; c0 < GT_N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + lane_base + (uint32_t)c0, v);
#pragma unroll
            for (int e = 0; e < 16; ++e) acc[c0 + e] += v[e];
        }
    };
    const int nch = (int)((Kd + GT_K - 1) / GT_K);
    constexpr uint32_t idesc = idesc_bf16_f32(GT_M, GT_N);
    for (int c = 0; c < nch; ++c) {
        const int st = c & 1;
        uint8_t *Ah = sm + st * GT_STAGE, *Al = Ah + GT_A, *Bh = Al + GT_A, *Bl = Bh + GT_B;
        if (c >= 2) wait(&bar[st], (uint32_t)(((c - 2) >> 1) & 1));   /* stage st is free again */
        const int64_t k0 = (int64_t)c * GT_K;
        /* A: thread t loads row m0 + t of the slice, 4 granules of 8 */
        {
            const int64_t m = m0 + tid;
#pragma unroll
            for (int gr = 0; gr < GT_K / 8; ++gr) {
                uint32_t h[4], l[4];
#pragma unroll
                for (int e = 0; e < 8; e += 2) {
                    const int64_t ka = k0 + 8 * gr + e;
                    const float v0 = (m < M && ka < Kd) ? A(m, ka) : 0.f;
                    const float v1 = (m < M && ka + 1 < Kd) ? A(m, ka + 1) : 0.f;
                    uint32_t h0, l0, h1, l1;
                    split_bf16(v0, h0, l0);
                    split_bf16(v1, h1, l1);
                    h[e / 2] = h0 | (h1 << 16);
                    l[e / 2] = l0 | (l1 << 16);
                }
                *(uint4 *)(Ah + gr * GT_A_LBO + 16 * tid) = make_uint4(h[0], h[1], h[2], h[3]);
                *(uint4 *)(Al + gr * GT_A_LBO + 16 * tid) = make_uint4(l[0], l[1], l[2], l[3]);
            }
        }
        /* B: 64 columns x 4 granules = 256 tasks, two per thread; B row n holds B(k, n0 + n) */
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int task = tid + 128 * u;
            const int n = task & (GT_N - 1), gr = task >> 6;
            const int64_t col = n0 + n;
            uint32_t h[4], l[4];
#pragma unroll
            for (int e = 0; e < 8; e += 2) {
                const int64_t ka = k0 + 8 * gr + e;
                const float v0 = (col < N && ka < Kd) ? B(ka, col) : 0.f;
                const float v1 = (col < N && ka + 1 < Kd) ? B(ka + 1, col) : 0.f;
                uint32_t h0, l0, h1, l1;
                split_bf16(v0, h0, l0);
                split_bf16(v1, h1, l1);
                h[e / 2] = h0 | (h1 << 16);
                l[e / 2] = l0 | (l1 << 16);
            }
            *(uint4 *)(Bh + gr * GT_B_LBO + 16 * n) = make_uint4(h[0], h[1], h[2], h[3]);
            *(uint4 *)(Bl + gr * GT_B_LBO + 16 * n) = make_uint4(l[0], l[1], l[2], l[3]);
        }
        fence_async_smem();
        if (c > 0 && c % GT_D == 0) {   /* the block ending at slice c-1: its MMAs done, into registers */
            wait(&bar[(c - 1) & 1], (uint32_t)(((c - 1) >> 1) & 1));
            if (ok) drain();
        }
        tc_fence_before_sync();
        __syncthreads();
        tc_fence_after_sync();
        if (tid == 0 && ok) {
            const uint32_t ah = smem_u32(Ah), al = smem_u32(Al), bh = smem_u32(Bh), bl = smem_u32(Bl);
#pragma unroll
            for (int ks = 0; ks < GT_K / 16; ++ks) {
                const uint32_t ao = ks * 2 * GT_A_LBO, bo = ks * 2 * GT_B_LBO;
                const uint32_t fresh = (c % GT_D == 0 && ks == 0) ? 0u : 1u;
                tc_mma_bf16(tmem, umma_desc_kmajor(ah + ao, GT_A_LBO, 128), umma_desc_kmajor(bh + bo, GT_B_LBO, 128),
                            idesc, fresh);
                tc_mma_bf16(tmem, umma_desc_kmajor(al + ao, GT_A_LBO, 128), umma_desc_kmajor(bh + bo, GT_B_LBO, 128),
                            idesc, 1u);
                tc_mma_bf16(tmem, umma_desc_kmajor(ah + ao, GT_A_LBO, 128), umma_desc_kmajor(bl + bo, GT_B_LBO, 128),
                            idesc, 1u);
            }
            tc_commit(&bar[st]);
        }
    }
    if (nch > 0) {   /* the last block */
        wait(&bar[(nch - 1) & 1], (uint32_t)(((nch - 1) >> 1) & 1));
        if (ok) drain();
    }
    ok = __syncthreads_and(ok);
    if (!ok && tid == 0) {   /* give MMAs still in flight a bounded moment before the TMEM goes */
        mbar_wait_bounded(&bar[0], 0u, 1024u); mbar_wait_bounded(&bar[0], 1u, 1024u);
        mbar_wait_bounded(&bar[1], 0u, 1024u); mbar_wait_bounded(&bar[1], 1u, 1024u);
    }
    const int64_t m = m0 + tid;
    if (m < M) {
#pragma unroll
        for (int n = 0; n < GT_N; ++n) {
            const int64_t col = n0 + n;
            if (col >= N) break;
            float v = alpha * acc[n] + (bias ? bias[col] : 0.f);
            if (act) v = fmaxf(v, 0.f);
            if (mask && !(mask[m * ldc + col] > 0.f)) v = 0.f;
            C[m * ldc + col] = ok ? v : __int_as_float(0x7fc00000);
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc_warp(tmem, GT_N);
}

template <class LA, class LB>
cudaError_t gemm(LA A, LB B, int64_t M, int64_t N, int64_t Kd, float alpha, const float *bias, int act,
                 const float *mask, float *C, int64_t ldc, cudaStream_t st)
{
    static bool ready = false;   /* the kernel's dynamic shared memory limit, set once per instantiation */
    if (!ready) {
        cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<LA, LB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GT_SMEM);
        if (e != cudaSuccess) return e;
        ready = true;
    }
    dim3 grid((unsigned)((N + GT_N - 1) / GT_N), (unsigned)((M + GT_M - 1) / GT_M));
    k_gemm_tc<LA, LB><<<grid, 128, GT_SMEM, st>>>(A, B, M, N, Kd, alpha, bias, act, mask, C, ldc);
    return cudaGetLastError();
}

/* row softmax of logits (n x K) into probs; with targets: dlogits = (probs - target) / n and the
 * summed cross-entropy added (atomically) into *loss */
__global__ void k_softmax_ce(const float *__restrict__ logits, int64_t n, int K, float *__restrict__ probs,
                             const float *__restrict__ target, float *__restrict__ dlogits, float *__restrict__ loss)
{
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const float *z = logits + m * K;
    float mx = z[0];
    for (int k = 1; k < K; ++k) mx = fmaxf(mx, z[k]);
    float s = 0.f;
    for (int k = 0; k < K; ++k) s += expf(z[k] - mx);
    const float ls = logf(s);
    float l = 0.f;
    for (int k = 0; k < K; ++k) {
        const float pk = expf(z[k] - mx - ls);
        probs[m * K + k] = pk;
        if (target) {
            dlogits[m * K + k] = (pk - target[m * K + k]) / (float)n;
            l -= target[m * K + k] * (z[k] - mx - ls);
        }
    }
    if (target && loss) atomicAdd(loss, l);
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, int64_t n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const float gt = g[t];
        const float a = b1 * m1[t] + (1.f - b1) * gt, b = b2 * m2[t] + (1.f - b2) * gt * gt;
        m1[t] = a; m2[t] = b;
        w[t] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    }
}

} // namespace

namespace {

__global__ void k_colsum_atomic(const float *__restrict__ dY, int64_t M, int64_t N, float *__restrict__ db)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int64_t rows = (M + gridDim.y - 1) / gridDim.y;
    const int64_t m0 = (int64_t)blockIdx.y * rows, m1 = min(M, m0 + rows);
    float s = 0.f;
    for (int64_t m = m0; m < m1; ++m) s += dY[m * N + n];
    atomicAdd(db + n, s);
}

cudaError_t colsum(const float *dY, int64_t M, int64_t N, float *db, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(db, 0, sizeof(float) * N, st);
    if (e != cudaSuccess) return e;
    const unsigned gy = (unsigned)std::min<int64_t>(64, std::max<int64_t>(1, M / 256));
    k_colsum_atomic<<<dim3((unsigned)((N + 127) / 128), gy), 128, 0, st>>>(dY, M, N, db);
    return cudaGetLastError();
}

/* closed-form P step from Q: p_kj = sum_i nm q_ki g_ij / (2 sum_i nm q_ki), clamped to
 * [1e-5, 1-1e-5] like project_p! (projections.jl:69-74).  Thread = SNP; q staged through shared
 * memory 64 individuals at a time as (k, k+1) pairs, both sums accumulated in FP32 pairs (one
 * paired FMA per k pair and cell); a missing cell adds zeros, so no thread branches on the
 * genotype, and one byte load serves four cells.  Each sum is the same per-k FP32 sequence as
 * a per-cell loop that skips the missing cells. */
template <int K>
__global__ void __launch_bounds__(128)
k_warm_p(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I, int64_t J, const double *__restrict__ q,
         double *__restrict__ p)
{
    constexpr int KH = (K + 1) / 2;                  /* k pairs (odd K: the last pair's second half is 0) */
    __shared__ __align__(16) float2 qs[64 * KH];
    const int64_t j = (int64_t)blockIdx.x * 128 + threadIdx.x;
    const uint8_t *col = bed + (size_t)(j < J ? j : 0) * pitch;
    float2 num[KH], den[KH];   /* sum_i q_ki g_ij and sum_i nm q_ki */
#pragma unroll
    for (int kh = 0; kh < KH; ++kh) num[kh] = den[kh] = make_float2(0.f, 0.f);
    for (int64_t i0 = 0; i0 < I; i0 += 64) {
        const int n = (int)min((int64_t)64, I - i0);
        __syncthreads();
        for (int t = threadIdx.x; t < 64 * KH; t += 128) {
            const int ii = t / KH, k = 2 * (t - ii * KH);
            float a = 0.f, b = 0.f;
            if (ii < n) {
                a = (float)q[(size_t)K * (i0 + ii) + k];
                if (k + 1 < K) b = (float)q[(size_t)K * (i0 + ii) + k + 1];
            }
            qs[t] = make_float2(a, b);
        }
        __syncthreads();
        if (j < J) {
            for (int ib = 0; 4 * ib < n; ++ib) {
                const uint32_t byte = col[(size_t)(i0 >> 2) + ib];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int ii = 4 * ib + t;
                    if (ii >= n) break;
                    const uint32_t c = (byte >> (2 * t)) & 3u;
                    const float g = c == 3u ? 2.f : (c == 2u ? 1.f : 0.f);   /* codes 00 -> 0, 10 -> 1, 11 -> 2 */
                    const float nm = c == 1u ? 0.f : 1.f;                    /* 01: missing */
                    const float2 g2 = make_float2(g, g), n2 = make_float2(nm, nm);
#pragma unroll
                    for (int kh = 0; kh < KH; ++kh) {
                        const float2 qv = qs[ii * KH + kh];
                        num[kh] = __ffma2_rn(qv, g2, num[kh]);
                        den[kh] = __ffma2_rn(qv, n2, den[kh]);
                    }
                }
            }
        }
    }
    if (j < J)
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const float nk = (k & 1) ? num[k >> 1].y : num[k >> 1].x;
            const float dk = 2.f * ((k & 1) ? den[k >> 1].y : den[k >> 1].x);
            const double v = dk > 0.f ? (double)nk / (double)dk : 0.5;
            p[(size_t)K * j + k] = fmin(fmax(v, 1e-5), 1.0 - 1e-5);
        }
}

} // namespace

extern "C" {

int admix_mlp_forward(const admix_mlp *net, int64_t n, const int8_t *dos, const float *center, const float *proj,
                      float *h1, float *h2, float *logits, float *probs, void *stream)
{
    if (!net || n < 1 || !dos || !center || !proj || !h1 || !h2 || !logits || !probs) return ADMIX_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t D = net->S + net->R, H = net->H, K = net->K;
    cudaError_t e = gemm(LoadX{dos, center, proj, net->S, net->R}, LoadF{net->w1, H, 1}, n, H, D, 1.f, net->b1, 1,
                         nullptr, h1, H, st);
    if (e == cudaSuccess) e = gemm(LoadF{h1, H, 1}, LoadF{net->w2, H, 1}, n, H, H, 1.f, net->b2, 1, nullptr, h2, H, st);
    if (e == cudaSuccess) e = gemm(LoadF{h2, H, 1}, LoadF{net->w3, K, 1}, n, K, H, 1.f, net->b3, 0, nullptr, logits, K, st);
    if (e == cudaSuccess) {
        k_softmax_ce<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(logits, n, (int)K, probs, nullptr, nullptr, nullptr);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? ADMIX_OK : ADMIX_ERR_CUDA;
}

int admix_mlp_backward(const admix_mlp *net, const admix_mlp_grads *grad, int64_t n, const int8_t *dos,
                       const float *center, const float *proj, const float *h1, const float *h2, const float *logits,
                       const float *target, float *probs, float *dlogits, float *dh2, float *dh1, float *loss,
                       void *stream)
{
    if (!net || !grad || n < 1 || !target || !dlogits || !dh2 || !dh1) return ADMIX_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t D = net->S + net->R, H = net->H, K = net->K;
    k_softmax_ce<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(logits, n, (int)K, probs, target, dlogits, loss);
    cudaError_t e = cudaGetLastError();
    /* layer 3 */
    if (e == cudaSuccess) e = gemm(LoadF{h2, 1, H}, LoadF{dlogits, K, 1}, H, K, n, 1.f, nullptr, 0, nullptr, grad->w3, K, st);
    if (e == cudaSuccess) e = colsum(dlogits, n, K, grad->b3, st);
    if (e == cudaSuccess) e = gemm(LoadF{dlogits, K, 1}, LoadF{net->w3, 1, K}, n, H, K, 1.f, nullptr, 0, h2, dh2, H, st);
    /* layer 2 */
    if (e == cudaSuccess) e = gemm(LoadF{h1, 1, H}, LoadF{dh2, H, 1}, H, H, n, 1.f, nullptr, 0, nullptr, grad->w2, H, st);
    if (e == cudaSuccess) e = colsum(dh2, n, H, grad->b2, st);
    if (e == cudaSuccess) e = gemm(LoadF{dh2, H, 1}, LoadF{net->w2, 1, H}, n, H, H, 1.f, nullptr, 0, h1, dh1, H, st);
    /* layer 1 */
    if (e == cudaSuccess)
        e = gemm(LoadXT{LoadX{dos, center, proj, net->S, net->R}}, LoadF{dh1, H, 1}, D, H, n, 1.f, nullptr, 0, nullptr,
                 grad->w1, H, st);
    if (e == cudaSuccess) e = colsum(dh1, n, H, grad->b1, st);
    return e == cudaSuccess ? ADMIX_OK : ADMIX_ERR_CUDA;
}

int admix_mlp_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float beta1, float beta2,
                   float eps, int32_t t, void *stream)
{
    if (!w || !g || !m || !v || n < 1 || t < 1) return ADMIX_ERR_ARG;
    const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
    const unsigned grid = (unsigned)std::min<int64_t>(4096, (n + 255) / 256);
    k_adam<<<grid, 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? ADMIX_OK : ADMIX_ERR_CUDA;
}

int admix_warm_p(const uint8_t *d_bed, int64_t pitch, int64_t I, int64_t J, int32_t K, const double *d_q,
                 double *d_p, void *stream)
{
    if (!d_bed || !d_q || !d_p || I < 1 || J < 1 || K < 1 || K > ADMIX_MAX_K || pitch < (I + 3) / 4)
        return ADMIX_ERR_ARG;
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, (k_warm_p<KK><<<(unsigned)((J + 127) / 128), 128, 0, (cudaStream_t)stream>>>(d_bed, pitch, I, J,
                                                                                                  d_q, d_p),
                         e = cudaGetLastError()));
    return e == cudaSuccess ? ADMIX_OK : ADMIX_ERR_CUDA;
}

} /* extern "C" */
