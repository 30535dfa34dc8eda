/*
 * sweeps_mixed.cu -- the mixed-precision ("chosen") form of the Q-block gradient / Hessian
 * sweep (update_q_loop_skipmissing!, loops.jl:867-894) on sm_100a tensor cores.
 *
 *   XtX_q[i] = sum_j w1_ij p_j p_j' + w2_ij pbar_j pbar_j'        (the Hessian, K x K)
 *   Xtz_q[i] = sum_j z1_ij p_j + z2_ij pbar_j                    (the gradient)
 *   z1 = nm g / qp, z2 = nm (2-g) / (1-qp), w1 = z1 / qp, w2 = z2 / (1-qp), pbar = 1 - p
 *
 * The Hessian is a GEMM: rows = 128 individuals of the CTA, reduction over SNPs, columns =
 * the K(K+1)/2 packed pairs (k <= k2):  D = [W1 | W2] x [P(x)P ; Pbar(x)Pbar].  Each 64-SNP chunk
 * the 256 threads (two per individual, 32 SNPs each) decode the genotypes, compute qp and
 * 1-qp = sum_k q_k (1-p_k) in FP32 (paired __ffma2_rn over two SNPs), one reciprocal per cell,
 * the weights, and the gradient in FP32 (chunk sums added into FP64); they write w1 and w2 as
 * BF16 into the A tiles and the pair products as BF16 into the B tiles.  One thread issues
 * eight tcgen05.mma (4 K-steps x 2 terms) accumulating in FP32 in TMEM; A/B tiles are double
 * buffered, the MMA of chunk c overlapping the production of chunk c+1, with completion
 * signalled through an mbarrier.  The epilogue reads the accumulator with tcgen05.ld and writes
 * the same FP64 partial layout as the FP64 sweep, so the QP kernels consume either.
 *
 * Requires sum_k q_k = 1 (true for every projected Q the SQP updates see).
 */
#include "common.cuh"
#include "kernels.h"
#include "tc05.cuh"

namespace {

constexpr int MQ_JC = 32;          /* SNPs per chunk = MMA K extent per chunk (2 K-steps) */
constexpr int MQ_THREADS = 128;    /* one thread per individual = per accumulator row */
constexpr uint32_t MQ_WAIT_LIMIT = 1u << 22;   /* polls; an MMA batch completes in microseconds */

template <int K>
struct MQ {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + 15) / 16) * 16;              /* MMA N (multiple of 16 for M = 128) */
    static constexpr uint32_t NCOLS = tmem_cols_for(N);
    static constexpr int E = T + K;                             /* partial entries per individual */
    static constexpr uint32_t A_BYTES = 128 * MQ_JC * 2;        /* one BF16 weight tile: 8 KB */
    static constexpr uint32_t B_BYTES = N * MQ_JC * 2;          /* one BF16 pair-product tile */
    static constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr uint32_t PBUF = 2 * K * MQ_JC * 4;         /* p and 1-p of one chunk, FP32 */
    static constexpr uint32_t GBUF = MQ_JC * 32;                /* genotype bytes of one chunk */
    static constexpr uint32_t OFF_P = 2 * STAGE_BYTES;          /* two P buffers */
    static constexpr uint32_t OFF_G = OFF_P + 2 * PBUF;         /* two G buffers, [pair][byte][2] */
    static constexpr uint32_t OFF_TAB = OFF_G + 2 * GBUF;       /* float4 [16] code-pair weights */
    static constexpr uint32_t SMEM = OFF_TAB + 16 * 16 + 1024;  /* + alignment slack */
    /* descriptor strides: A core matrices 128 B apart along M, 2048 B along K;
     * B core matrices 128 B apart along N, 16 N bytes along K */
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr int PREF_P = (K * MQ_JC + MQ_THREADS - 1) / MQ_THREADS;   /* p values per thread */
};

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

/* Global loads of one chunk's inputs into registers (issued a chunk ahead). */
template <int K>
struct ChunkRegs {
    uint32_t g[2];                 /* 8 genotype bytes: columns 2*(tid/32)+{0,1}... see load */
    double pv[MQ<K>::PREF_P];
};

template <int K>
__device__ __forceinline__ void chunk_load(ChunkRegs<K> &cr, const uint8_t *__restrict__ bed, int64_t Ib,
                                           const double *__restrict__ p, int64_t i0, int64_t jc, int n, int tid)
{
    /* genotype bytes: thread (b = tid & 31, q4 = tid >> 5) loads byte b of columns 8*q4 .. 8*q4+7 */
    const int b = tid & 31, q4 = tid >> 5;
    const int64_t bi = i0 / 4 + b;
    uint32_t w[2] = {0u, 0u};
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int jj = q4 * 8 + u;
        const uint32_t v = (jj < n && bi < Ib) ? (uint32_t)__ldg(bed + (size_t)(jc + jj) * Ib + bi) : 0x55u;
        w[u >> 2] |= v << (8 * (u & 3));
    }
    cr.g[0] = w[0];
    cr.g[1] = w[1];
#pragma unroll
    for (int u = 0; u < MQ<K>::PREF_P; ++u) {
        const int t = tid + u * MQ_THREADS;          /* t = jj * K + k over the chunk's K*JC values */
        const int jj = t / K;
        cr.pv[u] = (t < K * MQ_JC && jj < n) ? p[(size_t)K * jc + t] : 0.5;
    }
}

/* Registers -> shared buffers: p / 1-p as FP32 [k][jj], genotypes as [pair m][byte b][2]. */
template <int K>
__device__ __forceinline__ void chunk_store(const ChunkRegs<K> &cr, float *Pb, uint8_t *Gb, int tid)
{
    const int b = tid & 31, q4 = tid >> 5;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int jj = q4 * 8 + u;
        Gb[((jj >> 1) * 32 + b) * 2 + (jj & 1)] = (uint8_t)(cr.g[u >> 2] >> (8 * (u & 3)));
    }
#pragma unroll
    for (int u = 0; u < MQ<K>::PREF_P; ++u) {
        const int t = tid + u * MQ_THREADS;
        if (t < K * MQ_JC) {
            const int jj = t / K, k = t - jj * K;
            Pb[k * MQ_JC + jj] = (float)cr.pv[u];
            Pb[K * MQ_JC + k * MQ_JC + jj] = (float)(1.0 - cr.pv[u]);
        }
    }
}

template <int K>
__global__ void __launch_bounds__(MQ_THREADS)
k_sweep_q_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t Ib,
                const double *__restrict__ q, const double *__restrict__ p, int64_t jslice,
                double *__restrict__ out, int *__restrict__ err)
{
    using C = MQ<K>;
    constexpr int T = C::T, N = C::N, E = C::E;
    extern __shared__ __align__(1024) uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    __shared__ uint64_t mbar[2];
    __shared__ uint32_t tmem_holder;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int64_t i0 = (int64_t)blockIdx.x * 128;
    const int64_t i = i0 + tid;
    const bool valid = i < I;
    const int64_t j0 = (int64_t)blockIdx.y * jslice;
    const int64_t j1 = min(J, j0 + jslice);
    const int nchunk = (int)((j1 - j0 + MQ_JC - 1) / MQ_JC);
    float4 *tab = (float4 *)(sm + C::OFF_TAB);

    if (warp == 0) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_fence_init();
    }
    if (tid < 16) {
        /* code pair (c0 | c1 << 2) -> (nm g, nm g, nm (2-g), nm (2-g)) of the two cells;
         * codes 00 -> (0, 2), 01 (missing) -> (0, 0), 10 -> (1, 1), 11 -> (2, 0) */
        const float A1[4] = {0.f, 0.f, 1.f, 2.f}, A2[4] = {2.f, 0.f, 1.f, 0.f};
        const int c0 = tid & 3, c1 = tid >> 2;
        tab[tid] = make_float4(A1[c0], A1[c1], A2[c0], A2[c1]);
    }
    ChunkRegs<K> cr;
    if (nchunk > 0) {
        chunk_load<K>(cr, bed, Ib, p, i0, j0, (int)min((int64_t)MQ_JC, j1 - j0), tid);
        chunk_store<K>(cr, (float *)(sm + C::OFF_P), sm + C::OFF_G, tid);
    }
    if (nchunk > 1) chunk_load<K>(cr, bed, Ib, p, i0, j0 + MQ_JC, (int)min((int64_t)MQ_JC, j1 - j0 - MQ_JC), tid);
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_holder;

    float2 qq[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const float v = valid ? (float)q[(size_t)K * i + k] : 1.0f / K;
        qq[k] = make_float2(v, v);
    }
    double gd[K];
#pragma unroll
    for (int k = 0; k < K; ++k) gd[k] = 0.0;
    const int sh = valid ? (int)(i & 3) * 2 : 0;
    const uint32_t gmask = valid ? 0xFFFFu : 0u;        /* invalid rows read code pair 01|01 -> missing */
    constexpr uint32_t idesc = idesc_bf16_f32(128, N);
    bool ok = true;

    for (int c = 0; c < nchunk; ++c) {
        const int s = c & 1;
        uint8_t *At = sm + s * C::STAGE_BYTES;                 /* W1 tile, then W2 tile */
        uint8_t *Bt = At + 2 * C::A_BYTES;                      /* PP tile, then PbarPbar tile */
        const float *Pb = (const float *)(sm + C::OFF_P + s * C::PBUF);
        const uint8_t *Gb = sm + C::OFF_G + s * C::GBUF;
        if (c >= 2 && ok) {                                     /* MMAs of chunk c-2 read this stage */
            if (!mbar_wait_bounded(&mbar[s], (uint32_t)(((c - 2) >> 1) & 1), MQ_WAIT_LIMIT)) {
                ok = false;
                if (tid == 0) atomicOr(err, 1);
            }
        }
        /* B tiles: bf16 pair products; task (term, kc, nn) writes row nn's 8 SNPs of k-chunk kc
         * at kc*16N + 16nn (consecutive tasks -> consecutive 16-byte rows) */
        for (int t = tid; t < 2 * 4 * N; t += MQ_THREADS) {
            const int term = t / (4 * N), rem = t - term * 4 * N;
            const int kc = rem / N, nn = rem - kc * N;
            uint32_t w[4] = {0u, 0u, 0u, 0u};
            if (nn < T) {
                int ka, kb;
                tri_pair(nn, ka, kb);
                const float *src = Pb + term * K * MQ_JC;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int jj = kc * 8 + 2 * e;
                    const float lo = src[ka * MQ_JC + jj] * src[kb * MQ_JC + jj];
                    const float hi = src[ka * MQ_JC + jj + 1] * src[kb * MQ_JC + jj + 1];
                    w[e] = pack_bf16x2(lo, hi);
                }
            }
            *(uint4 *)(Bt + term * C::B_BYTES + kc * C::B_LBO + 16 * nn) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        /* producer: this thread's individual, the chunk's 32 SNPs as 16 pairs */
        const float2 *P2 = (const float2 *)Pb;                  /* [k][pair] */
        const float2 *Pb2 = (const float2 *)(Pb + K * MQ_JC);
        const uint16_t *G2 = (const uint16_t *)Gb + (tid >> 2);  /* [pair][byte]: both SNPs of a pair */
        float2 ga[K];
#pragma unroll
        for (int k = 0; k < K; ++k) ga[k] = make_float2(0.f, 0.f);
#pragma unroll
        for (int kc = 0; kc < 4; ++kc) {
            uint32_t w1p[4], w2p[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = kc * 4 + e;                       /* SNPs 2m, 2m+1 of the chunk */
                const uint32_t gw = ((uint32_t)G2[m * 32] & gmask) | (~gmask & 0x5555u);
                const uint32_t tb = gw >> sh;
                const float4 a = tab[(tb & 3u) | ((tb >> 6) & 12u)];
                float2 qp = make_float2(0.f, 0.f), om = make_float2(0.f, 0.f);
                float2 pv[K], pbv[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    pv[k] = P2[k * (MQ_JC / 2) + m];
                    pbv[k] = Pb2[k * (MQ_JC / 2) + m];
                    qp = __ffma2_rn(qq[k], pv[k], qp);
                    om = __ffma2_rn(qq[k], pbv[k], om);
                }
                const float2 pr = __fmul2_rn(qp, om);
                const float2 rr = make_float2(rcp_approx(pr.x), rcp_approx(pr.y));
                const float2 r1 = __fmul2_rn(om, rr), r2 = __fmul2_rn(qp, rr);   /* 1/qp, 1/(1-qp) */
                const float2 z1 = __fmul2_rn(make_float2(a.x, a.y), r1);
                const float2 z2 = __fmul2_rn(make_float2(a.z, a.w), r2);
                const float2 w1 = __fmul2_rn(z1, r1), w2 = __fmul2_rn(z2, r2);
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    ga[k] = __ffma2_rn(z1, pv[k], ga[k]);
                    ga[k] = __ffma2_rn(z2, pbv[k], ga[k]);
                }
                w1p[e] = pack_bf16x2(w1.x, w1.y);
                w2p[e] = pack_bf16x2(w2.x, w2.y);
            }
            /* A tiles: row tid, k-chunk kc at kc*2048 + 16 tid */
            *(uint4 *)(At + kc * C::A_LBO + 16 * tid) = make_uint4(w1p[0], w1p[1], w1p[2], w1p[3]);
            *(uint4 *)(At + C::A_BYTES + kc * C::A_LBO + 16 * tid) = make_uint4(w2p[0], w2p[1], w2p[2], w2p[3]);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) gd[k] += (double)ga[k].x + (double)ga[k].y;
        /* next chunk's inputs: registers -> the other buffer; then prefetch the one after */
        if (c + 1 < nchunk) {
            chunk_store<K>(cr, (float *)(sm + C::OFF_P + (s ^ 1) * C::PBUF), sm + C::OFF_G + (s ^ 1) * C::GBUF, tid);
            if (c + 2 < nchunk) {
                const int64_t jn = j0 + (int64_t)(c + 2) * MQ_JC;
                chunk_load<K>(cr, bed, Ib, p, i0, jn, (int)min((int64_t)MQ_JC, j1 - jn), tid);
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_fence_after_sync();
            const uint32_t abase = smem_u32(At), bbase = smem_u32(Bt);
#pragma unroll
            for (int term = 0; term < 2; ++term) {
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    const uint64_t ad = umma_desc_kmajor(abase + term * C::A_BYTES + ks * 2 * C::A_LBO, C::A_LBO, C::A_SBO);
                    const uint64_t bd = umma_desc_kmajor(bbase + term * C::B_BYTES + ks * 2 * C::B_LBO, C::B_LBO, C::B_SBO);
                    tc_mma_bf16(tmem, ad, bd, idesc, (c > 0 || term > 0 || ks > 0) ? 1u : 0u);
                }
            }
            tc_commit(&mbar[s]);
        }
    }
    /* wait for the last MMAs of both stages (bounded even after a failed wait, so the TMEM
     * is not released under an MMA still in flight) */
    for (int c = max(0, nchunk - 2); c < nchunk; ++c) {
        const int s = c & 1;
        if (!mbar_wait_bounded(&mbar[s], (uint32_t)((c >> 1) & 1), ok ? MQ_WAIT_LIMIT : 1024u)) {
            ok = false;
            if (tid == 0) atomicOr(err, 1);
        }
    }
    tc_fence_after_sync();
    double *o = out + ((size_t)blockIdx.y * I + (valid ? i : 0)) * E;
    if (valid) {
#pragma unroll
        for (int k = 0; k < K; ++k) o[T + k] = gd[k];
    }
    if (nchunk > 0) {
        /* Hessian: warp w reads TMEM lanes 32w .. 32w+31 (= this thread's row) */
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (valid) {
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    if (c0 + e < T) o[c0 + e] = ok ? (double)v[e] : __longlong_as_double(0x7ff8000000000000LL);
            }
        }
    } else if (valid) {
        for (int e = 0; e < T; ++e) o[e] = 0.0;
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc_warp(tmem, C::NCOLS);
}

template <int K>
cudaError_t prepare_mixed_t()
{
    return cudaFuncSetAttribute(k_sweep_q_mixed<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MQ<K>::SMEM);
}

template <int K>
cudaError_t launch_q_mixed_t(const uint8_t *bed, int64_t I, int64_t J, const double *q, const double *p,
                             const SweepPlan &pl, double *out, int *err, cudaStream_t st)
{
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_sweep_q_mixed<K><<<grid, MQ_THREADS, MQ<K>::SMEM, st>>>(bed, I, J, (I + 3) / 4, q, p, pl.slice, out, err);
    return cudaGetLastError();
}

} // namespace

cudaError_t prepare_mixed(int K)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = prepare_mixed_t<KK>());
    return e;
}

/* One CTA per 128 individuals and SNP slice; slices chosen so the grid covers the GPU. */
SweepPlan plan_sweep_q_mixed(int K, int64_t I, int64_t J, int sms)
{
    (void)K;
    SweepPlan pl;
    pl.gx = (int)((I + 127) / 128);
    const int64_t target = (int64_t)sms * 4;
    int64_t S = (target + pl.gx - 1) / pl.gx;
    S = std::max<int64_t>(1, std::min<int64_t>(S, (J + 255) / 256));
    pl.slice = (J + S - 1) / S;
    pl.S = (int)((J + pl.slice - 1) / pl.slice);
    return pl;
}

cudaError_t launch_sweep_q_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, const double *q,
                                 const double *p, const SweepPlan &pl, double *out, int *err,
                                 cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_q_mixed_t<KK>(bed, I, J, q, p, pl, out, err, st));
    return e;
}
