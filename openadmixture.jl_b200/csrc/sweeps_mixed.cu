/*
 * sweeps_mixed.cu -- the mixed-precision ("chosen") form of the gradient / Hessian sweeps and
 * of the log-likelihood pass on sm_100a tensor cores.
 *
 * Q side (update_q_loop_skipmissing!, loops.jl:867-894):
 *   XtX_q[i] = sum_j w1_ij p_j p_j' + w2_ij pbar_j pbar_j',  Xtz_q[i] = sum_j z1_ij p_j + z2_ij pbar_j
 *   z1 = nm g / qp, z2 = nm (2-g) / (1-qp), w1 = z1 / qp, w2 = z2 / (1-qp), pbar = 1 - p
 * P side (update_p_loop_skipmissing!, loops.jl:923-950):
 *   XtX_p[j] = sum_i (w1 + w2)_ij q_i q_i',  Xtz_p[j] = sum_i (z1 - z2)_ij q_i
 *
 * Each Hessian is a GEMM whose rows are the 128 problems of a CTA (individuals or SNPs), whose
 * reduction runs over the other axis and whose columns are the K(K+1)/2 packed pairs k <= k2.
 * CUDA cores produce the BF16 weight tile (A) and the BF16 pair-product tile (B) of each chunk in
 * shared memory -- qp and 1-qp = sum_k q_k (1-p_k) in FP32 with paired __ffma2_rn, one
 * reciprocal per cell, the gradient in FP32 summed into FP64 per chunk -- and one thread issues
 * tcgen05.mma into an FP32 accumulator in tensor memory.  Tiles are double buffered, so the MMAs
 * of chunk c run while chunk c+1 is produced; completion is signalled on an mbarrier.  The
 * epilogue reads the accumulator with tcgen05.ld and writes the FP64 partial layout of the FP64
 * sweeps, so the QP kernels consume either.
 *
 * Genotypes are read from the handle's padded layout: columns at a pitch that is a multiple of
 * 16 bytes, padding bytes and padding bits coded missing (01), so whole 16-byte groups can be
 * loaded without per-individual bound checks.  Requires sum_k q_k = 1 (every projected Q).
 */
#include "common.cuh"
#include "kernels.h"
#include "tc05.cuh"

namespace {

constexpr uint32_t MX_WAIT_LIMIT = 1u << 22;   /* polls; an MMA batch completes in microseconds */

__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

/* Code-pair table: index c0 | c1 << 2 of two cells -> (nm g, nm g, nm (2-g), nm (2-g));
 * codes 00 -> (0, 2), 01 (missing) -> (0, 0), 10 -> (1, 1), 11 -> (2, 0).  Stored 8 times so
 * lane l of a quarter-warp always reads bank group l: entry e, copy l at float4 index 8e + l. */
__device__ __forceinline__ void code_table_init(float4 *tab, int tid, int nthreads)
{
    const float A1[4] = {0.f, 0.f, 1.f, 2.f}, A2[4] = {2.f, 0.f, 1.f, 0.f};
    for (int t = tid; t < 128; t += nthreads) {
        const int e = t >> 3, c0 = e & 3, c1 = e >> 2;
        tab[t] = make_float4(A1[c0], A1[c1], A2[c0], A2[c1]);
    }
}

/* 8 individuals' codes of two SNP columns interleaved byte-wise: [a0 b0 a1 b1 ...] */
__device__ __forceinline__ uint4 interleave8(uint2 a, uint2 b)
{
    return make_uint4(__byte_perm(a.x, b.x, 0x5140), __byte_perm(a.x, b.x, 0x7362),
                      __byte_perm(a.y, b.y, 0x5140), __byte_perm(a.y, b.y, 0x7362));
}

/* ===================================================================== Q side */

constexpr int MQ_JC = 32;          /* SNPs per chunk = 2 MMA K-steps */
constexpr int MQ_THREADS = 128;    /* one thread per individual = accumulator row */

template <int K>
struct MQ {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + 15) / 16) * 16;              /* MMA N (multiple of 16 for M = 128) */
    static constexpr uint32_t NCOLS = tmem_cols_for(N);
    static constexpr int E = T + K;                             /* partial entries per individual */
    static constexpr uint32_t A_BYTES = 128 * MQ_JC * 2;        /* one BF16 weight tile: 8 KB */
    static constexpr uint32_t B_BYTES = N * MQ_JC * 2;          /* one BF16 pair-product tile */
    static constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int PS = MQ_JC + 2;                        /* P row stride (floats): rows on distinct banks */
    static constexpr uint32_t PBUF = 2 * K * PS * 4;            /* p and 1-p of one chunk, FP32 [k][jj] */
    static constexpr uint32_t GBUF = MQ_JC * 32;                /* genotype bytes of one chunk */
    static constexpr uint32_t OFF_P = 2 * STAGE_BYTES;          /* two P buffers */
    static constexpr uint32_t OFF_G = OFF_P + 2 * PBUF;         /* two G buffers, [pair][byte][2] */
    static constexpr uint32_t OFF_TAB = OFF_G + 2 * GBUF;       /* float4 [16][8] code table */
    static constexpr uint32_t SMEM = OFF_TAB + 128 * 16 + 1024; /* + alignment slack */
    /* A core matrices 128 B apart along M, 2048 B along K; B 128 B along N, 16 N bytes along K */
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr int PREF_P = (K * MQ_JC + MQ_THREADS - 1) / MQ_THREADS;
};

/* One chunk's inputs in registers (loaded a chunk ahead): threads 0..63 hold 8 bytes of each of
 * the SNP pair's two columns (pair t >> 2, bytes 8 (t & 3) .. +7 of the CTA's 32); every thread
 * holds up to PREF_P allele frequencies. */
template <int K>
struct QChunk {
    uint2 ga, gb;
    double pv[MQ<K>::PREF_P];
};

template <int K>
__device__ __forceinline__ void qchunk_load(QChunk<K> &cr, const uint8_t *__restrict__ bed, int64_t pitch,
                                            const double *__restrict__ p, int64_t i0, int64_t jc, int n, int tid)
{
    if (tid < 64) {
        const int m = tid >> 2, qb = tid & 3;
        const size_t off = (size_t)(i0 / 4) + 8 * qb;
        const uint2 miss = make_uint2(0x55555555u, 0x55555555u);
        cr.ga = (2 * m < n) ? __ldg((const uint2 *)(bed + (size_t)(jc + 2 * m) * pitch + off)) : miss;
        cr.gb = (2 * m + 1 < n) ? __ldg((const uint2 *)(bed + (size_t)(jc + 2 * m + 1) * pitch + off)) : miss;
    }
#pragma unroll
    for (int u = 0; u < MQ<K>::PREF_P; ++u) {
        const int t = tid + u * MQ_THREADS;          /* t = jj * K + k: coalesced loads; the padded */
        const int jj = t / K;                        /* row stride keeps the stores <= 2-way conflicted */
        cr.pv[u] = (t < K * MQ_JC && jj < n) ? p[(size_t)K * jc + t] : 0.5;
    }
}

/* registers -> shared: p / 1-p as FP32 [k][jj]; genotypes as [pair m][byte b][2] */
template <int K>
__device__ __forceinline__ void qchunk_store(const QChunk<K> &cr, float *Pb, uint8_t *Gb, int tid)
{
    if (tid < 64) {
        const int m = tid >> 2, qb = tid & 3;
        *(uint4 *)(Gb + (m * 32 + 8 * qb) * 2) = interleave8(cr.ga, cr.gb);
    }
#pragma unroll
    for (int u = 0; u < MQ<K>::PREF_P; ++u) {
        const int t = tid + u * MQ_THREADS;
        if (t < K * MQ_JC) {
            const int jj = t / K, k = t - jj * K;
            Pb[k * MQ<K>::PS + jj] = (float)cr.pv[u];
            Pb[K * MQ<K>::PS + k * MQ<K>::PS + jj] = (float)(1.0 - cr.pv[u]);
        }
    }
}

template <int K>
__global__ void __launch_bounds__(MQ_THREADS)
k_sweep_q_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
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
    const float4 *tab = (const float4 *)(sm + C::OFF_TAB) + (tid & 7);

    if (warp == 0) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_fence_init();
    }
    code_table_init((float4 *)(sm + C::OFF_TAB), tid, MQ_THREADS);
    QChunk<K> cr;
    if (nchunk > 0) {
        qchunk_load<K>(cr, bed, pitch, p, i0, j0, (int)min((int64_t)MQ_JC, j1 - j0), tid);
        qchunk_store<K>(cr, (float *)(sm + C::OFF_P), sm + C::OFF_G, tid);
    }
    if (nchunk > 1) qchunk_load<K>(cr, bed, pitch, p, i0, j0 + MQ_JC, (int)min((int64_t)MQ_JC, j1 - j0 - MQ_JC), tid);
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
    const uint32_t gmask = valid ? 0xFFFFu : 0u;        /* rows beyond I read code pair 01|01 */
    constexpr uint32_t idesc = idesc_bf16_f32(128, N);
    bool ok = true;

    for (int c = 0; c < nchunk; ++c) {
        const int s = c & 1;
        uint8_t *At = sm + s * C::STAGE_BYTES;                 /* W1 tile, then W2 tile */
        uint8_t *Bt = At + 2 * C::A_BYTES;                      /* PP tile, then PbarPbar tile */
        const float *Pb = (const float *)(sm + C::OFF_P + s * C::PBUF);
        const uint8_t *Gb = sm + C::OFF_G + s * C::GBUF;
        if (c >= 2 && ok) {                                     /* MMAs of chunk c-2 read this stage */
            if (!mbar_wait_bounded(&mbar[s], (uint32_t)(((c - 2) >> 1) & 1), MX_WAIT_LIMIT)) {
                ok = false;
                if (tid == 0) atomicOr(err, 1);
            }
        }
        /* B tiles: task (term, kc, nn) writes pair nn's 8 SNPs of k-chunk kc at kc*16N + 16nn */
        for (int t = tid; t < 2 * 4 * N; t += MQ_THREADS) {
            const int term = t / (4 * N), rem = t - term * 4 * N;
            const int kc = rem / N, nn = rem - kc * N;
            uint32_t w[4] = {0u, 0u, 0u, 0u};
            if (nn < T) {
                int ka, kb;
                tri_pair(nn, ka, kb);
                const float *src = Pb + term * K * C::PS;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int jj = kc * 8 + 2 * e;
                    w[e] = pack_bf16x2(src[ka * C::PS + jj] * src[kb * C::PS + jj],
                                       src[ka * C::PS + jj + 1] * src[kb * C::PS + jj + 1]);
                }
            }
            *(uint4 *)(Bt + term * C::B_BYTES + kc * C::B_LBO + 16 * nn) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        /* producer: this thread's individual, the chunk's 32 SNPs as 16 pairs */
        const float2 *P2 = (const float2 *)Pb;                  /* [k][pair], row stride PS / 2 */
        const float2 *Pb2 = (const float2 *)(Pb + K * C::PS);
        const uint16_t *G2 = (const uint16_t *)Gb + (tid >> 2);  /* [pair][byte]: both SNPs */
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
                const float4 a = tab[8 * ((tb & 3u) | ((tb >> 6) & 12u))];
                float2 qp = make_float2(0.f, 0.f), om = make_float2(0.f, 0.f);
                float2 pv[K], pbv[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    pv[k] = P2[k * (C::PS / 2) + m];
                    pbv[k] = Pb2[k * (C::PS / 2) + m];
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
        if (c + 1 < nchunk) {
            qchunk_store<K>(cr, (float *)(sm + C::OFF_P + (s ^ 1) * C::PBUF), sm + C::OFF_G + (s ^ 1) * C::GBUF, tid);
            if (c + 2 < nchunk) {
                const int64_t jn = j0 + (int64_t)(c + 2) * MQ_JC;
                qchunk_load<K>(cr, bed, pitch, p, i0, jn, (int)min((int64_t)MQ_JC, j1 - jn), tid);
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
    /* wait for the last MMAs of both stages (bounded even after a failed wait, so the TMEM is
     * not released under an MMA still in flight) */
    for (int c = max(0, nchunk - 2); c < nchunk; ++c) {
        const int s = c & 1;
        if (!mbar_wait_bounded(&mbar[s], (uint32_t)((c >> 1) & 1), ok ? MX_WAIT_LIMIT : 1024u)) {
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

/* ===================================================================== P side
 * Thread = SNP row; individuals in chunks of 64 (one 16-byte load of the thread's own column);
 * the 4 bits of an individual pair index the code table directly. */
constexpr int MP_IC = 64;
constexpr int MP_THREADS = 128;

template <int K>
struct MP {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + 15) / 16) * 16;
    static constexpr uint32_t NCOLS = tmem_cols_for(N);
    static constexpr int E = T + K;
    static constexpr uint32_t A_BYTES = 128 * MP_IC * 2;        /* one BF16 weight tile: 16 KB */
    static constexpr uint32_t B_BYTES = N * MP_IC * 2;
    static constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int QS = MP_IC + 2;                        /* q row stride (floats) */
    static constexpr uint32_t QBUF = K * QS * 4;                /* q of one chunk, FP32 [k][i] */
    static constexpr uint32_t OFF_Q = 2 * STAGE_BYTES;
    static constexpr uint32_t OFF_TAB = OFF_Q + 2 * QBUF;
    static constexpr uint32_t SMEM = OFF_TAB + 128 * 16 + 1024;
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr int PREF_Q = (K * MP_IC + MP_THREADS - 1) / MP_THREADS;
};

/* 64 individuals' codes of SNP column j from individual ic (a multiple of 64) */
__device__ __forceinline__ uint4 col_load64(const uint8_t *__restrict__ bed, int64_t pitch, int64_t j, bool valid,
                                            int64_t ic)
{
    return valid ? __ldg((const uint4 *)(bed + (size_t)j * pitch + (size_t)(ic / 4)))
                 : make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u);
}

__device__ __forceinline__ uint32_t pair_code(const uint4 &g, int m)
{
    const uint32_t w = (m < 8) ? g.x : ((m < 16) ? g.y : ((m < 24) ? g.z : g.w));
    return (w >> (4 * (m & 7))) & 15u;
}

template <int K>
__global__ void __launch_bounds__(MP_THREADS)
k_sweep_p_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
                const double *__restrict__ q, const double *__restrict__ p, int64_t islice,
                double *__restrict__ out, int *__restrict__ err)
{
    using C = MP<K>;
    constexpr int T = C::T, N = C::N, E = C::E;
    extern __shared__ __align__(1024) uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    __shared__ uint64_t mbar[2];
    __shared__ uint32_t tmem_holder;

    const int tid = threadIdx.x, warp = tid >> 5;
    const int64_t j = (int64_t)blockIdx.x * 128 + tid;
    const bool valid = j < J;
    const int64_t ia = (int64_t)blockIdx.y * islice;
    const int64_t ib = min(I, ia + islice);
    const int nchunk = (int)((ib - ia + MP_IC - 1) / MP_IC);
    const float4 *tab = (const float4 *)(sm + C::OFF_TAB) + (tid & 7);

    if (warp == 0) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_fence_init();
    }
    code_table_init((float4 *)(sm + C::OFF_TAB), tid, MP_THREADS);
    double qr[C::PREF_Q];
    auto qload = [&](int64_t ic) {
#pragma unroll
        for (int u = 0; u < C::PREF_Q; ++u) {
            const int t = tid + u * MP_THREADS;              /* t = ii * K + k: coalesced */
            const int ii = t / K;
            qr[u] = (t < K * MP_IC && ic + ii < ib) ? q[(size_t)K * ic + t] : 1.0 / K;
        }
    };
    auto qstore = [&](float *Qb) {
#pragma unroll
        for (int u = 0; u < C::PREF_Q; ++u) {
            const int t = tid + u * MP_THREADS;
            if (t < K * MP_IC) {
                const int ii = t / K, k = t - ii * K;
                Qb[k * C::QS + ii] = (float)qr[u];
            }
        }
    };
    uint4 gcur = make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u), gnext = gcur;
    if (nchunk > 0) {
        qload(ia);
        qstore((float *)(sm + C::OFF_Q));
        gcur = col_load64(bed, pitch, j, valid, ia);
    }
    if (nchunk > 1) {
        qload(ia + MP_IC);
        gnext = col_load64(bed, pitch, j, valid, ia + MP_IC);
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_holder;

    float2 pd[K], pbd[K];            /* p_k and 1 - p_k duplicated into pairs */
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double pv = valid ? p[(size_t)K * j + k] : 0.5;
        pd[k] = make_float2((float)pv, (float)pv);
        const float pb = (float)(1.0 - pv);
        pbd[k] = make_float2(pb, pb);
    }
    double gd[K];
#pragma unroll
    for (int k = 0; k < K; ++k) gd[k] = 0.0;
    constexpr uint32_t idesc = idesc_bf16_f32(128, N);
    bool ok = true;

    for (int c = 0; c < nchunk; ++c) {
        const int s = c & 1;
        uint8_t *At = sm + s * C::STAGE_BYTES;
        uint8_t *Bt = At + C::A_BYTES;
        const float *Qb = (const float *)(sm + C::OFF_Q + s * C::QBUF);
        if (c >= 2 && ok) {
            if (!mbar_wait_bounded(&mbar[s], (uint32_t)(((c - 2) >> 1) & 1), MX_WAIT_LIMIT)) {
                ok = false;
                if (tid == 0) atomicOr(err, 1);
            }
        }
        /* B tile: QQ[n][i] = q_ka(i) q_kb(i) in BF16, task (kc, nn) -> 16-byte row chunk */
        for (int t = tid; t < 8 * N; t += MP_THREADS) {
            const int kc = t / N, nn = t - kc * N;
            uint32_t w[4] = {0u, 0u, 0u, 0u};
            if (nn < T) {
                int ka, kb;
                tri_pair(nn, ka, kb);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int ii = kc * 8 + 2 * e;
                    w[e] = pack_bf16x2(Qb[ka * C::QS + ii] * Qb[kb * C::QS + ii],
                                       Qb[ka * C::QS + ii + 1] * Qb[kb * C::QS + ii + 1]);
                }
            }
            *(uint4 *)(Bt + kc * C::B_LBO + 16 * nn) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        const float2 *Q2 = (const float2 *)Qb;                  /* [k][pair] */
        float2 ga[K];
#pragma unroll
        for (int k = 0; k < K; ++k) ga[k] = make_float2(0.f, 0.f);
#pragma unroll
        for (int kc = 0; kc < 8; ++kc) {
            uint32_t cp[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = kc * 4 + e;                       /* individuals 2m, 2m+1 of the chunk */
                const float4 a = tab[8 * pair_code(gcur, m)];
                float2 qp = make_float2(0.f, 0.f), om = make_float2(0.f, 0.f);
                float2 qv[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    qv[k] = Q2[k * (C::QS / 2) + m];
                    qp = __ffma2_rn(qv[k], pd[k], qp);
                    om = __ffma2_rn(qv[k], pbd[k], om);
                }
                const float2 pr = __fmul2_rn(qp, om);
                const float2 rr = make_float2(rcp_approx(pr.x), rcp_approx(pr.y));
                const float2 r1 = __fmul2_rn(om, rr), r2 = __fmul2_rn(qp, rr);
                const float2 z1 = __fmul2_rn(make_float2(a.x, a.y), r1);
                const float2 z2 = __fmul2_rn(make_float2(a.z, a.w), r2);
                const float2 cw = __ffma2_rn(z1, r1, __fmul2_rn(z2, r2));   /* nm (g/qp^2 + (2-g)/(1-qp)^2) */
                const float2 zz = make_float2(z1.x - z2.x, z1.y - z2.y);    /* nm (g/qp - (2-g)/(1-qp)) */
#pragma unroll
                for (int k = 0; k < K; ++k) ga[k] = __ffma2_rn(zz, qv[k], ga[k]);
                cp[e] = pack_bf16x2(cw.x, cw.y);
            }
            *(uint4 *)(At + kc * C::A_LBO + 16 * tid) = make_uint4(cp[0], cp[1], cp[2], cp[3]);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) gd[k] += (double)ga[k].x + (double)ga[k].y;
        if (c + 1 < nchunk) {
            qstore((float *)(sm + C::OFF_Q + (s ^ 1) * C::QBUF));
            gcur = gnext;
            if (c + 2 < nchunk) {
                const int64_t icn = ia + (int64_t)(c + 2) * MP_IC;
                qload(icn);
                gnext = col_load64(bed, pitch, j, valid, icn);
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_fence_after_sync();
            const uint32_t abase = smem_u32(At), bbase = smem_u32(Bt);
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const uint64_t ad = umma_desc_kmajor(abase + ks * 2 * C::A_LBO, C::A_LBO, C::A_SBO);
                const uint64_t bd = umma_desc_kmajor(bbase + ks * 2 * C::B_LBO, C::B_LBO, C::B_SBO);
                tc_mma_bf16(tmem, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
            }
            tc_commit(&mbar[s]);
        }
    }
    for (int c = max(0, nchunk - 2); c < nchunk; ++c) {
        const int s = c & 1;
        if (!mbar_wait_bounded(&mbar[s], (uint32_t)((c >> 1) & 1), ok ? MX_WAIT_LIMIT : 1024u)) {
            ok = false;
            if (tid == 0) atomicOr(err, 1);
        }
    }
    tc_fence_after_sync();
    double *o = out + ((size_t)blockIdx.y * J + (valid ? j : 0)) * E;
    if (valid) {
#pragma unroll
        for (int k = 0; k < K; ++k) o[T + k] = gd[k];
    }
    if (nchunk > 0) {
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

/* ===================================================================== loglik
 * loglikelihood_loop_skipmissing (loops.jl:517-539) with FP32 cells: thread = SNP, individuals
 * in pairs; each cell contributes qp^g (1-qp)^(2-g) (1 when missing), two cells' factors are
 * multiplied in FP32 and folded into an FP64 running product whose exponent moves into an
 * integer every 12 pairs; one FP64 log per thread at the end.  Every product is rounded to
 * nearest, so the rounding error is a random walk far below the convergence test's resolution. */
constexpr int ML_IC = 64;

template <int K>
__global__ void __launch_bounds__(128)
k_loglik_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
               const double *__restrict__ q, const double *__restrict__ p, int64_t islice,
               double *__restrict__ partial)
{
    constexpr int PREF = (K * ML_IC + 127) / 128;
    __shared__ float2 Qs[2][K][ML_IC / 2];
    __shared__ double red[4];
    const int tid = threadIdx.x;
    const int64_t j = (int64_t)blockIdx.x * 128 + tid;
    const bool valid = j < J;
    const int64_t ia = (int64_t)blockIdx.y * islice;
    const int64_t ib = min(I, ia + islice);
    const int nchunk = (int)((ib - ia + ML_IC - 1) / ML_IC);
    float2 pd[K], pbd[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const double pv = valid ? p[(size_t)K * j + k] : 0.5;
        pd[k] = make_float2((float)pv, (float)pv);
        const float pb = (float)(1.0 - pv);
        pbd[k] = make_float2(pb, pb);
    }
    float qr[PREF];
    uint4 gnext = make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u), g = gnext;
    auto load = [&](int64_t ic) {
#pragma unroll
        for (int u = 0; u < PREF; ++u) {
            const int t = tid + u * 128;                 /* t = k * IC + ii */
            const int k = t / ML_IC, ii = t - k * ML_IC;
            qr[u] = (t < K * ML_IC && ic + ii < ib) ? (float)q[(size_t)K * (ic + ii) + k] : 1.0f / K;
        }
        gnext = col_load64(bed, pitch, j, valid, ic);
    };
    auto store = [&](int s) {
#pragma unroll
        for (int u = 0; u < PREF; ++u) {
            const int t = tid + u * 128;
            if (t < K * ML_IC) {
                const int k = t / ML_IC, ii = t - k * ML_IC;
                ((float *)Qs[s][k])[ii] = qr[u];
            }
        }
    };
    if (nchunk > 0) { load(ia); store(0); g = gnext; }
    if (nchunk > 1) load(ia + ML_IC);
    __syncthreads();
    double prod = 1.0;
    int64_t ex = 0;
    for (int c = 0; c < nchunk; ++c) {
        const int s = c & 1;
#pragma unroll
        for (int m = 0; m < ML_IC / 2; ++m) {
            const uint32_t code4 = pair_code(g, m);
            float2 qp = make_float2(0.f, 0.f), om = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const float2 qv = Qs[s][k][m];
                qp = __ffma2_rn(qv, pd[k], qp);
                om = __ffma2_rn(qv, pbd[k], om);
            }
            /* factor per code: 00 -> om^2, 01 -> 1, 10 -> qp om, 11 -> qp^2 */
            const uint32_t c0 = code4 & 3u, c1 = code4 >> 2;
            const float u0 = (c0 & 2u) ? qp.x : om.x, v0 = (c0 == 3u) ? qp.x : om.x;
            const float u1 = (c1 & 2u) ? qp.y : om.y, v1 = (c1 == 3u) ? qp.y : om.y;
            const float f0 = (c0 == 1u) ? 1.f : u0 * v0;
            const float f1 = (c1 == 1u) ? 1.f : u1 * v1;
            prod *= (double)(f0 * f1);
            if ((m % 12) == 11) {
                const int64_t bits = __double_as_longlong(prod);
                ex += ((bits >> 52) & 0x7FF) - 1023;
                prod = __longlong_as_double((bits & ~(0x7FFLL << 52)) | (1023LL << 52));
            }
        }
        const int64_t bits = __double_as_longlong(prod);
        ex += ((bits >> 52) & 0x7FF) - 1023;
        prod = __longlong_as_double((bits & ~(0x7FFLL << 52)) | (1023LL << 52));
        if (c + 1 < nchunk) {
            store(s ^ 1);
            g = gnext;
            if (c + 2 < nchunk) load(ia + (int64_t)(c + 2) * ML_IC);
        }
        __syncthreads();
    }
    double ll = valid ? (log(prod) + (double)ex * 0.69314718055994530942) : 0.0;
    for (int o = 16; o > 0; o >>= 1) ll += __shfl_down_sync(0xffffffffu, ll, o);
    if ((tid & 31) == 0) red[tid >> 5] = ll;
    __syncthreads();
    if (tid == 0) partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = red[0] + red[1] + red[2] + red[3];
}

__global__ void __launch_bounds__(1024)
k_sum_partials_mixed(const double *__restrict__ partial, int64_t n, double *__restrict__ out)
{
    __shared__ double red[32];
    double v = 0.0;
    for (int64_t t = threadIdx.x; t < n; t += blockDim.x) v += partial[t];
    const double s = block_sum(v, red);
    if (threadIdx.x == 0) *out = s;
}

template <int K>
cudaError_t prepare_mixed_t()
{
    cudaError_t e = cudaFuncSetAttribute(k_sweep_q_mixed<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MQ<K>::SMEM);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sweep_p_mixed<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MP<K>::SMEM);
    return e;
}

template <int K>
cudaError_t launch_q_mixed_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                             const double *p, const SweepPlan &pl, double *out, int *err, cudaStream_t st)
{
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_sweep_q_mixed<K><<<grid, MQ_THREADS, MQ<K>::SMEM, st>>>(bed, I, J, pitch, q, p, pl.slice, out, err);
    return cudaGetLastError();
}

template <int K>
cudaError_t launch_p_mixed_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                             const double *p, const SweepPlan &pl, double *out, int *err, cudaStream_t st)
{
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_sweep_p_mixed<K><<<grid, MP_THREADS, MP<K>::SMEM, st>>>(bed, I, J, pitch, q, p, pl.slice, out, err);
    return cudaGetLastError();
}

template <int K>
cudaError_t launch_ll_mixed_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                              const double *p, const SweepPlan &pl, double *partial, double *out, cudaStream_t st)
{
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_loglik_mixed<K><<<grid, 128, 0, st>>>(bed, I, J, pitch, q, p, pl.slice, partial);
    k_sum_partials_mixed<<<1, 1024, 0, st>>>(partial, (int64_t)pl.gx * pl.S, out);
    return cudaGetLastError();
}

/* slices over the second axis: enough CTAs to cover the GPU, each slice a multiple of `unit` */
SweepPlan plan_rows(int64_t rows, int64_t cols, int sms, int per_sm, int64_t unit)
{
    SweepPlan pl;
    pl.gx = (int)((rows + 127) / 128);
    const int64_t target = (int64_t)sms * per_sm;
    int64_t S = (target + pl.gx - 1) / pl.gx;
    S = std::max<int64_t>(1, std::min<int64_t>(S, (cols + 4 * unit - 1) / (4 * unit)));
    int64_t slice = (cols + S - 1) / S;
    slice = (slice + unit - 1) / unit * unit;
    pl.slice = slice;
    pl.S = (int)((cols + slice - 1) / slice);
    return pl;
}

} // namespace

cudaError_t prepare_mixed(int K)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = prepare_mixed_t<KK>());
    return e;
}

/* One CTA per 128 individuals and SNP slice. */
SweepPlan plan_sweep_q_mixed(int K, int64_t I, int64_t J, int sms)
{
    (void)K;
    return plan_rows(I, J, sms, 4, MQ_JC);
}

/* One CTA per 128 SNPs and individual slice (slices are multiples of 64 individuals). */
SweepPlan plan_sweep_p_mixed(int K, int64_t I, int64_t J, int sms)
{
    (void)K;
    return plan_rows(J, I, sms, 4, MP_IC);
}

SweepPlan plan_loglik_mixed(int64_t I, int64_t J, int sms)
{
    return plan_rows(J, I, sms, 8, ML_IC);
}

cudaError_t launch_sweep_q_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                 const double *p, const SweepPlan &pl, double *out, int *err, cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_q_mixed_t<KK>(bed, I, J, pitch, q, p, pl, out, err, st));
    return e;
}

cudaError_t launch_sweep_p_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                 const double *p, const SweepPlan &pl, double *out, int *err, cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_p_mixed_t<KK>(bed, I, J, pitch, q, p, pl, out, err, st));
    return e;
}

cudaError_t launch_loglik_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                const double *p, const SweepPlan &pl, double *partial, double *out, cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_ll_mixed_t<KK>(bed, I, J, pitch, q, p, pl, partial, out, st));
    return e;
}
