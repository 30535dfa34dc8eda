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

/* ===================================================================== P side
 *
 * update_p_loop_skipmissing! (loops.jl:923-950):
 *   XtX_p[j] = sum_i c_ij q_i q_i',  c = nm (g/qp^2 + (2-g)/(1-qp)^2)
 *   Xtz_p[j] = sum_i z_ij q_i,       z = nm (g/qp - (2-g)/(1-qp))
 * GEMM rows = 128 SNPs of the CTA (thread = SNP), reduction over individuals in chunks of 32,
 * columns = the K(K+1)/2 pairs: D = C x QQ'.  A thread reads its own column's 8 genotype bytes
 * per chunk (32 individuals); the 4 bits of an individual pair index the code table directly.
 */
constexpr int MP_IC = 32;
constexpr int MP_THREADS = 128;

template <int K>
struct MP {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + 15) / 16) * 16;
    static constexpr uint32_t NCOLS = tmem_cols_for(N);
    static constexpr int E = T + K;
    static constexpr uint32_t A_BYTES = 128 * MP_IC * 2;        /* one BF16 weight tile: 8 KB */
    static constexpr uint32_t B_BYTES = N * MP_IC * 2;
    static constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr uint32_t QBUF = K * MP_IC * 4;             /* q of one chunk, FP32 [k][i] */
    static constexpr uint32_t OFF_Q = 2 * STAGE_BYTES;
    static constexpr uint32_t OFF_TAB = OFF_Q + 2 * QBUF;
    static constexpr uint32_t SMEM = OFF_TAB + 16 * 16 + 1024;
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr int PREF_Q = (K * MP_IC + MP_THREADS - 1) / MP_THREADS;
};

/* 8 genotype bytes of column j for individuals ic .. ic+31, individuals >= I forced missing */
__device__ __forceinline__ uint2 pcol_load(const uint8_t *__restrict__ bed, int64_t I, int64_t Ib, int64_t j,
                                           bool valid, int64_t ic)
{
    uint32_t w[2] = {0x55555555u, 0x55555555u};
    if (valid) {
        const uint8_t *col = bed + (size_t)j * Ib;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int64_t bi = ic / 4 + u;
            uint32_t v = 0x55u;
            if (bi < Ib) {
                v = __ldg(col + bi);
                const int64_t nvalid = I - 4 * bi;            /* individuals of this byte below I */
                if (nvalid < 4) {
                    const uint32_t keep = (1u << (2 * (int)nvalid)) - 1u;
                    v = (v & keep) | (0x55u & ~keep);
                }
            }
            w[u >> 2] = (w[u >> 2] & ~(0xFFu << (8 * (u & 3)))) | (v << (8 * (u & 3)));
        }
    }
    return make_uint2(w[0], w[1]);
}

template <int K>
__global__ void __launch_bounds__(MP_THREADS)
k_sweep_p_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t Ib,
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
    float4 *tab = (float4 *)(sm + C::OFF_TAB);

    if (warp == 0) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        mbar_fence_init();
    }
    if (tid < 16) {
        const float A1[4] = {0.f, 0.f, 1.f, 2.f}, A2[4] = {2.f, 0.f, 1.f, 0.f};
        const int c0 = tid & 3, c1 = tid >> 2;
        tab[tid] = make_float4(A1[c0], A1[c1], A2[c0], A2[c1]);
    }
    /* q chunk staging: registers one chunk ahead, shared double buffer [k][i] */
    double qr[C::PREF_Q];
    auto qload = [&](int64_t ic) {
#pragma unroll
        for (int u = 0; u < C::PREF_Q; ++u) {
            const int t = tid + u * MP_THREADS;              /* t = ii * K + k */
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
                Qb[k * MP_IC + ii] = (float)qr[u];
            }
        }
    };
    uint2 gcur = make_uint2(0x55555555u, 0x55555555u), gnext = gcur;
    if (nchunk > 0) {
        qload(ia);
        qstore((float *)(sm + C::OFF_Q));
        gcur = pcol_load(bed, I, Ib, j, valid, ia);
    }
    if (nchunk > 1) {
        qload(ia + MP_IC);
        gnext = pcol_load(bed, I, Ib, j, valid, ia + MP_IC);
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
            if (!mbar_wait_bounded(&mbar[s], (uint32_t)(((c - 2) >> 1) & 1), MQ_WAIT_LIMIT)) {
                ok = false;
                if (tid == 0) atomicOr(err, 1);
            }
        }
        /* B tile: QQ[n][i] = q_ka(i) q_kb(i) in BF16, task (kc, nn) -> 16-byte row chunk */
        for (int t = tid; t < 4 * N; t += MP_THREADS) {
            const int kc = t / N, nn = t - kc * N;
            uint32_t w[4] = {0u, 0u, 0u, 0u};
            if (nn < T) {
                int ka, kb;
                tri_pair(nn, ka, kb);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int ii = kc * 8 + 2 * e;
                    w[e] = pack_bf16x2(Qb[ka * MP_IC + ii] * Qb[kb * MP_IC + ii],
                                       Qb[ka * MP_IC + ii + 1] * Qb[kb * MP_IC + ii + 1]);
                }
            }
            *(uint4 *)(Bt + kc * C::B_LBO + 16 * nn) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        const float2 *Q2 = (const float2 *)Qb;                  /* [k][pair] */
        float2 ga[K];
#pragma unroll
        for (int k = 0; k < K; ++k) ga[k] = make_float2(0.f, 0.f);
#pragma unroll
        for (int kc = 0; kc < 4; ++kc) {
            uint32_t cp[4];
            const uint32_t gw = kc < 2 ? gcur.x : gcur.y;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = kc * 4 + e;                       /* individuals 2m, 2m+1 of the chunk */
                const float4 a = tab[(gw >> (4 * (m & 7))) & 15u];
                float2 qp = make_float2(0.f, 0.f), om = make_float2(0.f, 0.f);
                float2 qv[K];
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    qv[k] = Q2[k * (MP_IC / 2) + m];
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
                gnext = pcol_load(bed, I, Ib, j, valid, icn);
            }
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0 && ok) {
            tc_fence_after_sync();
            const uint32_t abase = smem_u32(At), bbase = smem_u32(Bt);
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                const uint64_t ad = umma_desc_kmajor(abase + ks * 2 * C::A_LBO, C::A_LBO, C::A_SBO);
                const uint64_t bd = umma_desc_kmajor(bbase + ks * 2 * C::B_LBO, C::B_LBO, C::B_SBO);
                tc_mma_bf16(tmem, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
            }
            tc_commit(&mbar[s]);
        }
    }
    for (int c = max(0, nchunk - 2); c < nchunk; ++c) {
        const int s = c & 1;
        if (!mbar_wait_bounded(&mbar[s], (uint32_t)((c >> 1) & 1), ok ? MQ_WAIT_LIMIT : 1024u)) {
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
 *
 * loglikelihood_loop_skipmissing (loops.jl:517-539) with FP32 cells: thread = SNP, individuals
 * in pairs; each cell contributes the factor qp^g (1-qp)^(2-g) (1 when missing), two cells'
 * factors are multiplied in FP32 and folded into an FP64 running product whose exponent is
 * moved into an integer every 12 pairs; one FP64 log per thread at the end.  The products are
 * rounded to nearest, so the error is a random walk far below the convergence test's resolution.
 */
constexpr int ML_IC = 64;          /* individuals per chunk (16 genotype bytes per SNP) */

template <int K>
__global__ void __launch_bounds__(128)
k_loglik_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t Ib,
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
    /* inputs of the next chunk are loaded into registers while this one is consumed */
    float qr[PREF];
    uint2 gn[2];
    auto load = [&](int64_t ic) {
#pragma unroll
        for (int u = 0; u < PREF; ++u) {
            const int t = tid + u * 128;                 /* t = ii * K + k */
            const int ii = t / K;
            qr[u] = (t < K * ML_IC && ic + ii < ib) ? (float)q[(size_t)K * ic + t] : 1.0f / K;
        }
        gn[0] = pcol_load(bed, I, Ib, j, valid, ic);
        gn[1] = pcol_load(bed, I, Ib, j, valid, ic + 32);
    };
    auto store = [&](int s) {
#pragma unroll
        for (int u = 0; u < PREF; ++u) {
            const int t = tid + u * 128;
            if (t < K * ML_IC) {
                const int ii = t / K, k = t - ii * K;
                ((float *)Qs[s][k])[ii] = qr[u];
            }
        }
    };
    uint2 g[2] = {make_uint2(0x55555555u, 0x55555555u), make_uint2(0x55555555u, 0x55555555u)};
    if (nchunk > 0) { load(ia); store(0); g[0] = gn[0]; g[1] = gn[1]; }
    if (nchunk > 1) load(ia + ML_IC);
    __syncthreads();
    double prod = 1.0;
    int64_t ex = 0;
    for (int c = 0; c < nchunk; ++c) {
        const int s = c & 1;
#pragma unroll
        for (int m = 0; m < ML_IC / 2; ++m) {
            const uint32_t word = (m < 16) ? ((m < 8) ? g[0].x : g[0].y) : ((m < 24) ? g[1].x : g[1].y);
            const uint32_t code4 = (word >> (4 * (m & 7))) & 15u;
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
            g[0] = gn[0]; g[1] = gn[1];
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
cudaError_t launch_p_mixed_t(const uint8_t *bed, int64_t I, int64_t J, const double *q, const double *p,
                             const SweepPlan &pl, double *out, int *err, cudaStream_t st)
{
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_sweep_p_mixed<K><<<grid, MP_THREADS, MP<K>::SMEM, st>>>(bed, I, J, (I + 3) / 4, q, p, pl.slice, out, err);
    return cudaGetLastError();
}

template <int K>
cudaError_t launch_ll_mixed_t(const uint8_t *bed, int64_t I, int64_t J, const double *q, const double *p,
                              const SweepPlan &pl, double *partial, double *out, cudaStream_t st)
{
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_loglik_mixed<K><<<grid, 128, 0, st>>>(bed, I, J, (I + 3) / 4, q, p, pl.slice, partial);
    k_sum_partials_mixed<<<1, 1024, 0, st>>>(partial, (int64_t)pl.gx * pl.S, out);
    return cudaGetLastError();
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

/* One CTA per 128 SNPs and individual slice (slices are multiples of 32 individuals). */
SweepPlan plan_sweep_p_mixed(int K, int64_t I, int64_t J, int sms)
{
    (void)K;
    SweepPlan pl;
    pl.gx = (int)((J + 127) / 128);
    const int64_t target = (int64_t)sms * 4;
    int64_t S = (target + pl.gx - 1) / pl.gx;
    S = std::max<int64_t>(1, std::min<int64_t>(S, (I + 255) / 256));
    int64_t slice = (I + S - 1) / S;
    slice = (slice + 31) / 32 * 32;
    pl.slice = slice;
    pl.S = (int)((I + slice - 1) / slice);
    return pl;
}

cudaError_t launch_sweep_p_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, const double *q,
                                 const double *p, const SweepPlan &pl, double *out, int *err,
                                 cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_p_mixed_t<KK>(bed, I, J, q, p, pl, out, err, st));
    return e;
}

SweepPlan plan_loglik_mixed(int64_t I, int64_t J, int sms)
{
    SweepPlan pl;
    pl.gx = (int)((J + 127) / 128);
    const int64_t target = (int64_t)sms * 8;
    int64_t S = (target + pl.gx - 1) / pl.gx;
    S = std::max<int64_t>(1, std::min<int64_t>(S, (I + 255) / 256));
    int64_t slice = (I + S - 1) / S;
    slice = (slice + 63) / 64 * 64;
    pl.slice = slice;
    pl.S = (int)((I + slice - 1) / slice);
    return pl;
}

cudaError_t launch_loglik_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, const double *q,
                                const double *p, const SweepPlan &pl, double *partial, double *out,
                                cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_ll_mixed_t<KK>(bed, I, J, q, p, pl, partial, out, st));
    return e;
}
