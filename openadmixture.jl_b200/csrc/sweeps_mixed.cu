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
 * The K-term dot products qp = sum_k q_k p_k and sum_k q_k (1-p_k) of every cell also run on the
 * tensor cores (TF32 split products); 1 - qp is that second sum plus 1 - sum_k q_k, which is the
 * reference's 1 - qp for any Q.  CUDA cores turn each cell into one reciprocal, the BF16 weights
 * of the Hessian GEMM and the FP32 gradient terms (summed into FP64 per chunk).  The epilogue
 * reads the accumulator with tcgen05.ld and writes the FP64 partial layout of the FP64 sweeps,
 * so the QP kernels consume either.
 *
 * Genotypes are read from the handle's padded layout: columns at a pitch that is a multiple of
 * 16 bytes, padding bytes and padding bits coded missing (01), so whole 16-byte groups can be
 * loaded without per-individual bound checks.
 */
#include "common.cuh"
#include "kernels.h"
#include "tc05.cuh"

namespace {

constexpr uint32_t MX_WAIT_LIMIT = 1u << 22;   /* polls; an MMA batch completes in microseconds */
/* Hessian accumulation blocks: every MX_HBLOCK chunks the FP32 TMEM accumulator is drained into
 * the row's FP64 partials and the next MMA starts a fresh sum, so no FP32 partial sum sees more
 * than 4 * MX_HBLOCK MMA accumulations (whose rounding is not to nearest) whatever J or I is. */
constexpr int MX_HBLOCK = 256;

/* add (or, for the first block, store) TMEM columns col .. col+N-1 of this thread's lane into the
 * FP64 Hessian entries o[0 .. T-1] */
template <int N, int T>
__device__ __forceinline__ void hess_drain(uint32_t taddr, double *o, bool first, bool valid)
{
#pragma unroll 1
    for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        tmem_ld16(taddr + (uint32_t)c0, v);
        if (valid) {
#pragma unroll
            for (int e = 0; e < 16; ++e)
                if (c0 + e < T) o[c0 + e] = first ? (double)v[e] : o[c0 + e] + (double)v[e];
        }
    }
}

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

/* ===================================================================== Q side
 *
 * Per 32-SNP chunk, two tensor-core products:
 *   qp / om    D[128 x 64] = Qtile * [p ; 1-p]^T in TF32 split form (hi*hi + lo*hi + hi*lo, about
 *              2^-21 relative): the K-term dot products of every (individual, SNP) cell;
 *   Hessian    D[128 x N] += [w1 | w2] * [PP ; PbarPbar]^T in BF16 (FP32 accumulation);
 * and on the CUDA cores, per cell: the code lookup, one reciprocal, z1, z2, w1, w2 and the FP32
 * gradient sum_j (z1 - z2) p_k + z2 (= sum_j z1 p_k + z2 (1 - p_k)), added into FP64 per chunk.
 *
 * Everything that depends on P alone -- the BF16 pair-product tiles, the TF32 hi / lo split of
 * [p ; 1-p] and p in FP32 -- is built once per sweep by k_q_pack, one "package" per chunk laid
 * out exactly as the sweep's shared memory wants it, and fetched by each CTA with one bulk
 * asynchronous copy (three package buffers in flight).  The qp MMA of chunk c+1 runs while the
 * CUDA cores work on chunk c. */

constexpr int MQ_JC = 32;          /* SNPs per chunk = 2 BF16 MMA K-steps */
constexpr int MQ_THREADS = 128;    /* one thread per individual = accumulator row */
constexpr int MQ_NPKG = 3;         /* package buffers */

template <int K>
struct MQ {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + 15) / 16) * 16;              /* Hessian MMA N (multiple of 16 for M = 128) */
    static constexpr int KP = ((K + 7) / 8) * 8;                /* TF32 K extent of the qp MMAs */
    static constexpr int QPN = 2 * MQ_JC;                       /* qp MMA N: the chunk's p rows, then 1-p rows */
    static constexpr uint32_t COL_H = 64;                       /* TMEM column of the Hessian accumulator */
    static constexpr uint32_t NCOLS = tmem_cols_for(COL_H + N);
    static constexpr int E = T + K;                             /* partial entries per individual */
    static constexpr uint32_t A_BYTES = 128 * MQ_JC * 2;        /* one BF16 weight tile: 8 KB */
    static constexpr uint32_t B_BYTES = N * MQ_JC * 2;          /* one BF16 pair-product tile */
    static constexpr uint32_t QA_BYTES = 128 * 2 * KP * 4;      /* TF32 Q tile [hi | lo] */
    static constexpr uint32_t QB_BYTES = QPN * 2 * KP * 4;      /* TF32 [p ; 1-p] chunk [hi | lo] */
    static constexpr int PS = MQ_JC + 4;                        /* FP32 p row stride (floats, 16-byte rows) */
    /* package of one chunk: [PP tile | PbarPbar tile | TF32 [p ; 1-p] | FP32 p [k][jj]] */
    static constexpr uint32_t PK_QB = 2 * B_BYTES;
    static constexpr uint32_t PK_PF = PK_QB + QB_BYTES;
    static constexpr uint32_t PKG = PK_PF + K * PS * 4;
    static constexpr uint32_t GBUF = MQ_JC * 32;                /* genotype bytes of one chunk */
    static constexpr uint32_t OFF_A = 0;                        /* W1 tile, then W2 tile */
    static constexpr uint32_t OFF_PKG = 2 * A_BYTES;
    static constexpr uint32_t OFF_QA = OFF_PKG + MQ_NPKG * PKG;
    static constexpr uint32_t OFF_G = OFF_QA + QA_BYTES;        /* two G buffers, [pair][byte][2] */
    static constexpr uint32_t OFF_TAB = OFF_G + 2 * GBUF;       /* float4 [16][8] code table */
    static constexpr uint32_t SMEM = OFF_TAB + 128 * 16 + 1024; /* + alignment slack */
    /* core matrices (8 rows x 16 B): BF16 A 128 B apart along M, 2048 B along K; BF16 B 128 B
     * along N, 16 N bytes along K; TF32 Q tile 128 B along M, 2048 B along K; TF32 [p ; 1-p]
     * 128 B along N, 1024 B along K */
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr uint32_t QA_LBO = 2048, QB_LBO = 1024, Q_SBO = 128;
    static_assert(PKG % 16 == 0 && OFF_QA % 16 == 0, "bulk copies and descriptors need 16-byte alignment");
};

/* byte offset of element (row r, 4-byte column f) in a K-major no-swizzle tile */
__device__ __forceinline__ uint32_t kmaj_off(int r, int f, uint32_t lbo)
{
    return (uint32_t)(f >> 2) * lbo + (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u + (uint32_t)(f & 3) * 4u;
}

/* One package per 32-SNP chunk of the whole SNP range (block = chunk).  SNPs beyond J get
 * p = 0.5; their genotypes read as missing, so they contribute nothing. */
template <int K>
__global__ void __launch_bounds__(128)
k_q_pack(const double *__restrict__ p, int64_t J, uint8_t *__restrict__ pkg)
{
    using C = MQ<K>;
    constexpr int T = C::T, N = C::N;
    __shared__ __align__(16) float pf[2 * K * C::PS];          /* p, then 1-p: [term][k][jj] */
    __shared__ __align__(16) uint8_t buf[C::PKG];
    const int tid = threadIdx.x;
    const int64_t jc = (int64_t)blockIdx.x * MQ_JC;
    for (uint32_t t = tid; t < C::PKG / 16; t += 128) ((uint4 *)buf)[t] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    for (int t = tid; t < K * MQ_JC; t += 128) {
        const int jj = t / K, k = t - jj * K;
        const double pd = (jc + jj < J) ? p[(size_t)K * jc + t] : 0.5;
        const float a = (float)pd, b = (float)(1.0 - pd);
        pf[k * C::PS + jj] = a;
        pf[K * C::PS + k * C::PS + jj] = b;
        ((float *)(buf + C::PK_PF))[k * C::PS + jj] = a;
        float h, l;
        tf32_split(a, h, l);
        *(float *)(buf + C::PK_QB + kmaj_off(jj, k, C::QB_LBO)) = h;
        *(float *)(buf + C::PK_QB + kmaj_off(jj, C::KP + k, C::QB_LBO)) = l;
        tf32_split(b, h, l);
        *(float *)(buf + C::PK_QB + kmaj_off(MQ_JC + jj, k, C::QB_LBO)) = h;
        *(float *)(buf + C::PK_QB + kmaj_off(MQ_JC + jj, C::KP + k, C::QB_LBO)) = l;
    }
    __syncthreads();
    /* pair-product tiles: task (term, kc, nn) writes pair nn's 8 SNPs of k-chunk kc at kc*16N + 16nn */
    for (int t = tid; t < 2 * 4 * N; t += 128) {
        const int term = t / (4 * N), rem = t - term * 4 * N;
        const int kc = rem / N, nn = rem - kc * N;
        uint32_t w[4] = {0u, 0u, 0u, 0u};
        if (nn < T) {
            int ka, kb;
            tri_pair(nn, ka, kb);
            const float *src = pf + term * K * C::PS + kc * 8;
            const float4 a0 = *(const float4 *)(src + ka * C::PS), a1 = *(const float4 *)(src + ka * C::PS + 4);
            const float4 b0 = *(const float4 *)(src + kb * C::PS), b1 = *(const float4 *)(src + kb * C::PS + 4);
            w[0] = pack_bf16x2(a0.x * b0.x, a0.y * b0.y);
            w[1] = pack_bf16x2(a0.z * b0.z, a0.w * b0.w);
            w[2] = pack_bf16x2(a1.x * b1.x, a1.y * b1.y);
            w[3] = pack_bf16x2(a1.z * b1.z, a1.w * b1.w);
        }
        *(uint4 *)(buf + term * C::B_BYTES + kc * C::B_LBO + 16 * nn) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    __syncthreads();
    uint4 *dst = (uint4 *)(pkg + (size_t)blockIdx.x * C::PKG);
    for (uint32_t t = tid; t < C::PKG / 16; t += 128) dst[t] = ((const uint4 *)buf)[t];
}

/* qp / om of the package's chunk into TMEM columns 0..63: 3 * KP/8 TF32 MMAs (one thread) */
template <int K>
__device__ __forceinline__ void issue_qp(uint32_t tmem, const uint8_t *sm, const uint8_t *pk)
{
    using C = MQ<K>;
    const uint32_t a = smem_u32(sm + C::OFF_QA), b = smem_u32(pk + C::PK_QB);
    constexpr uint32_t id = idesc_tf32_f32(128, C::QPN);
    constexpr uint32_t alo = (C::KP / 4) * C::QA_LBO, blo = (C::KP / 4) * C::QB_LBO;
#pragma unroll
    for (int s = 0; s < C::KP / 8; ++s) {
        const uint32_t ao = a + s * 2 * C::QA_LBO, bo = b + s * 2 * C::QB_LBO;
        const uint64_t ahi = umma_desc_kmajor(ao, C::QA_LBO, C::Q_SBO);
        const uint64_t alw = umma_desc_kmajor(ao + alo, C::QA_LBO, C::Q_SBO);
        const uint64_t bhi = umma_desc_kmajor(bo, C::QB_LBO, C::Q_SBO);
        const uint64_t blw = umma_desc_kmajor(bo + blo, C::QB_LBO, C::Q_SBO);
        tc_mma_tf32(tmem, ahi, bhi, id, s > 0 ? 1u : 0u);
        tc_mma_tf32(tmem, alw, bhi, id, 1u);
        tc_mma_tf32(tmem, ahi, blw, id, 1u);
    }
}

/* Warp roles: warps 0-3 are producers (thread = accumulator row), warp 4 is the controller
 * (bulk copies, genotype staging, MMA issue).  No CTA-wide barrier inside the chunk loop: the
 * roles hand off through mbarriers.  Every wait is bounded; after a failed wait a thread sets
 * the shared abort flag and both roles run to the end without waiting. */
constexpr int MQ_CTA = MQ_THREADS + 32;

template <int K>
__global__ void __launch_bounds__(MQ_CTA, (K <= 10 ? 3 : (K <= 12 ? 2 : 1)))
k_sweep_q_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
                const double *__restrict__ q, const uint8_t *__restrict__ pkg, int64_t jslice,
                double *__restrict__ out, int *__restrict__ err)
{
    using C = MQ<K>;
    constexpr int T = C::T, N = C::N, E = C::E;
    extern __shared__ __align__(1024) uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    /* qp ready, qp consumed (4 warps), A tile written (4 warps), Hessian done, G staged [2], package [3] */
    __shared__ uint64_t mbar[6 + MQ_NPKG];
    __shared__ uint32_t tmem_holder;
    __shared__ volatile int abort_flag;
    uint64_t *bar_qp = &mbar[0], *bar_qfree = &mbar[1], *bar_afull = &mbar[2], *bar_h = &mbar[3];
    uint64_t *bar_g = &mbar[4], *bar_p = &mbar[6];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp < 4;
    const int64_t i0 = (int64_t)blockIdx.x * 128;
    const int64_t i = i0 + tid;
    const bool valid = producer && i < I;
    const int64_t j0 = (int64_t)blockIdx.y * jslice;    /* jslice is a multiple of MQ_JC */
    const int64_t j1 = min(J, j0 + jslice);
    const int nchunk = (int)((j1 - j0 + MQ_JC - 1) / MQ_JC);
    const uint8_t *pk0 = pkg + (size_t)(j0 / MQ_JC) * C::PKG;
    uint8_t *At = sm + C::OFF_A;

    if (warp == 4) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        mbar_init(bar_qp, 1);
        mbar_init(bar_qfree, 4);
        mbar_init(bar_afull, 4);
        mbar_init(bar_h, 1);
        mbar_init(&bar_g[0], 1);
        mbar_init(&bar_g[1], 1);
        for (int b = 0; b < MQ_NPKG; ++b) mbar_init(&bar_p[b], 1);
        abort_flag = 0;
        mbar_fence_init();
    }
    code_table_init((float4 *)(sm + C::OFF_TAB), tid, MQ_CTA);
    if (producer) {   /* this thread's row of the TF32 Q tile: columns 0..K-1 hi, KP..KP+K-1 lo */
        float hv[C::KP], lv[C::KP];
#pragma unroll
        for (int k = 0; k < C::KP; ++k) {
            hv[k] = 0.f; lv[k] = 0.f;
            if (k < K) tf32_split(valid ? (float)q[(size_t)K * i + k] : 1.0f / K, hv[k], lv[k]);
        }
#pragma unroll
        for (int f = 0; f < C::KP; f += 4) {
            *(float4 *)(sm + C::OFF_QA + kmaj_off(tid, f, C::QA_LBO)) = make_float4(hv[f], hv[f + 1], hv[f + 2], hv[f + 3]);
            *(float4 *)(sm + C::OFF_QA + kmaj_off(tid, C::KP + f, C::QA_LBO)) = make_float4(lv[f], lv[f + 1], lv[f + 2], lv[f + 3]);
        }
    }
    fence_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_holder;
    bool ok = true;
    auto wait = [&](uint64_t *b, uint32_t parity) -> bool {
        if (!ok) return false;
        for (uint32_t n = 0; n < MX_WAIT_LIMIT; ++n) {
            if (mbar_try_wait(b, parity)) return true;
            if ((n & 255u) == 255u && abort_flag) break;
        }
        ok = false;
        abort_flag = 1;
        atomicOr(err, 1);
        return false;
    };

    if (!producer) {
        /* ---------------------------------------------------------------- controller warp */
        const bool leader = lane == 0;
        /* genotypes of chunk c into G buffer c & 1: lane l loads SNP jc + l (32 bytes: the CTA's 128
         * individuals); lanes 2m, 2m+1 exchange and write pair m interleaved as [byte][2] */
        auto stage_g = [&](int c) {
            const int64_t jc = j0 + (int64_t)c * MQ_JC;
            uint4 a0 = make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u), a1 = a0;
            if (jc + lane < j1) {
                const uint4 *src = (const uint4 *)(bed + (size_t)(jc + lane) * pitch + (size_t)(i0 / 4));
                a0 = __ldg(src);
                a1 = __ldg(src + 1);
            }
            uint4 b0, b1;                                   /* the partner lane's bytes */
            b0.x = __shfl_xor_sync(0xffffffffu, a0.x, 1); b0.y = __shfl_xor_sync(0xffffffffu, a0.y, 1);
            b0.z = __shfl_xor_sync(0xffffffffu, a0.z, 1); b0.w = __shfl_xor_sync(0xffffffffu, a0.w, 1);
            b1.x = __shfl_xor_sync(0xffffffffu, a1.x, 1); b1.y = __shfl_xor_sync(0xffffffffu, a1.y, 1);
            b1.z = __shfl_xor_sync(0xffffffffu, a1.z, 1); b1.w = __shfl_xor_sync(0xffffffffu, a1.w, 1);
            const bool even = (lane & 1) == 0;
            /* even lane: bytes 0..15 of (own, partner); odd lane: bytes 16..31 of (partner, own) */
            const uint4 s0 = even ? a0 : b1, s1 = even ? b0 : a1;   /* SNP 2m bytes, SNP 2m+1 bytes */
            uint8_t *Gb = sm + C::OFF_G + (c & 1) * C::GBUF + (lane >> 1) * 64 + (even ? 0 : 32);
            *(uint4 *)(Gb) = interleave8(make_uint2(s0.x, s0.y), make_uint2(s1.x, s1.y));
            *(uint4 *)(Gb + 16) = interleave8(make_uint2(s0.z, s0.w), make_uint2(s1.z, s1.w));
            __syncwarp();
            if (leader) mbar_arrive(&bar_g[c & 1]);
        };
        auto copy_pkg = [&](int c) {
            if (leader) {
                mbar_arrive_expect_tx(&bar_p[c % MQ_NPKG], C::PKG);
                bulk_g2s(sm + C::OFF_PKG + (c % MQ_NPKG) * C::PKG, pk0 + (size_t)c * C::PKG, C::PKG,
                         &bar_p[c % MQ_NPKG]);
            }
        };
        for (int c = 0; c < min(nchunk, MQ_NPKG); ++c) copy_pkg(c);
        if (nchunk > 0) stage_g(0);
        if (nchunk > 1) stage_g(1);
        if (nchunk > 0 && wait(&bar_p[0], 0u) && leader) {
            tc_fence_after_sync();
            issue_qp<K>(tmem, sm, sm + C::OFF_PKG);
            tc_commit(bar_qp);
        }
        constexpr uint32_t idesc = idesc_bf16_f32(128, N);
        for (int c = 0; c < nchunk && ok; ++c) {
            /* qp of chunk c+1 once its package landed and the producers read qp of chunk c */
            if (c + 1 < nchunk) {
                const int cn = c + 1;
                const bool landed = wait(&bar_p[cn % MQ_NPKG], (uint32_t)((cn / MQ_NPKG) & 1));
                if (landed && wait(bar_qfree, (uint32_t)(c & 1)) && leader) {
                    tc_fence_after_sync();
                    issue_qp<K>(tmem, sm, sm + C::OFF_PKG + (cn % MQ_NPKG) * C::PKG);
                    tc_commit(bar_qp);
                }
            }
            /* Hessian of chunk c once the producers wrote its weight tile */
            if (wait(bar_afull, (uint32_t)(c & 1))) {
                if (leader) {
                    tc_fence_after_sync();
                    const uint8_t *pk = sm + C::OFF_PKG + (c % MQ_NPKG) * C::PKG;
                    const uint32_t abase = smem_u32(At), bbase = smem_u32(pk);
#pragma unroll
                    for (int term = 0; term < 2; ++term) {
#pragma unroll
                        for (int ks = 0; ks < 2; ++ks) {
                            const uint64_t ad = umma_desc_kmajor(abase + term * C::A_BYTES + ks * 2 * C::A_LBO, C::A_LBO, C::A_SBO);
                            const uint64_t bd = umma_desc_kmajor(bbase + term * C::B_BYTES + ks * 2 * C::B_LBO, C::B_LBO, C::B_SBO);
                            tc_mma_bf16(tmem + C::COL_H, ad, bd, idesc, (c % MX_HBLOCK != 0 || term > 0 || ks > 0) ? 1u : 0u);
                        }
                    }
                    tc_commit(bar_h);
                }
                /* the producers are done with G buffer c & 1: stage chunk c+2 into it */
                if (c + 2 < nchunk) stage_g(c + 2);
            }
            /* package c is free once the Hessian of chunk c is done: fetch chunk c+3 into it */
            if (c + MQ_NPKG < nchunk && wait(bar_h, (uint32_t)(c & 1))) {
                fence_async_smem();
                copy_pkg(c + MQ_NPKG);
            }
        }
    } else {
        /* ---------------------------------------------------------------- producer warps */
        const float4 *tab = (const float4 *)(sm + C::OFF_TAB) + (tid & 7);
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        const int sh = valid ? (int)(i & 3) * 2 : 0;
        const uint32_t gmask = valid ? 0xFFFFu : 0u;    /* rows beyond I read code pair 01|01 */
        /* 1 - qp = sum_k q_k (1 - p_k) + (1 - sum_k q_k): exact for any Q (the reference forms 1 - qp;
         * EM priming leaves sum_k q_k < 1 where genotypes are missing) */
        float sres = 0.f;
        if (valid) {
            double sq = 0.0;
#pragma unroll
            for (int k = 0; k < K; ++k) sq += q[(size_t)K * i + k];
            sres = (float)(1.0 - sq);
        }
        const float2 sres2 = make_float2(sres, sres);
        double gd[K];
#pragma unroll
        for (int k = 0; k < K; ++k) gd[k] = 0.0;
        for (int c = 0; c < nchunk && ok; ++c) {
            const uint8_t *pk = sm + C::OFF_PKG + (c % MQ_NPKG) * C::PKG;
            const float *Pf = (const float *)(pk + C::PK_PF);
            const uint8_t *Gb = sm + C::OFF_G + (c & 1) * C::GBUF;
            /* qp / om of the chunk's 32 SNPs, read in two halves of 16 columns (SNPs 0-15, then
             * 16-31) to keep the producer within its registers */
            uint32_t rq[16], ro[16];
            if (!wait(bar_qp, (uint32_t)(c & 1))) break;
            tc_fence_after_sync();
            tmem_ld16_raw(tmem + lane_base, rq);
            tmem_ld16_raw(tmem + lane_base + 32u, ro);
            tmem_wait_ld();
            if (!wait(&bar_p[c % MQ_NPKG], (uint32_t)((c / MQ_NPKG) & 1))) break;
            if (!wait(&bar_g[c & 1], (uint32_t)((c >> 1) & 1))) break;
            if (c > 0 && !wait(bar_h, (uint32_t)((c - 1) & 1))) break;   /* the weight tile is free */
            if (c > 0 && c % MX_HBLOCK == 0) {   /* drain the block of chunks c-MX_HBLOCK .. c-1 */
                tc_fence_after_sync();
                hess_drain<N, T>(tmem + lane_base + C::COL_H, out + ((size_t)blockIdx.y * I + (valid ? i : 0)) * E,
                                 c == MX_HBLOCK, valid);
                tc_fence_before_sync();
            }
            const uint16_t *G2 = (const uint16_t *)Gb + (tid >> 2);
            float2 gk[K], zs = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < K; ++k) gk[k] = make_float2(0.f, 0.f);
#pragma unroll
            for (int kc = 0; kc < 4; ++kc) {
                if (kc == 2) {   /* the second half of the columns; then the qp columns are free */
                    tc_fence_after_sync();
                    tmem_ld16_raw(tmem + lane_base + 16u, rq);
                    tmem_ld16_raw(tmem + lane_base + 48u, ro);
                    tmem_wait_ld();
                    tc_fence_before_sync();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(bar_qfree);
                }
                uint32_t w1p[4], w2p[4];
                float2 dz[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int m = kc * 4 + e;
                    const int r = 2 * (m & 7);   /* this pair's column in rq / ro */
                    const uint32_t gw = ((uint32_t)G2[m * 32] & gmask) | (~gmask & 0x5555u);
                    const uint32_t tb = gw >> sh;
                    const float4 a = tab[8 * ((tb & 3u) | ((tb >> 6) & 12u))];
                    const float2 qp = make_float2(__uint_as_float(rq[r]), __uint_as_float(rq[r + 1]));
                    const float2 om = __fadd2_rn(make_float2(__uint_as_float(ro[r]), __uint_as_float(ro[r + 1])), sres2);
                    const float2 pr = __fmul2_rn(qp, om);
                    const float2 rr = make_float2(rcp_approx(pr.x), rcp_approx(pr.y));
                    const float2 r1 = __fmul2_rn(om, rr), r2 = __fmul2_rn(qp, rr);
                    const float2 z1 = __fmul2_rn(make_float2(a.x, a.y), r1);
                    const float2 z2 = __fmul2_rn(make_float2(a.z, a.w), r2);
                    const float2 w1 = __fmul2_rn(z1, r1), w2 = __fmul2_rn(z2, r2);
                    dz[e] = make_float2(z1.x - z2.x, z1.y - z2.y);
                    zs = __fadd2_rn(zs, z2);
                    w1p[e] = pack_bf16x2(w1.x, w1.y);
                    w2p[e] = pack_bf16x2(w2.x, w2.y);
                }
                *(uint4 *)(At + kc * C::A_LBO + 16 * tid) = make_uint4(w1p[0], w1p[1], w1p[2], w1p[3]);
                *(uint4 *)(At + C::A_BYTES + kc * C::A_LBO + 16 * tid) = make_uint4(w2p[0], w2p[1], w2p[2], w2p[3]);
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float4 p0 = *(const float4 *)(Pf + k * C::PS + kc * 8);
                    const float4 p1 = *(const float4 *)(Pf + k * C::PS + kc * 8 + 4);
                    gk[k] = __ffma2_rn(dz[0], make_float2(p0.x, p0.y), gk[k]);
                    gk[k] = __ffma2_rn(dz[1], make_float2(p0.z, p0.w), gk[k]);
                    gk[k] = __ffma2_rn(dz[2], make_float2(p1.x, p1.y), gk[k]);
                    gk[k] = __ffma2_rn(dz[3], make_float2(p1.z, p1.w), gk[k]);
                }
            }
            const double zsum = (double)zs.x + (double)zs.y;
#pragma unroll
            for (int k = 0; k < K; ++k) gd[k] += (double)gk[k].x + (double)gk[k].y + zsum;
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_afull);
        }
        if (nchunk > 0) wait(bar_h, (uint32_t)((nchunk - 1) & 1));   /* the last Hessian MMAs */
        if (valid) {
            double *o = out + ((size_t)blockIdx.y * I + i) * E;
#pragma unroll
            for (int k = 0; k < K; ++k) o[T + k] = gd[k];
        }
    }
    /* every role is past its loop; after a failure, give MMAs and copies still in flight a
     * bounded moment before the TMEM is read and released */
    ok = __syncthreads_and(ok);
    if (!ok && tid == MQ_THREADS) {
        mbar_wait_bounded(bar_h, 0u, 1024u);
        mbar_wait_bounded(bar_h, 1u, 1024u);
        mbar_wait_bounded(bar_qp, 0u, 1024u);
        mbar_wait_bounded(bar_qp, 1u, 1024u);
        for (int b = 0; b < MQ_NPKG; ++b) { mbar_wait_bounded(&bar_p[b], 0u, 1024u); mbar_wait_bounded(&bar_p[b], 1u, 1024u); }
    }
    __syncthreads();
    tc_fence_after_sync();
    if (producer) {
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        if (nchunk > 0) {
#pragma unroll 1
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + lane_base + C::COL_H + (uint32_t)c0, v);
                if (valid) {   /* the last accumulation block, added to the drained ones */
                    double *o = out + ((size_t)blockIdx.y * I + i) * E;
                    const bool first = nchunk <= MX_HBLOCK;
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        if (c0 + e < T)
                            o[c0 + e] = ok ? (first ? (double)v[e] : o[c0 + e] + (double)v[e])
                                           : __longlong_as_double(0x7ff8000000000000LL);
                }
            }
        } else if (valid) {
            double *o = out + ((size_t)blockIdx.y * I + i) * E;
            for (int e = 0; e < T; ++e) o[e] = 0.0;
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 4) tmem_dealloc_warp(tmem, C::NCOLS);
}

/* ===================================================================== P side
 *
 * Mirror of the Q side with the roles of the axes swapped: rows = 128 SNPs, reduction over
 * chunks of 32 individuals.  Per chunk:
 *   qp, om     D[128 x 32] = Ptile * Qchunk^T and (1-P)tile * Qchunk^T, TF32 split form;
 *   Hessian    D[128 x N] += C * QQ^T in BF16, C = nm (g/qp^2 + (2-g)/(1-qp)^2);
 * and per cell on the CUDA cores the code (from the thread's own genotype word), one reciprocal
 * and the FP32 gradient sum_i nm (g/qp - (2-g)/(1-qp)) q_k, added into FP64 per chunk.  The
 * Q-derived tiles of each chunk (QQ in BF16, Q split into TF32 hi / lo, q in FP32) are built
 * once per sweep by k_p_pack and fetched with one bulk copy per chunk. */

constexpr int MP_IC = 32;          /* individuals per chunk = 2 BF16 MMA K-steps */
constexpr int MP_THREADS = 128;    /* one thread per SNP = accumulator row */
constexpr int MP_NPKG = 3;

template <int K>
struct MP {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + 15) / 16) * 16;
    static constexpr int KP = ((K + 7) / 8) * 8;
    static constexpr uint32_t COL_OM = 32, COL_H = 64;          /* TMEM: qp 0..31, om 32..63, Hessian */
    static constexpr uint32_t NCOLS = tmem_cols_for(COL_H + N);
    static constexpr int E = T + K;
    static constexpr uint32_t A_BYTES = 128 * MP_IC * 2;        /* BF16 C tile: 8 KB */
    static constexpr uint32_t B_BYTES = N * MP_IC * 2;          /* BF16 QQ tile */
    static constexpr uint32_t PA_BYTES = 128 * 2 * KP * 4;      /* TF32 P tile [hi | lo] (and 1-P) */
    static constexpr uint32_t QB_BYTES = MP_IC * 2 * KP * 4;    /* TF32 Q chunk [hi | lo] */
    static constexpr int QS = MP_IC + 4;                        /* FP32 q row stride (floats) */
    static constexpr uint32_t PK_QB = B_BYTES;
    static constexpr uint32_t PK_QF = PK_QB + QB_BYTES;
    static constexpr uint32_t PK_S = PK_QF + K * QS * 4;         /* 1 - sum_k q_k per individual */
    static constexpr uint32_t PKG = PK_S + MP_IC * 4;
    static constexpr uint32_t OFF_A = 0;
    static constexpr uint32_t OFF_PKG = A_BYTES;
    static constexpr uint32_t OFF_PA = OFF_PKG + MP_NPKG * PKG; /* P tile, then (1-P) tile */
    static constexpr uint32_t OFF_TAB = OFF_PA + 2 * PA_BYTES;
    static constexpr uint32_t SMEM = OFF_TAB + 128 * 16 + 1024;
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr uint32_t PA_LBO = 2048, QB_LBO = 512, T_SBO = 128;
    static_assert(PKG % 16 == 0 && OFF_PA % 16 == 0, "bulk copies and descriptors need 16-byte alignment");
};

/* One package per 32-individual chunk of the whole individual range (block = chunk).
 * Individuals beyond I get q = 1/K; their genotype codes read as missing. */
template <int K>
__global__ void __launch_bounds__(128)
k_p_pack(const double *__restrict__ q, int64_t I, uint8_t *__restrict__ pkg)
{
    using C = MP<K>;
    constexpr int T = C::T, N = C::N;
    __shared__ __align__(16) uint8_t buf[C::PKG];
    const int tid = threadIdx.x;
    const int64_t ic = (int64_t)blockIdx.x * MP_IC;
    float *qf = (float *)(buf + C::PK_QF);
    for (uint32_t t = tid; t < C::PKG / 16; t += 128) ((uint4 *)buf)[t] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    if (tid < MP_IC) {   /* 1 - qp = sum_k q_k (1 - p_k) + (1 - sum_k q_k), exact for any Q */
        double sq = 1.0;
        if (ic + tid < I) {
            sq = 0.0;
            for (int k = 0; k < K; ++k) sq += q[(size_t)K * (ic + tid) + k];
        }
        ((float *)(buf + C::PK_S))[tid] = (float)(1.0 - sq);
    }
    for (int t = tid; t < K * MP_IC; t += 128) {
        const int ii = t / K, k = t - ii * K;
        const float a = (ic + ii < I) ? (float)q[(size_t)K * ic + t] : 1.0f / K;
        qf[k * C::QS + ii] = a;
        float h, l;
        tf32_split(a, h, l);
        *(float *)(buf + C::PK_QB + kmaj_off(ii, k, C::QB_LBO)) = h;
        *(float *)(buf + C::PK_QB + kmaj_off(ii, C::KP + k, C::QB_LBO)) = l;
    }
    __syncthreads();
    /* QQ tile: task (kc, nn) writes pair nn's 8 individuals of k-chunk kc at kc*16N + 16nn */
    for (int t = tid; t < 4 * N; t += 128) {
        const int kc = t / N, nn = t - kc * N;
        uint32_t w[4] = {0u, 0u, 0u, 0u};
        if (nn < T) {
            int ka, kb;
            tri_pair(nn, ka, kb);
            const float *src = qf + kc * 8;
            const float4 a0 = *(const float4 *)(src + ka * C::QS), a1 = *(const float4 *)(src + ka * C::QS + 4);
            const float4 b0 = *(const float4 *)(src + kb * C::QS), b1 = *(const float4 *)(src + kb * C::QS + 4);
            w[0] = pack_bf16x2(a0.x * b0.x, a0.y * b0.y);
            w[1] = pack_bf16x2(a0.z * b0.z, a0.w * b0.w);
            w[2] = pack_bf16x2(a1.x * b1.x, a1.y * b1.y);
            w[3] = pack_bf16x2(a1.z * b1.z, a1.w * b1.w);
        }
        *(uint4 *)(buf + kc * C::B_LBO + 16 * nn) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    __syncthreads();
    uint4 *dst = (uint4 *)(pkg + (size_t)blockIdx.x * C::PKG);
    for (uint32_t t = tid; t < C::PKG / 16; t += 128) dst[t] = ((const uint4 *)buf)[t];
}

/* qp (TMEM columns 0..31) and om (32..63) of a chunk: 2 * 3 * KP/8 TF32 MMAs of the P tile (the
 * (1-P) tile follows at +PA_BYTES) with the chunk's TF32 Q tile */
template <int K>
__device__ __forceinline__ void issue_qp_p(uint32_t tmem, const uint8_t *pa, const uint8_t *qb)
{
    using C = MP<K>;
    const uint32_t a0 = smem_u32(pa), b = smem_u32(qb);
    constexpr uint32_t id = idesc_tf32_f32(128, MP_IC);
    constexpr uint32_t alo = (C::KP / 4) * C::PA_LBO, blo = (C::KP / 4) * C::QB_LBO;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const uint32_t a = a0 + t * C::PA_BYTES, d = tmem + (t ? C::COL_OM : 0u);
#pragma unroll
        for (int s = 0; s < C::KP / 8; ++s) {
            const uint32_t ao = a + s * 2 * C::PA_LBO, bo = b + s * 2 * C::QB_LBO;
            const uint64_t ahi = umma_desc_kmajor(ao, C::PA_LBO, C::T_SBO);
            const uint64_t alw = umma_desc_kmajor(ao + alo, C::PA_LBO, C::T_SBO);
            const uint64_t bhi = umma_desc_kmajor(bo, C::QB_LBO, C::T_SBO);
            const uint64_t blw = umma_desc_kmajor(bo + blo, C::QB_LBO, C::T_SBO);
            tc_mma_tf32(d, ahi, bhi, id, s > 0 ? 1u : 0u);
            tc_mma_tf32(d, alw, bhi, id, 1u);
            tc_mma_tf32(d, ahi, blw, id, 1u);
        }
    }
}

/* 32 individuals' codes of SNP column j from individual ic (a multiple of 32) */
__device__ __forceinline__ uint2 col_load32(const uint8_t *__restrict__ bed, int64_t pitch, int64_t j, bool valid,
                                            int64_t ic)
{
    return valid ? __ldg((const uint2 *)(bed + (size_t)j * pitch + (size_t)(ic / 4)))
                 : make_uint2(0x55555555u, 0x55555555u);
}

/* Warp roles as in the Q sweep: warps 0-3 producers (thread = SNP row), warp 4 controller.
 *
 * EMS = true is the EM P-step of em_p! (algorithms_inner.jl:108-141, loops.jl:700-721) on the
 * same pipeline: per SNP the two sums sum_i nm g q_k / qp and sum_i nm (2-g) q_k / (1-qp)
 * (rows of 2K, the FP64 EM sweep's layout, finalised by k_emp_finalize), with no Hessian tile,
 * MMAs or drains; a package slot is handed back once the four producer warps have read it. */
constexpr int MP_CTA = MP_THREADS + 32;

template <int K, bool EMS>
__global__ void __launch_bounds__(MP_CTA, (K <= 10 ? 3 : 2))
k_sweep_p_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
                const uint8_t *__restrict__ pkg, const double *__restrict__ p, int64_t islice,
                double *__restrict__ out, int *__restrict__ err)
{
    using C = MP<K>;
    constexpr int T = C::T, N = C::N, E = EMS ? 2 * K : C::E;
    extern __shared__ __align__(1024) uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    /* qp ready, qp consumed (4 warps), C tile written (4 warps), Hessian done, package landed [3],
     * package read (4 warps, EM sums only) [3] */
    __shared__ uint64_t mbar[4 + 2 * MP_NPKG];
    __shared__ uint32_t tmem_holder;
    __shared__ volatile int abort_flag;
    uint64_t *bar_qp = &mbar[0], *bar_qfree = &mbar[1], *bar_afull = &mbar[2], *bar_h = &mbar[3], *bar_p = &mbar[4];
    uint64_t *bar_read = &mbar[4 + MP_NPKG];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp < 4;
    const int64_t j = (int64_t)blockIdx.x * 128 + tid;
    const bool valid = producer && j < J;
    const int64_t ia = (int64_t)blockIdx.y * islice;    /* islice is a multiple of MP_IC */
    const int64_t ib = min(I, ia + islice);
    const int nchunk = (int)((ib - ia + MP_IC - 1) / MP_IC);
    const uint8_t *pk0 = pkg + (size_t)(ia / MP_IC) * C::PKG;
    uint8_t *At = sm + C::OFF_A;

    if (warp == 4) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        mbar_init(bar_qp, 1);
        mbar_init(bar_qfree, 4);
        mbar_init(bar_afull, 4);
        mbar_init(bar_h, 1);
        for (int b = 0; b < MP_NPKG; ++b) mbar_init(&bar_p[b], 1);
        for (int b = 0; b < MP_NPKG; ++b) mbar_init(&bar_read[b], 4);
        abort_flag = 0;
        mbar_fence_init();
    }
    code_table_init((float4 *)(sm + C::OFF_TAB), tid, MP_CTA);
    if (producer) {   /* this thread's rows of the TF32 P and (1-P) tiles */
        float hv[C::KP], lv[C::KP], hb[C::KP], lb[C::KP];
#pragma unroll
        for (int k = 0; k < C::KP; ++k) {
            hv[k] = lv[k] = hb[k] = lb[k] = 0.f;
            if (k < K) {
                const double pv = valid ? p[(size_t)K * j + k] : 0.5;
                tf32_split((float)pv, hv[k], lv[k]);
                tf32_split((float)(1.0 - pv), hb[k], lb[k]);
            }
        }
        uint8_t *pa = sm + C::OFF_PA, *pb = pa + C::PA_BYTES;
#pragma unroll
        for (int f = 0; f < C::KP; f += 4) {
            *(float4 *)(pa + kmaj_off(tid, f, C::PA_LBO)) = make_float4(hv[f], hv[f + 1], hv[f + 2], hv[f + 3]);
            *(float4 *)(pa + kmaj_off(tid, C::KP + f, C::PA_LBO)) = make_float4(lv[f], lv[f + 1], lv[f + 2], lv[f + 3]);
            *(float4 *)(pb + kmaj_off(tid, f, C::PA_LBO)) = make_float4(hb[f], hb[f + 1], hb[f + 2], hb[f + 3]);
            *(float4 *)(pb + kmaj_off(tid, C::KP + f, C::PA_LBO)) = make_float4(lb[f], lb[f + 1], lb[f + 2], lb[f + 3]);
        }
    }
    fence_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_holder;
    bool ok = true;
    auto wait = [&](uint64_t *b, uint32_t parity) -> bool {
        if (!ok) return false;
        for (uint32_t n = 0; n < MX_WAIT_LIMIT; ++n) {
            if (mbar_try_wait(b, parity)) return true;
            if ((n & 255u) == 255u && abort_flag) break;
        }
        ok = false;
        abort_flag = 1;
        atomicOr(err, 1);
        return false;
    };

    if (!producer) {
        /* ---------------------------------------------------------------- controller warp */
        const bool leader = lane == 0;
        auto copy_pkg = [&](int c) {
            if (leader) {
                mbar_arrive_expect_tx(&bar_p[c % MP_NPKG], C::PKG);
                bulk_g2s(sm + C::OFF_PKG + (c % MP_NPKG) * C::PKG, pk0 + (size_t)c * C::PKG, C::PKG,
                         &bar_p[c % MP_NPKG]);
            }
        };
        for (int c = 0; c < min(nchunk, MP_NPKG); ++c) copy_pkg(c);
        if (nchunk > 0 && wait(&bar_p[0], 0u) && leader) {
            tc_fence_after_sync();
            issue_qp_p<K>(tmem, sm + C::OFF_PA, sm + C::OFF_PKG + C::PK_QB);
            tc_commit(bar_qp);
        }
        constexpr uint32_t idesc = idesc_bf16_f32(128, N);
        for (int c = 0; c < nchunk && ok; ++c) {
            if (c + 1 < nchunk) {
                const int cn = c + 1;
                const bool landed = wait(&bar_p[cn % MP_NPKG], (uint32_t)((cn / MP_NPKG) & 1));
                if (landed && wait(bar_qfree, (uint32_t)(c & 1)) && leader) {
                    tc_fence_after_sync();
                    issue_qp_p<K>(tmem, sm + C::OFF_PA, sm + C::OFF_PKG + (cn % MP_NPKG) * C::PKG + C::PK_QB);
                    tc_commit(bar_qp);
                }
            }
            if constexpr (EMS) {
                /* slot c % 3's (c / 3)-th reading; its next one needs the copy issued here */
                if (c + MP_NPKG < nchunk && wait(&bar_read[c % MP_NPKG], (uint32_t)((c / MP_NPKG) & 1))) {
                    fence_async_smem();
                    copy_pkg(c + MP_NPKG);
                }
                continue;
            }
            if (wait(bar_afull, (uint32_t)(c & 1)) && leader) {
                tc_fence_after_sync();
                const uint8_t *pk = sm + C::OFF_PKG + (c % MP_NPKG) * C::PKG;
                const uint32_t abase = smem_u32(At), bbase = smem_u32(pk);
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    const uint64_t ad = umma_desc_kmajor(abase + ks * 2 * C::A_LBO, C::A_LBO, C::A_SBO);
                    const uint64_t bd = umma_desc_kmajor(bbase + ks * 2 * C::B_LBO, C::B_LBO, C::B_SBO);
                    tc_mma_bf16(tmem + C::COL_H, ad, bd, idesc, (c % MX_HBLOCK != 0 || ks > 0) ? 1u : 0u);
                }
                tc_commit(bar_h);
            }
            if (c + MP_NPKG < nchunk && wait(bar_h, (uint32_t)(c & 1))) {
                fence_async_smem();
                copy_pkg(c + MP_NPKG);
            }
        }
    } else {
        /* ---------------------------------------------------------------- producer warps */
        const float4 *tab = (const float4 *)(sm + C::OFF_TAB) + (tid & 7);
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        uint2 gcur = make_uint2(0x55555555u, 0x55555555u), gnext = gcur;
        if (nchunk > 0) gcur = col_load32(bed, pitch, j, valid, ia);
        if (nchunk > 1) gnext = col_load32(bed, pitch, j, valid, ia + MP_IC);
        double gd[K], hd[EMS ? K : 1];
#pragma unroll
        for (int k = 0; k < K; ++k) gd[k] = 0.0;
#pragma unroll
        for (int k = 0; k < (EMS ? K : 1); ++k) hd[k] = 0.0;
        for (int c = 0; c < nchunk && ok; ++c) {
            const uint8_t *pk = sm + C::OFF_PKG + (c % MP_NPKG) * C::PKG;
            const float *Qf = (const float *)(pk + C::PK_QF);
            const float2 *Sres = (const float2 *)(pk + C::PK_S);
            /* qp / om of the chunk's 32 individuals, read in two halves of 16 columns
             * (individuals 0-15, then 16-31) to keep the producer within its registers */
            uint32_t rq[16], ro[16];
            if (!wait(bar_qp, (uint32_t)(c & 1))) break;
            tc_fence_after_sync();
            tmem_ld16_raw(tmem + lane_base, rq);
            tmem_ld16_raw(tmem + lane_base + C::COL_OM, ro);
            tmem_wait_ld();
            if (!wait(&bar_p[c % MP_NPKG], (uint32_t)((c / MP_NPKG) & 1))) break;
            if constexpr (!EMS) {
                if (c > 0 && !wait(bar_h, (uint32_t)((c - 1) & 1))) break;   /* the C tile is free */
                if (c > 0 && c % MX_HBLOCK == 0) {   /* drain the block of chunks c-MX_HBLOCK .. c-1 */
                    tc_fence_after_sync();
                    hess_drain<N, T>(tmem + lane_base + C::COL_H,
                                     out + ((size_t)blockIdx.y * J + (valid ? j : 0)) * E, c == MX_HBLOCK, valid);
                    tc_fence_before_sync();
                }
            }
            float2 gk[K], hk[EMS ? K : 1];
#pragma unroll
            for (int k = 0; k < K; ++k) gk[k] = make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < (EMS ? K : 1); ++k) hk[k] = make_float2(0.f, 0.f);
#pragma unroll
            for (int kc = 0; kc < 4; ++kc) {
                if (kc == 2) {   /* the second half of the columns; then the qp columns are free */
                    tc_fence_after_sync();
                    tmem_ld16_raw(tmem + lane_base + 16u, rq);
                    tmem_ld16_raw(tmem + lane_base + C::COL_OM + 16u, ro);
                    tmem_wait_ld();
                    tc_fence_before_sync();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(bar_qfree);
                }
                uint32_t cp[4];
                float2 zz[4], z2s[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int m = kc * 4 + e;
                    const int r = 2 * (m & 7);   /* this pair's column in rq / ro */
                    const uint32_t w = (m < 8) ? gcur.x : gcur.y;
                    const float4 a = tab[8 * ((w >> (4 * (m & 7))) & 15u)];
                    const float2 qp = make_float2(__uint_as_float(rq[r]), __uint_as_float(rq[r + 1]));
                    const float2 om = __fadd2_rn(make_float2(__uint_as_float(ro[r]), __uint_as_float(ro[r + 1])),
                                                 Sres[m]);
                    const float2 pr = __fmul2_rn(qp, om);
                    const float2 rr = make_float2(rcp_approx(pr.x), rcp_approx(pr.y));
                    const float2 r1 = __fmul2_rn(om, rr), r2 = __fmul2_rn(qp, rr);
                    const float2 z1 = __fmul2_rn(make_float2(a.x, a.y), r1);
                    const float2 z2 = __fmul2_rn(make_float2(a.z, a.w), r2);
                    if constexpr (EMS) {
                        zz[e] = z1;                                             /* nm g / qp */
                        z2s[e] = z2;                                            /* nm (2-g) / (1-qp) */
                    } else {
                        const float2 cw = __ffma2_rn(z1, r1, __fmul2_rn(z2, r2));   /* nm (g/qp^2 + (2-g)/(1-qp)^2) */
                        zz[e] = make_float2(z1.x - z2.x, z1.y - z2.y);              /* nm (g/qp - (2-g)/(1-qp)) */
                        cp[e] = pack_bf16x2(cw.x, cw.y);
                    }
                }
                if constexpr (!EMS)
                    *(uint4 *)(At + kc * C::A_LBO + 16 * tid) = make_uint4(cp[0], cp[1], cp[2], cp[3]);
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float4 q0 = *(const float4 *)(Qf + k * C::QS + kc * 8);
                    const float4 q1 = *(const float4 *)(Qf + k * C::QS + kc * 8 + 4);
                    gk[k] = __ffma2_rn(zz[0], make_float2(q0.x, q0.y), gk[k]);
                    gk[k] = __ffma2_rn(zz[1], make_float2(q0.z, q0.w), gk[k]);
                    gk[k] = __ffma2_rn(zz[2], make_float2(q1.x, q1.y), gk[k]);
                    gk[k] = __ffma2_rn(zz[3], make_float2(q1.z, q1.w), gk[k]);
                    if constexpr (EMS) {
                        hk[k] = __ffma2_rn(z2s[0], make_float2(q0.x, q0.y), hk[k]);
                        hk[k] = __ffma2_rn(z2s[1], make_float2(q0.z, q0.w), hk[k]);
                        hk[k] = __ffma2_rn(z2s[2], make_float2(q1.x, q1.y), hk[k]);
                        hk[k] = __ffma2_rn(z2s[3], make_float2(q1.z, q1.w), hk[k]);
                    }
                }
            }
            if constexpr (EMS) {   /* the package is read: hand its slot back */
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar_read[c % MP_NPKG]);
            }
#pragma unroll
            for (int k = 0; k < K; ++k) gd[k] += (double)gk[k].x + (double)gk[k].y;
            if constexpr (EMS) {
#pragma unroll
                for (int k = 0; k < K; ++k) hd[k] += (double)hk[k].x + (double)hk[k].y;
            }
            if (c + 1 < nchunk) {
                gcur = gnext;
                if (c + 2 < nchunk) gnext = col_load32(bed, pitch, j, valid, ia + (int64_t)(c + 2) * MP_IC);
            }
            if constexpr (!EMS) {
                fence_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(bar_afull);
            }
        }
        if constexpr (EMS) {
            if (valid) {   /* a thread whose wait gave up writes NaN sums (and err is set) */
                double *o = out + ((size_t)blockIdx.y * J + j) * E;
                const double bad = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    o[k] = ok ? gd[k] : bad;
                    o[K + k] = ok ? hd[k] : bad;
                }
            }
        } else {
            if (nchunk > 0) wait(bar_h, (uint32_t)((nchunk - 1) & 1));   /* the last Hessian MMAs */
            if (valid) {
                double *o = out + ((size_t)blockIdx.y * J + j) * E;
#pragma unroll
                for (int k = 0; k < K; ++k) o[T + k] = gd[k];
            }
        }
    }
    ok = __syncthreads_and(ok);
    if (!ok && tid == MP_THREADS) {
        mbar_wait_bounded(bar_h, 0u, 1024u);
        mbar_wait_bounded(bar_h, 1u, 1024u);
        mbar_wait_bounded(bar_qp, 0u, 1024u);
        mbar_wait_bounded(bar_qp, 1u, 1024u);
        for (int b = 0; b < MP_NPKG; ++b) { mbar_wait_bounded(&bar_p[b], 0u, 1024u); mbar_wait_bounded(&bar_p[b], 1u, 1024u); }
    }
    __syncthreads();
    tc_fence_after_sync();
    if (producer && !EMS) {
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        if (nchunk > 0) {
#pragma unroll 1
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + lane_base + C::COL_H + (uint32_t)c0, v);
                if (valid) {   /* the last accumulation block, added to the drained ones */
                    double *o = out + ((size_t)blockIdx.y * J + j) * E;
                    const bool first = nchunk <= MX_HBLOCK;
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        if (c0 + e < T)
                            o[c0 + e] = ok ? (first ? (double)v[e] : o[c0 + e] + (double)v[e])
                                           : __longlong_as_double(0x7ff8000000000000LL);
                }
            }
        } else if (valid) {
            double *o = out + ((size_t)blockIdx.y * J + j) * E;
            for (int e = 0; e < T; ++e) o[e] = 0.0;
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 4) tmem_dealloc_warp(tmem, C::NCOLS);
}

/* 64 individuals' codes of SNP column j from individual ic (a multiple of 64) */
__device__ __forceinline__ uint4 col_load64(const uint8_t *__restrict__ bed, int64_t pitch, int64_t j, bool valid,
                                            int64_t ic)
{
    return valid ? __ldg((const uint4 *)(bed + (size_t)j * pitch + (size_t)(ic / 4)))
                 : make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u);
}

/* ===================================================================== loglik
 * loglikelihood_loop_skipmissing (loops.jl:517-539) with FP32 cells: thread = SNP, individuals
 * in pairs; qp is an FP32 FMA chain and 1 - qp is formed from it by one subtraction (exact for
 * qp >= 1/2), as the reference forms it; each cell contributes qp^g (1-qp)^(2-g) (1 when
 * missing), two cells' factors are
 * multiplied in FP32 and folded into an FP64 running product whose exponent moves into an
 * integer every 12 pairs; one FP64 log per thread at the end.  Every product is rounded to
 * nearest, so the rounding error is a random walk far below the convergence test's resolution. */
constexpr int ML_IC = 64;

constexpr int ML_JT = 2;   /* SNPs per thread (j and j + 128): each broadcast load of q serves both */

template <int K>
__global__ void __launch_bounds__(128, (K <= 10 ? 6 : 4))
k_loglik_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
               const double *__restrict__ q, const double *__restrict__ p, int64_t islice,
               double *__restrict__ partial)
{
    constexpr int PREF = (K * ML_IC + 127) / 128;
    __shared__ float4 Qs[2][K][ML_IC / 4];              /* q of individuals 4m .. 4m+3 */
    __shared__ double red[4];
    const int tid = threadIdx.x;
    const int64_t j0 = (int64_t)blockIdx.x * (128 * ML_JT) + tid;
    const int64_t ia = (int64_t)blockIdx.y * islice;
    const int64_t ib = min(I, ia + islice);
    const int nchunk = (int)((ib - ia + ML_IC - 1) / ML_IC);
    bool valid[ML_JT];
    float2 pd[ML_JT][K];
#pragma unroll
    for (int t = 0; t < ML_JT; ++t) {
        const int64_t j = j0 + 128 * t;
        valid[t] = j < J;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double pv = valid[t] ? p[(size_t)K * j + k] : 0.5;
            pd[t][k] = make_float2((float)pv, (float)pv);
        }
    }
    float qr[PREF];
    const uint4 none = make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u);
    uint4 g[ML_JT], gnext[ML_JT];
#pragma unroll
    for (int t = 0; t < ML_JT; ++t) g[t] = gnext[t] = none;
    auto load = [&](int64_t ic) {
#pragma unroll
        for (int u = 0; u < PREF; ++u) {
            const int t = tid + u * 128;                 /* t = k * IC + ii */
            const int k = t / ML_IC, ii = t - k * ML_IC;
            qr[u] = (t < K * ML_IC && ic + ii < ib) ? (float)q[(size_t)K * (ic + ii) + k] : 1.0f / K;
        }
#pragma unroll
        for (int t = 0; t < ML_JT; ++t) gnext[t] = col_load64(bed, pitch, j0 + 128 * t, valid[t], ic);
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
    auto fold = [&](double &prod, int64_t &ex) {   /* move the exponent into the integer */
        const int64_t bits = __double_as_longlong(prod);
        ex += ((bits >> 52) & 0x7FF) - 1023;
        prod = __longlong_as_double((bits & ~(0x7FFLL << 52)) | (1023LL << 52));
    };
    if (nchunk > 0) {
        load(ia);
        store(0);
#pragma unroll
        for (int t = 0; t < ML_JT; ++t) g[t] = gnext[t];
    }
    if (nchunk > 1) load(ia + ML_IC);
    __syncthreads();
    double prod[ML_JT];
    int64_t ex[ML_JT];
#pragma unroll
    for (int t = 0; t < ML_JT; ++t) { prod[t] = 1.0; ex[t] = 0; }
    for (int c = 0; c < nchunk; ++c) {
        const int s = c & 1;
        uint4 gw[ML_JT];   /* the chunk's 4 code words per SNP, consumed from .x and shifted down */
#pragma unroll
        for (int t = 0; t < ML_JT; ++t) gw[t] = g[t];
#pragma unroll 1
        for (int wd = 0; wd < 4; ++wd) {   /* 16 individuals per 32-bit code word */
#pragma unroll
            for (int m2l = 0; m2l < 4; ++m2l) {
                const int m2 = 4 * wd + m2l;
                /* qp of two individual pairs for both SNPs (one 16-byte broadcast load of q per k) */
                float2 qpa[ML_JT], qpb[ML_JT];
#pragma unroll
                for (int t = 0; t < ML_JT; ++t) qpa[t] = qpb[t] = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float4 qv = Qs[s][k][m2];
#pragma unroll
                    for (int t = 0; t < ML_JT; ++t) {
                        qpa[t] = __ffma2_rn(make_float2(qv.x, qv.y), pd[t][k], qpa[t]);
                        qpb[t] = __ffma2_rn(make_float2(qv.z, qv.w), pd[t][k], qpb[t]);
                    }
                }
#pragma unroll
                for (int t = 0; t < ML_JT; ++t) {
                    float2 fa, fb;   /* (first, second) cell factors of pair a (hm = 0) and pair b */
#pragma unroll
                    for (int hm = 0; hm < 2; ++hm) {
                        /* the pair's 4 code bits, tested in place in their 32-bit word */
                        const uint32_t w = gw[t].x;
                        const int b = 4 * (2 * m2l + hm);
                        const float2 qp = hm ? qpb[t] : qpa[t];
                        /* 1 - qp as the reference forms it (one rounding), from the unbiased FP32 qp */
                        const float2 om = __ffma2_rn(qp, make_float2(-1.f, -1.f), make_float2(1.f, 1.f));
                        /* factor per code: 00 -> om^2, 01 -> 1 (missing), 10 -> qp om, 11 -> qp^2;
                         * the three products are formed for both cells and one is selected */
                        const float2 oo = __fmul2_rn(om, om), qo = __fmul2_rn(qp, om), qq = __fmul2_rn(qp, qp);
                        const bool lo0 = (w >> b) & 1u, hi0 = (w >> (b + 1)) & 1u;
                        const bool lo1 = (w >> (b + 2)) & 1u, hi1 = (w >> (b + 3)) & 1u;
                        const float f0 = hi0 ? (lo0 ? qq.x : qo.x) : (lo0 ? 1.f : oo.x);
                        const float f1 = hi1 ? (lo1 ? qq.y : qo.y) : (lo1 ? 1.f : oo.y);
                        if (hm) fb = make_float2(f0, f1);
                        else fa = make_float2(f0, f1);
                    }
                    /* the two pairs' products f0 f1 in one paired multiply, each into the FP64 product */
                    const float2 ff = __fmul2_rn(make_float2(fa.x, fb.x), make_float2(fa.y, fb.y));
                    prod[t] *= (double)ff.x;
                    prod[t] *= (double)ff.y;
                }
            }
            /* 8 pairs per word: each pair's factor is >= 1e-20, so the product stays normal */
#pragma unroll
            for (int t = 0; t < ML_JT; ++t) {
                fold(prod[t], ex[t]);
                gw[t] = make_uint4(gw[t].y, gw[t].z, gw[t].w, 0u);
            }
        }
        if (c + 1 < nchunk) {
            store(s ^ 1);
#pragma unroll
            for (int t = 0; t < ML_JT; ++t) g[t] = gnext[t];
            if (c + 2 < nchunk) load(ia + (int64_t)(c + 2) * ML_IC);
        }
        __syncthreads();
    }
    double ll = 0.0;
#pragma unroll
    for (int t = 0; t < ML_JT; ++t)
        if (valid[t]) ll += log(prod[t]) + (double)ex[t] * 0.69314718055994530942;
    for (int o = 16; o > 0; o >>= 1) ll += __shfl_down_sync(0xffffffffu, ll, o);
    if ((tid & 31) == 0) red[tid >> 5] = ll;
    __syncthreads();
    if (tid == 0) partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = red[0] + red[1] + red[2] + red[3];
}

/* A bounded mbarrier wait that nothing completes: it gives up after `polls` polls and raises the
 * error flag as the sweeps' pipeline waits do (the failure-reporting self-test). */
__global__ void k_wait_probe(int *__restrict__ err, uint32_t polls)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
        if (!mbar_wait_bounded(&bar, 0u, polls)) atomicOr(err, 1);
    }
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
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sweep_p_mixed<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MP<K>::SMEM);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sweep_p_mixed<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MP<K>::SMEM);
    return e;
}

template <int K>
cudaError_t launch_q_mixed_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                             const double *p, const SweepPlan &pl, double *out, int *err, uint8_t *pkg,
                             cudaStream_t st)
{
    k_q_pack<K><<<(unsigned)((J + MQ_JC - 1) / MQ_JC), 128, 0, st>>>(p, J, pkg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_sweep_q_mixed<K><<<grid, MQ_CTA, MQ<K>::SMEM, st>>>(bed, I, J, pitch, q, pkg, pl.slice, out, err);
    return cudaGetLastError();
}

template <int K>
size_t q_pkg_bytes_t(int64_t J)
{
    return (size_t)((J + MQ_JC - 1) / MQ_JC) * MQ<K>::PKG;
}

template <int K>
cudaError_t launch_p_mixed_t(int mode, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                             const double *p, const SweepPlan &pl, double *out, int *err, uint8_t *pkg,
                             cudaStream_t st)
{
    k_p_pack<K><<<(unsigned)((I + MP_IC - 1) / MP_IC), 128, 0, st>>>(q, I, pkg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    if (mode == 1)
        k_sweep_p_mixed<K, true><<<grid, MP_CTA, MP<K>::SMEM, st>>>(bed, I, J, pitch, pkg, p, pl.slice, out, err);
    else
        k_sweep_p_mixed<K, false><<<grid, MP_CTA, MP<K>::SMEM, st>>>(bed, I, J, pitch, pkg, p, pl.slice, out, err);
    return cudaGetLastError();
}

template <int K>
size_t p_pkg_bytes_t(int64_t I)
{
    return (size_t)((I + MP_IC - 1) / MP_IC) * MP<K>::PKG;
}

template <int K>
cudaError_t launch_ll_mixed_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                              const double *p, const SweepPlan &pl, double *partial, double *out, int *err,
                              uint8_t *pkg, cudaStream_t st)
{
    (void)err;
    (void)pkg;
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_loglik_mixed<K><<<grid, 128, 0, st>>>(bed, I, J, pitch, q, p, pl.slice, partial);
    k_sum_partials_mixed<<<1, 1024, 0, st>>>(partial, (int64_t)pl.gx * pl.S, out);
    return cudaGetLastError();
}

/* Slices over the second axis for CTAs of 128 rows, `per_sm` of which are resident per SM.  CTAs
 * of one launch take equal time, so the launch lasts ceil(gx S / (sms per_sm)) waves of CTAs that
 * each do 1/S of a row tile's work; S minimises waves / S, plus 0.5 % per extra slice (each adds a
 * partial slice for the consumer to read).  Slices are multiples of `unit`, at least 4 units
 * long, and at most smax. */
SweepPlan plan_rows(int64_t rows, int64_t cols, int sms, int per_sm, int64_t unit, int64_t smax)
{
    SweepPlan pl;
    pl.gx = (int)std::max<int64_t>(1, (rows + 127) / 128);
    pl.S = 1;
    pl.slice = std::max<int64_t>(unit, (cols + unit - 1) / unit * unit);
    if (cols <= 0) return pl;
    const int64_t cap = std::max<int64_t>(1, (int64_t)sms * per_sm);
    const int64_t fill = (cap + pl.gx - 1) / pl.gx;   /* slices that fill the GPU once */
    const int64_t top = std::min<int64_t>({std::max<int64_t>(1, (cols + 4 * unit - 1) / (4 * unit)),
                                           std::max<int64_t>(16, 2 * fill), std::max<int64_t>(1, smax)});
    double best = 1e300;
    for (int64_t s = 1; s <= top; ++s) {
        const int64_t slice = ((cols + s - 1) / s + unit - 1) / unit * unit;
        const int64_t S = (cols + slice - 1) / slice;
        const int64_t waves = ((int64_t)pl.gx * S + cap - 1) / cap;
        const double cost = (double)waves / (double)S * (1.0 + 0.005 * (double)(S - 1));
        if (cost < best - 1e-12) {
            best = cost;
            pl.S = (int)S;
            pl.slice = slice;
        }
    }
    return pl;
}

/* resident CTAs per SM of the mixed kernels (occupancy at their shared memory; needs
 * prepare_mixed(K) first), cached per kernel and K; `fallback` when it cannot be queried */
template <int K>
int resident_t(int kind)
{
    int n = 0;
    cudaError_t e;
    if (kind == 0) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_q_mixed<K>, MQ_CTA, MQ<K>::SMEM);
    else if (kind == 1) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_p_mixed<K, false>, MP_CTA, MP<K>::SMEM);
    else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_loglik_mixed<K>, 128, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int resident(int kind, int K, int fallback)
{
    static int cache[3][17] = {};
    if (K < 1 || K > 16) return fallback;
    int &c = cache[kind][K];
    if (c <= 0) {
        int n = 0;
        ADMIX_DISPATCH_K(K, n = resident_t<KK>(kind));
        if (n <= 0) return fallback;
        c = n;
    }
    return c;
}

} // namespace

cudaError_t prepare_mixed(int K)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = prepare_mixed_t<KK>());
    return e;
}

/* One CTA per 128 individuals and SNP slice. */
SweepPlan plan_sweep_q_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax)
{
    return plan_rows(I, J, sms, resident(0, K, 3), MQ_JC, smax);
}

/* One CTA per 128 SNPs and individual slice (slices are multiples of 64 individuals). */
SweepPlan plan_sweep_p_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax)
{
    return plan_rows(J, I, sms, resident(1, K, 3), MP_IC, smax);
}

SweepPlan plan_loglik_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax)
{
    /* CTAs of 128 threads x ML_JT SNPs */
    return plan_rows((J + ML_JT - 1) / ML_JT, I, sms, resident(2, K, 4), ML_IC, smax);
}

cudaError_t launch_sweep_q_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                 const double *p, const SweepPlan &pl, double *out, int *err, uint8_t *pkg,
                                 cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_q_mixed_t<KK>(bed, I, J, pitch, q, p, pl, out, err, pkg, st));
    return e;
}

size_t sweep_q_mixed_pkg_bytes(int K, int64_t J)
{
    size_t b = 0;
    ADMIX_DISPATCH_K(K, b = q_pkg_bytes_t<KK>(J));
    return b;
}

cudaError_t launch_sweep_p_mixed(int K, int mode, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                                 const double *q, const double *p, const SweepPlan &pl, double *out, int *err,
                                 uint8_t *pkg, cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    if (mode != 0 && mode != 1) return e;
    ADMIX_DISPATCH_K(K, e = launch_p_mixed_t<KK>(mode, bed, I, J, pitch, q, p, pl, out, err, pkg, st));
    return e;
}

cudaError_t launch_wait_probe(int *err, uint32_t polls, cudaStream_t st)
{
    k_wait_probe<<<1, 32, 0, st>>>(err, polls);
    return cudaGetLastError();
}

size_t sweep_p_mixed_pkg_bytes(int K, int64_t I)
{
    size_t b = 0;
    ADMIX_DISPATCH_K(K, b = p_pkg_bytes_t<KK>(I));
    return b;
}

cudaError_t launch_loglik_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                const double *p, const SweepPlan &pl, double *partial, double *out, int *err,
                                uint8_t *pkg, cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_ll_mixed_t<KK>(bed, I, J, pitch, q, p, pl, partial, out, err, pkg, st));
    return e;
}
