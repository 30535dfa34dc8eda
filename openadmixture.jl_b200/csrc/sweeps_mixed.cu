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
/* The Hessian diagonal columns and the gradient accumulator are read into FP64 (and the diagonal
 * cleared) every MX_DRAIN chunks: each such FP32 sum covers at most 4 * MX_DRAIN accumulations.
 * MX_HBLOCK is a multiple of MX_DRAIN, so a block drain always follows a diagonal drain. */
constexpr int MX_DRAIN = 2;
static_assert(MX_HBLOCK % MX_DRAIN == 0, "block drains coincide with diagonal drains");

/* Column order of the Hessian accumulators (T = K (K + 1) / 2 pairs): the K diagonal pairs first
 * (column k = pair (k, k)), then the off-diagonal pairs (a, b), b < a, in the packed order of the
 * FP64 partial rows, then K residual columns: column T + k holds the diagonal's B-operand rounding
 * residual sum_j w (x_k^2 - bf16(x_k^2)), which belongs to entry (k, k).
 * col_out: the packed FP64 index a (a + 1) / 2 + b that column col adds into; col_pair: the
 * factors of a pair column. */
__host__ __device__ constexpr int col_out(int K, int col)
{
    if (col < K) return col * (col + 1) / 2 + col;
    const int T = K * (K + 1) / 2;
    if (col >= T) return (col - T) * (col - T + 1) / 2 + (col - T);
    int m = col - K, a = 1;
    while ((a + 1) * a / 2 <= m) ++a;
    return a * (a + 1) / 2 + (m - a * (a - 1) / 2);
}

__device__ __forceinline__ void col_pair(int K, int col, int &ka, int &kb)
{
    if (col < K) { ka = kb = col; return; }
    int m = col - K, a = 1;
    while ((a + 1) * a / 2 <= m) ++a;
    ka = a;
    kb = m - a * (a - 1) / 2;
}

/* add (or, for the first block, store) the Hessian accumulator's columns K .. T+K-1 (off-diagonal
 * pairs and diagonal residuals; the diagonal columns 0..K-1 are drained every MX_DRAIN chunks) of this
 * thread's lane into the FP64 entries o[col_out(K, e)] */
template <int K, int N, int T>
__device__ __forceinline__ void hess_drain(uint32_t taddr, double *o, bool first, bool valid)
{
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        tmem_ld16(taddr + (uint32_t)c0, v);
        if (valid) {
#pragma unroll
            for (int e = 0; e < 16; ++e)
                if (c0 + e >= K && c0 + e < T + K) {
                    double &x = o[col_out(K, c0 + e)];
                    x = first ? (double)v[e] : x + (double)v[e];
                }
        }
    }
}

/* After a chunk's MMAs completed (one producer thread = one TMEM lane; lane = this lane's base):
 * the chunk's Hessian diagonal -- columns 0..K-1 of the Hessian accumulator at col_h -- is added
 * into dd[] and those columns are set to zero for the next chunk; the chunk's gradient sums
 * (columns 0..K-1 and K..2K-1 of the accumulator at col_g) are added into gd[]. */
template <int K, int NDG>
__device__ __forceinline__ void drain_chunk(uint32_t lane, uint32_t col_h, uint32_t col_g, double (&dd)[K], double (&gd)[K])
{
    static_assert(K <= 16 && 2 * K <= NDG && NDG <= 32, "diagonal columns within one 16-column load");
    tc_fence_after_sync();
    float h[16], g0[16], g1[16];
    tmem_ld16(lane + col_h, h);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        dd[k] += (double)h[k];
        h[k] = 0.f;
    }
    tmem_st16(lane + col_h, h);
    tmem_ld16(lane + col_g, g0);
    if constexpr (NDG == 32) tmem_ld16(lane + col_g + 16u, g1);
#pragma unroll
    for (int k = 0; k < K; ++k) {   /* hi * hi + lo * hi, plus hi * lo (2^-8 of it: one FP32 rounding) */
        const float hl = (K + k < 16) ? g0[K + k] : g1[(K + k) & 15];
        gd[k] += (double)(g0[k] + hl);
    }
    tmem_wait_st();
    tc_fence_before_sync();
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
 * Per 32-SNP chunk, three tensor-core products:
 *   qp / om    D[128 x 64] = Qtile * [p ; 1-p]^T in TF32 split form (hi*hi + lo*hi + hi*lo, about
 *              2^-21 relative): the K-term dot products of every (individual, SNP) cell;
 *   Hessian    D[128 x N] += [w1 | w2] * [PP ; PbarPbar]^T in BF16 (FP32 accumulation), drained
 *              into FP64 every MX_HBLOCK chunks; its columns hold the K diagonal pairs first;
 *   gradient   D[128 x NDG] = dz_hi * [p_hi | p_lo]^T + dz_lo * [p_hi | 0]^T, the gradient sum_j dz p_k
 *              with dz = z1 - z2 and both factors split into two BF16 parts (hi*hi + lo*hi in
 *              columns 0..K-1, hi*lo in K..2K-1: about 2^-17 relative), a fresh FP32 sum every
 *              MX_DRAIN chunks that the producers add into FP64;
 * and on the CUDA cores, per cell: the code lookup, one reciprocal, z1, z2, w1, w2, dz and its
 * split, and sum_j z2 (FP32 per chunk, FP64 across chunks).  The gradient is
 * sum_j (z1 - z2) p_k + z2 (= sum_j z1 p_k + z2 (1 - p_k)).
 *
 * The compensated diagonal: the tensor core's FP32 accumulation rounds toward zero, so a sum
 * carried over many chunks drifts low (about 5e-5 relative over 256 chunks).  Every MX_DRAIN
 * chunks the producers read the Hessian's K diagonal columns, add them into FP64 and store zeros
 * back (tcgen05.st), so the diagonal is a sum of fresh FP32 sums of 4 * MX_DRAIN accumulations
 * carried on in FP64.  The off-diagonal entries keep the MX_HBLOCK drains.
 *
 * Everything that depends on P alone -- the BF16 pair-product tiles, the TF32 hi / lo split of
 * [p ; 1-p], the gradient B blocks -- is built once per sweep by k_q_pack, one "package" per
 * chunk laid out exactly as the sweep's shared memory wants it, and fetched by each CTA with
 * one bulk asynchronous copy.  The qp MMA of chunk c+1 runs while the CUDA cores work on
 * chunk c. */

constexpr int MQ_JC = 32;          /* SNPs per chunk = 2 BF16 MMA K-steps */
constexpr int MQ_THREADS = 128;    /* one thread per individual = accumulator row */
constexpr int MQ_NPKG = 2;   /* package buffers (a third one leaves room for two CTAs per SM only: slower) */

/* The gradient accumulator: NDG columns, sum_j dz_hi p_hi + dz_lo p_hi in columns 0..K-1 and
 * sum_j dz_hi p_lo in columns K..2K-1.  It starts afresh every MX_DRAIN chunks and the producers
 * add it into FP64, so no FP32 partial of the gradient sees more than MX_DRAIN chunks'
 * accumulations. */
template <int K> struct DGShape {
    static constexpr int NDG = K <= 8 ? 16 : 32;
};

template <int K>
struct MQ {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + K + 15) / 16) * 16;          /* Hessian MMA N: pairs + diagonal residuals, a multiple of 16 */
    static constexpr int KP = ((K + 7) / 8) * 8;                /* TF32 K extent of the qp MMAs */
    static constexpr int QPN = 2 * MQ_JC;                       /* qp MMA N: the chunk's p rows, then 1-p rows */
    static constexpr int NDG = DGShape<K>::NDG;
    static constexpr uint32_t COL_H = 64;                       /* TMEM column of the Hessian accumulator */
    static constexpr uint32_t COL_DG = COL_H + N;               /* TMEM column of the gradient accumulator */
    static constexpr uint32_t NCOLS = tmem_cols_for(COL_DG + NDG);
    static constexpr int E = T + K;                             /* partial entries per individual */
    static constexpr uint32_t A_BYTES = 128 * MQ_JC * 2;        /* one BF16 A tile (128 rows x 32 SNPs): 8 KB */
    static constexpr uint32_t B_BYTES = N * MQ_JC * 2;          /* one BF16 pair-product tile */
    static constexpr uint32_t QA_BYTES = 128 * 2 * KP * 4;      /* TF32 Q tile [hi | lo] */
    static constexpr uint32_t QB_BYTES = QPN * 2 * KP * 4;      /* TF32 [p ; 1-p] chunk [hi | lo] */
    static constexpr uint32_t DGB_BYTES = NDG * MQ_JC * 2;      /* one BF16 B block of the gradient MMAs */
    /* package of one chunk: [PP tile | PbarPbar tile | TF32 [p ; 1-p] | gradient B blocks
     * [p_hi | p_lo] and [p_hi | 0]] */
    static constexpr uint32_t PK_QB = 2 * B_BYTES;
    static constexpr uint32_t PK_DG = PK_QB + QB_BYTES;
    static constexpr uint32_t PKG = PK_DG + 2 * DGB_BYTES;
    static constexpr uint32_t GBUF = MQ_JC * 32;                /* genotype bytes of one chunk */
    static constexpr uint32_t OFF_A = 0;                        /* W1, W2, DZ0, DZ1 tiles */
    static constexpr uint32_t OFF_PKG = 4 * A_BYTES;
    static constexpr uint32_t OFF_QA = OFF_PKG + MQ_NPKG * PKG;
    static constexpr uint32_t OFF_G = OFF_QA + QA_BYTES;        /* two G buffers, [pair][byte][2] */
    static constexpr uint32_t OFF_TAB = OFF_G + 2 * GBUF;       /* float4 [16][8] code table */
    static constexpr uint32_t SMEM = OFF_TAB + 128 * 16 + 1024; /* + alignment slack */
    /* core matrices (8 rows x 16 B): BF16 A 128 B apart along M, 2048 B along K; BF16 B 128 B
     * along N, 16 N bytes along K; TF32 Q tile 128 B along M, 2048 B along K; TF32 [p ; 1-p]
     * 128 B along N, 1024 B along K; gradient B blocks 128 B along N, 16 NDG bytes along K */
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr uint32_t QA_LBO = 2048, QB_LBO = 1024, Q_SBO = 128;
    static constexpr uint32_t DG_LBO = 16 * NDG;
    static_assert(PKG % 16 == 0 && OFF_QA % 16 == 0, "bulk copies and descriptors need 16-byte alignment");
    static_assert(K <= 16, "K up to 16");
};

/* byte offset of element (row r, 4-byte column f) in a K-major no-swizzle tile */
__device__ __forceinline__ uint32_t kmaj_off(int r, int f, uint32_t lbo)
{
    return (uint32_t)(f >> 2) * lbo + (uint32_t)(r >> 3) * 128u + (uint32_t)(r & 7) * 16u + (uint32_t)(f & 3) * 4u;
}

/* BF16 high part of x (round to nearest) and the BF16 of the remainder: hi + lo = x to about
 * 2^-17 relative */
__device__ __forceinline__ void bf16_split(float x, uint16_t &hi, uint16_t &lo)
{
    const uint32_t h = pack_bf16x2(x, 0.f) & 0xFFFFu;
    const float r = x - __uint_as_float(h << 16);
    hi = (uint16_t)h;
    lo = (uint16_t)(pack_bf16x2(r, 0.f) & 0xFFFFu);
}

/* BF16 pair (x in the low half) of non-negative x, y rounded with dither (stochastic rounding,
 * the sm_100a conversion cvt.rs): rbits[15:0] are added below the 16 dropped bits of x and
 * rbits[31:16] below those of y, and the sums are truncated, so x rounds up with probability
 * (dropped bits + d) / 2^16 -- without bias when d is uniform on [0, 2^16) and independent of x.
 * (Measured on a B200: identical, bit for bit, to adding d to the FP32 bit pattern and keeping
 * the high 16 bits.)  Round to nearest is biased for these operands: applied to the Hessian
 * weights it biased the BF16 Hessian diagonal by -3e-6 (Q side) and -4.5e-5 (P side) relative,
 * the same in an exact-arithmetic emulation of the rounding alone. */
__device__ __forceinline__ uint32_t pack_bf16x2_dither(float x, float y, uint32_t rbits)
{
    uint32_t r;
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(y), "f"(x), "r"(rbits));
    return r;
}

/* Dither stream of one accumulator row: a 32-bit LCG stepped once per cell pair; the pair's two
 * cells use its high 16 bits (first cell, rbits[15:0]) and their complement modulo 2^16 (second
 * cell, rbits[31:16]: antithetic) */
__device__ __forceinline__ uint32_t dither_seed(int64_t row, int64_t slice)
{
    return (uint32_t)row * 2654435761u + (uint32_t)slice * 40503u + 12345u;
}
__device__ __forceinline__ uint32_t dither_step(uint32_t &st)
{
    st = st * 1664525u + 1013904223u;
    return __byte_perm(st, st ^ 0x80000000u, 0x7632);
}

/* BF16 pair of the rounding residuals x - bf16(x), y - bf16(y) (bf16 rounding to nearest) */
__device__ __forceinline__ uint32_t pack_bf16x2_res(float x, float y)
{
    const uint32_t h = pack_bf16x2(x, y);
    return pack_bf16x2(x - __uint_as_float(h << 16), y - __uint_as_float(h & 0xFFFF0000u));
}

/* Row n's 8 BF16 values of granule kc (8 SNPs) in a B block of `rows` rows */
__device__ __forceinline__ uint32_t bblk_off(int n, int kc, uint32_t lbo) { return (uint32_t)kc * lbo + 16u * (uint32_t)n; }

/* One package per 32-SNP chunk of the whole SNP range (block = chunk).  SNPs beyond J get
 * p = 0.5; their genotypes read as missing, so they contribute nothing. */
template <int K>
__global__ void __launch_bounds__(128)
k_q_pack(const double *__restrict__ p, int64_t J, uint8_t *__restrict__ pkg)
{
    using C = MQ<K>;
    constexpr int T = C::T, N = C::N, PS = MQ_JC + 4;
    __shared__ __align__(16) float pf[2 * K * PS];             /* p, then 1-p: [term][k][jj] */
    __shared__ __align__(16) uint8_t buf[C::PKG];
    const int tid = threadIdx.x;
    const int64_t jc = (int64_t)blockIdx.x * MQ_JC;
    for (uint32_t t = tid; t < C::PKG / 16; t += 128) ((uint4 *)buf)[t] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    for (int t = tid; t < K * MQ_JC; t += 128) {
        const int jj = t / K, k = t - jj * K;
        const double pd = (jc + jj < J) ? p[(size_t)K * jc + t] : 0.5;
        const float a = (float)pd, b = (float)(1.0 - pd);
        pf[k * PS + jj] = a;
        pf[K * PS + k * PS + jj] = b;
        float h, l;
        tf32_split(a, h, l);
        *(float *)(buf + C::PK_QB + kmaj_off(jj, k, C::QB_LBO)) = h;
        *(float *)(buf + C::PK_QB + kmaj_off(jj, C::KP + k, C::QB_LBO)) = l;
        tf32_split(b, h, l);
        *(float *)(buf + C::PK_QB + kmaj_off(MQ_JC + jj, k, C::QB_LBO)) = h;
        *(float *)(buf + C::PK_QB + kmaj_off(MQ_JC + jj, C::KP + k, C::QB_LBO)) = l;
        /* gradient B blocks [p_hi | p_lo] and [p_hi | 0]: element (row n, SNP jj) at granule jj / 8,
         * half-word jj % 8 */
        uint16_t *g0 = (uint16_t *)(buf + C::PK_DG + bblk_off(k, jj >> 3, C::DG_LBO)) + (jj & 7);
        uint16_t *g0l = (uint16_t *)(buf + C::PK_DG + bblk_off(K + k, jj >> 3, C::DG_LBO)) + (jj & 7);
        uint16_t *g1 = (uint16_t *)(buf + C::PK_DG + C::DGB_BYTES + bblk_off(k, jj >> 3, C::DG_LBO)) + (jj & 7);
        uint16_t hi, lo;
        bf16_split(a, hi, lo);
        *g0 = hi;
        *g0l = lo;
        *g1 = hi;
    }
    __syncthreads();
    /* pair-product tiles: task (term, kc, nn) writes column nn's pair (diagonal pairs first, then the
     * diagonal residual rows), 8 SNPs of k-chunk kc, at kc*16N + 16nn */
    for (int t = tid; t < 2 * 4 * N; t += 128) {
        const int term = t / (4 * N), rem = t - term * 4 * N;
        const int kc = rem / N, nn = rem - kc * N;
        uint32_t w[4] = {0u, 0u, 0u, 0u};
        if (nn < T + K) {
            int ka, kb;
            if (nn < T) col_pair(K, nn, ka, kb);
            else ka = kb = nn - T;
            const float *src = pf + term * K * PS + kc * 8;
            const float4 a0 = *(const float4 *)(src + ka * PS), a1 = *(const float4 *)(src + ka * PS + 4);
            const float4 b0 = *(const float4 *)(src + kb * PS), b1 = *(const float4 *)(src + kb * PS + 4);
            if (nn < T) {   /* pair products */
                w[0] = pack_bf16x2(a0.x * b0.x, a0.y * b0.y);
                w[1] = pack_bf16x2(a0.z * b0.z, a0.w * b0.w);
                w[2] = pack_bf16x2(a1.x * b1.x, a1.y * b1.y);
                w[3] = pack_bf16x2(a1.z * b1.z, a1.w * b1.w);
            } else {        /* the rounding residuals of the diagonal pair products */
                w[0] = pack_bf16x2_res(a0.x * b0.x, a0.y * b0.y);
                w[1] = pack_bf16x2_res(a0.z * b0.z, a0.w * b0.w);
                w[2] = pack_bf16x2_res(a1.x * b1.x, a1.y * b1.y);
                w[3] = pack_bf16x2_res(a1.z * b1.z, a1.w * b1.w);
            }
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

/* K-step ks (0 or 1) of a chunk's gradient MMAs (one thread), a fresh sum into TMEM columns
 * COL_DG.. that K-step 0 starts:
 *   DZ0 x [hi | lo block]   dz_hi p_hi in columns 0..K-1, dz_hi p_lo in K..2K-1
 *   DZ1 x [hi | 0 block]    dz_lo p_hi added into columns 0..K-1
 * a_dz: the A tile DZ0 (DZ1 follows at +A_BYTES); b_base: the package's two gradient B blocks.
 * Shared by both sides (P side: p -> q). */
template <int K, uint32_t A_BYTES, uint32_t A_LBO, uint32_t DGB_BYTES, uint32_t DG_LBO>
__device__ __forceinline__ void issue_grad(uint32_t tmem_dg, uint32_t a_dz, uint32_t b_base, int ks, uint32_t first_acc)
{
    constexpr uint32_t id = idesc_bf16_f32(128, DGShape<K>::NDG);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const uint64_t ad = umma_desc_kmajor(a_dz + t * A_BYTES + ks * 2 * A_LBO, A_LBO, 128);
        const uint64_t bd = umma_desc_kmajor(b_base + t * DGB_BYTES + ks * 2 * DG_LBO, DG_LBO, 128);
        tc_mma_bf16(tmem_dg, ad, bd, id, (t > 0 || ks > 0) ? 1u : first_acc);
    }
}

/* Warp roles: warps 0-3 are producers (thread = accumulator row), warp 4 is the controller
 * (bulk copies, genotype staging, MMA issue).  No CTA-wide barrier inside the chunk loop: the
 * roles hand off through mbarriers.  Every wait is bounded; after a failed wait a thread sets
 * the shared abort flag and both roles run to the end without waiting.  The controller issues
 * the global loads of a chunk's genotypes one chunk before it stages them, so their latency does
 * not hold up its MMA issue (Q sweep at I=200k, J=100k, K=8: 27.8 -> 25.7 ms). */
constexpr int MQ_CTA = MQ_THREADS + 32;

template <int K>
__global__ void __launch_bounds__(MQ_CTA, (K <= 8 ? 3 : (K <= 12 ? 2 : 1)))
k_sweep_q_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
                const double *__restrict__ q, const uint8_t *__restrict__ pkg, int64_t jslice,
                double *__restrict__ out, int *__restrict__ err)
{
    using C = MQ<K>;
    constexpr int T = C::T, N = C::N, E = C::E;
    extern __shared__ __align__(1024) uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    /* qp ready, qp consumed (4 warps), A tiles written (4 warps), the chunk's Hessian and
     * gradient MMAs done, G staged [2], package [NPKG], first half of the A tiles written (4
     * warps), the first K-step's MMAs done */
    __shared__ uint64_t mbar[8 + MQ_NPKG];
    __shared__ uint32_t tmem_holder;
    __shared__ volatile int abort_flag;
    uint64_t *bar_qp = &mbar[0], *bar_qfree = &mbar[1], *bar_afull = &mbar[2], *bar_h = &mbar[3];
    uint64_t *bar_g = &mbar[4], *bar_p = &mbar[6], *bar_ahalf = &mbar[6 + MQ_NPKG], *bar_h0 = &mbar[7 + MQ_NPKG];

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
        mbar_init(bar_ahalf, 4);
        mbar_init(bar_h0, 1);
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
         * individuals) into a0 / a1 one chunk before the staging, where lanes 2m, 2m+1 exchange and
         * write pair m interleaved as [byte][2] */
        uint4 a0 = make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u), a1 = a0;
        auto load_g = [&](int c) {
            const int64_t jc = j0 + (int64_t)c * MQ_JC;
            a0 = a1 = make_uint4(0x55555555u, 0x55555555u, 0x55555555u, 0x55555555u);
            if (jc + lane < j1) {
                const uint4 *src = (const uint4 *)(bed + (size_t)(jc + lane) * pitch + (size_t)(i0 / 4));
                a0 = __ldg(src);
                a1 = __ldg(src + 1);
            }
        };
        auto stage_g = [&](int c) {   /* the loaded genotypes of chunk c */
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
        if (nchunk > 0) { load_g(0); stage_g(0); }
        if (nchunk > 1) { load_g(1); stage_g(1); }
        if (nchunk > 2) load_g(2);
        if (nchunk > 0 && wait(&bar_p[0], 0u) && leader) {
            tc_fence_after_sync();
            issue_qp<K>(tmem, sm, sm + C::OFF_PKG);
            tc_commit(bar_qp);
        }
        constexpr uint32_t idesc = idesc_bf16_f32(128, N);
        /* K-step ks of chunk c's Hessian and gradient MMAs (leader thread) */
        auto issue_ks = [&](int c, int ks) {
            tc_fence_after_sync();
            const uint8_t *pk = sm + C::OFF_PKG + (c % MQ_NPKG) * C::PKG;
            const uint32_t abase = smem_u32(At), bbase = smem_u32(pk);
#pragma unroll
            for (int term = 0; term < 2; ++term) {
                const uint64_t ad = umma_desc_kmajor(abase + term * C::A_BYTES + ks * 2 * C::A_LBO, C::A_LBO, C::A_SBO);
                const uint64_t bd = umma_desc_kmajor(bbase + term * C::B_BYTES + ks * 2 * C::B_LBO, C::B_LBO, C::B_SBO);
                tc_mma_bf16(tmem + C::COL_H, ad, bd, idesc, (c % MX_HBLOCK != 0 || term > 0 || ks > 0) ? 1u : 0u);
            }
            issue_grad<K, C::A_BYTES, C::A_LBO, C::DGB_BYTES, C::DG_LBO>(tmem + C::COL_DG, abase + 2 * C::A_BYTES,
                                                                         bbase + C::PK_DG, ks, (c % MX_DRAIN != 0) ? 1u : 0u);
        };
        for (int c = 0; c < nchunk && ok; ++c) {
            /* the first K-step (SNPs 0-15) of chunk c as soon as the producers wrote it, so its MMAs
             * run while they compute the second */
            if (wait(bar_ahalf, (uint32_t)(c & 1)) && leader) {
                issue_ks(c, 0);
                tc_commit(bar_h0);
            }
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
            /* the second K-step once the producers wrote the rest of chunk c's A tiles */
            if (wait(bar_afull, (uint32_t)(c & 1))) {
                if (leader) {
                    issue_ks(c, 1);
                    tc_commit(bar_h);
                }
                /* the producers are done with G buffer c & 1: stage chunk c+2 into it */
                if (c + 2 < nchunk) stage_g(c + 2);
                if (c + 3 < nchunk) load_g(c + 3);
            }
            /* package c is free once the MMAs of chunk c are done: fetch chunk c+NPKG into it */
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
        uint32_t dst = dither_seed(i, blockIdx.y);   /* rounding dither of this row's Hessian weights */
        double gd[K], dd[K], zsd = 0.0;   /* gradient sum_j (z1 - z2) p_k, Hessian diagonal, sum_j z2 */
#pragma unroll
        for (int k = 0; k < K; ++k) gd[k] = dd[k] = 0.0;
        /* the last chunk whose MMAs completed: its Hessian diagonal (columns 0..K-1 of the Hessian
         * accumulator, cleared for the next chunk) and its gradient sums, into FP64 */
        auto drain_dg = [&]() { drain_chunk<K, C::NDG>(tmem + lane_base, C::COL_H, C::COL_DG, dd, gd); };
        for (int c = 0; c < nchunk && ok; ++c) {
            const uint8_t *Gb = sm + C::OFF_G + (c & 1) * C::GBUF;
            /* chunk c-1's first K-step MMAs are done: the A tiles' first half is free */
            if (c > 0 && !wait(bar_h0, (uint32_t)((c - 1) & 1))) break;
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
            const uint16_t *G2 = (const uint16_t *)Gb + (tid >> 2);
            float2 zs = make_float2(0.f, 0.f);
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
                uint32_t w1p[4], w2p[4], d0p[4], d1p[4];
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
                    const float2 dz = __ffma2_rn(z2, make_float2(-1.f, -1.f), z1);
                    zs = __fadd2_rn(zs, z2);
                    const uint32_t rb = dither_step(dst);
                    w1p[e] = pack_bf16x2_dither(w1.x, w1.y, rb);
                    w2p[e] = pack_bf16x2_dither(w2.x, w2.y, rb);
                    /* dz = hi + lo in BF16: hi rounded to nearest, lo the BF16 of the remainder */
                    const uint32_t h = pack_bf16x2(dz.x, dz.y);
                    const float2 hf = make_float2(__uint_as_float(h << 16), __uint_as_float(h & 0xFFFF0000u));
                    const float2 lr = __fadd2_rn(dz, make_float2(-hf.x, -hf.y));
                    d0p[e] = h;
                    d1p[e] = pack_bf16x2(lr.x, lr.y);
                }
                *(uint4 *)(At + kc * C::A_LBO + 16 * tid) = make_uint4(w1p[0], w1p[1], w1p[2], w1p[3]);
                *(uint4 *)(At + C::A_BYTES + kc * C::A_LBO + 16 * tid) = make_uint4(w2p[0], w2p[1], w2p[2], w2p[3]);
                *(uint4 *)(At + 2 * C::A_BYTES + kc * C::A_LBO + 16 * tid) = make_uint4(d0p[0], d0p[1], d0p[2], d0p[3]);
                *(uint4 *)(At + 3 * C::A_BYTES + kc * C::A_LBO + 16 * tid) = make_uint4(d1p[0], d1p[1], d1p[2], d1p[3]);
                if (kc == 1) {
                    /* all of chunk c-1's MMAs are done: its diagonal and gradient sums (and, at a block
                     * boundary, the Hessian block), and the A tiles' second half is free */
                    if (c > 0 && wait(bar_h, (uint32_t)((c - 1) & 1))) {
                        if (c % MX_DRAIN == 0) drain_dg();
                        if (c % MX_HBLOCK == 0) {   /* the Hessian block of chunks c-MX_HBLOCK .. c-1 */
                            tc_fence_after_sync();
                            hess_drain<K, N, T>(tmem + lane_base + C::COL_H,
                                                out + ((size_t)blockIdx.y * I + (valid ? i : 0)) * E, c == MX_HBLOCK, valid);
                            tc_fence_before_sync();
                        }
                    }
                    /* the first K-step's A tiles are written and chunk c-1 drained: its MMAs may start */
                    fence_async_smem();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(bar_ahalf);
                }
            }
            zsd += (double)zs.x + (double)zs.y;
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_afull);
        }
        if (nchunk > 0 && wait(bar_h, (uint32_t)((nchunk - 1) & 1))) drain_dg();   /* the last chunk */
        if (valid) {
            double *o = out + ((size_t)blockIdx.y * I + i) * E;
#pragma unroll
            for (int k = 0; k < K; ++k) o[T + k] = ok ? gd[k] + zsd : __longlong_as_double(0x7ff8000000000000LL);
        }
        /* every role is past its loop; the controller gives MMAs and copies still in flight a
         * bounded moment (after a failure) before the TMEM is read and released */
        ok = __syncthreads_and(ok);
        __syncthreads();
        tc_fence_after_sync();
        if (nchunk > 0) {
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + lane_base + C::COL_H + (uint32_t)c0, v);
                if (valid) {   /* the last accumulation block, added to the drained ones */
                    double *o = out + ((size_t)blockIdx.y * I + i) * E;
                    const bool first = nchunk <= MX_HBLOCK;
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        if (c0 + e >= K && c0 + e < T + K) {
                            double &x = o[col_out(K, c0 + e)];
                            x = ok ? (first ? (double)v[e] : x + (double)v[e]) : __longlong_as_double(0x7ff8000000000000LL);
                        }
                }
            }
        }
        if (valid) {   /* the diagonal: per-chunk sums (FP64 across chunks) plus the residual columns */
            double *o = out + ((size_t)blockIdx.y * I + i) * E;
            if (nchunk == 0) {
                for (int e = 0; e < T; ++e) o[e] = 0.0;
            } else {
#pragma unroll
                for (int k = 0; k < K; ++k)
                    o[k * (k + 1) / 2 + k] = ok ? o[k * (k + 1) / 2 + k] + dd[k] : __longlong_as_double(0x7ff8000000000000LL);
            }
        }
        tc_fence_before_sync();
        __syncthreads();
        return;
    }
    /* controller: the same three CTA-wide barriers as the producers' epilogue */
    ok = __syncthreads_and(ok);
    if (!ok && tid == MQ_THREADS) {
        mbar_wait_bounded(bar_h0, 0u, 1024u);
        mbar_wait_bounded(bar_h0, 1u, 1024u);
        mbar_wait_bounded(bar_h, 0u, 1024u);
        mbar_wait_bounded(bar_h, 1u, 1024u);
        mbar_wait_bounded(bar_qp, 0u, 1024u);
        mbar_wait_bounded(bar_qp, 1u, 1024u);
        for (int b = 0; b < MQ_NPKG; ++b) { mbar_wait_bounded(&bar_p[b], 0u, 1024u); mbar_wait_bounded(&bar_p[b], 1u, 1024u); }
    }
    __syncthreads();
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 4) tmem_dealloc_warp(tmem, C::NCOLS);
}

/* ===================================================================== P side
 *
 * Mirror of the Q side with the roles of the axes swapped: rows = 128 SNPs, reduction over
 * chunks of 32 individuals.  Per chunk:
 *   qp, om     D[128 x 32] = Ptile * Qchunk^T and (1-P)tile * Qchunk^T, TF32 split form;
 *   Hessian    D[128 x N] += C * QQ^T in BF16, C = nm (g/qp^2 + (2-g)/(1-qp)^2), diagonal pairs
 *              in the first K columns, read, added into FP64 and cleared every MX_DRAIN chunks;
 *   gradient   D[128 x NDG] = dz_hi * [q_hi | q_lo]^T + dz_lo * [q_hi | 0]^T (the gradient
 *              sum_i dz q_k, dz = nm (g/qp - (2-g)/(1-qp))), afresh every MX_DRAIN chunks and
 *              added into FP64;
 * and per cell on the CUDA cores the code (from the thread's own genotype word), one reciprocal,
 * C, dz and its BF16 split.  The Q-derived tiles of each chunk (QQ in BF16, Q split into TF32
 * hi / lo, the gradient B blocks, q in FP32 for the EM mode) are built once per sweep by
 * k_p_pack and fetched with one bulk copy per chunk. */

constexpr int MP_IC = 32;          /* individuals per chunk = 2 BF16 MMA K-steps */
constexpr int MP_THREADS = 128;    /* one thread per SNP = accumulator row */
constexpr int MP_NPKG = 3;

template <int K>
struct MP {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int N = ((T + K + 15) / 16) * 16;          /* pairs + diagonal residuals */
    static constexpr int KP = ((K + 7) / 8) * 8;
    static constexpr int NDG = DGShape<K>::NDG;
    static constexpr uint32_t COL_OM = 32, COL_H = 64;          /* TMEM: qp 0..31, om 32..63, Hessian */
    static constexpr uint32_t COL_DG = COL_H + N;               /* gradient accumulator */
    static constexpr uint32_t NCOLS = tmem_cols_for(COL_DG + NDG);
    static constexpr int E = T + K;
    static constexpr uint32_t A_BYTES = 128 * MP_IC * 2;        /* one BF16 A tile (C, DZ0, DZ1): 8 KB */
    static constexpr uint32_t B_BYTES = N * MP_IC * 2;          /* BF16 QQ tile */
    static constexpr uint32_t PA_BYTES = 128 * 2 * KP * 4;      /* TF32 P tile [hi | lo] (and 1-P) */
    static constexpr uint32_t QB_BYTES = MP_IC * 2 * KP * 4;    /* TF32 Q chunk [hi | lo] */
    static constexpr uint32_t DGB_BYTES = NDG * MP_IC * 2;      /* one BF16 B block of the gradient MMAs */
    static constexpr int QS = MP_IC + 4;                        /* FP32 q row stride (floats) */
    /* package: [QQ | TF32 Q | FP32 q (EM mode) | 1 - sum q | gradient blocks [q_hi | q_lo], [q_hi | 0]] */
    static constexpr uint32_t PK_QB = B_BYTES;
    static constexpr uint32_t PK_QF = PK_QB + QB_BYTES;
    static constexpr uint32_t PK_S = PK_QF + K * QS * 4;         /* 1 - sum_k q_k per individual */
    static constexpr uint32_t PK_DG = PK_S + MP_IC * 4;
    static constexpr uint32_t PKG = PK_DG + 2 * DGB_BYTES;
    static constexpr uint32_t OFF_A = 0;                        /* C, DZ0, DZ1 */
    static constexpr uint32_t OFF_PKG = 3 * A_BYTES;
    static constexpr uint32_t OFF_PA = OFF_PKG + MP_NPKG * PKG; /* P tile, then (1-P) tile */
    static constexpr uint32_t OFF_TAB = OFF_PA + 2 * PA_BYTES;
    static constexpr uint32_t SMEM = OFF_TAB + 128 * 16 + 1024;
    static constexpr uint32_t A_LBO = 2048, A_SBO = 128;
    static constexpr uint32_t B_LBO = 16 * N, B_SBO = 128;
    static constexpr uint32_t PA_LBO = 2048, QB_LBO = 512, T_SBO = 128;
    static constexpr uint32_t DG_LBO = 16 * NDG;
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
        /* gradient B blocks [q_hi | q_lo] and [q_hi | 0]: element (row n, individual ii) at granule
         * ii / 8, half-word ii % 8 */
        uint16_t *g0 = (uint16_t *)(buf + C::PK_DG + bblk_off(k, ii >> 3, C::DG_LBO)) + (ii & 7);
        uint16_t *g0l = (uint16_t *)(buf + C::PK_DG + bblk_off(K + k, ii >> 3, C::DG_LBO)) + (ii & 7);
        uint16_t *g1 = (uint16_t *)(buf + C::PK_DG + C::DGB_BYTES + bblk_off(k, ii >> 3, C::DG_LBO)) + (ii & 7);
        uint16_t hi, lo;
        bf16_split(a, hi, lo);
        *g0 = hi;
        *g0l = lo;
        *g1 = hi;
    }
    __syncthreads();
    /* QQ tile: task (kc, nn) writes column nn's pair (diagonal pairs first, then the diagonal
     * residual rows), 8 individuals of k-chunk kc, at kc*16N + 16nn */
    for (int t = tid; t < 4 * N; t += 128) {
        const int kc = t / N, nn = t - kc * N;
        uint32_t w[4] = {0u, 0u, 0u, 0u};
        if (nn < T + K) {
            int ka, kb;
            if (nn < T) col_pair(K, nn, ka, kb);
            else ka = kb = nn - T;
            const float *src = qf + kc * 8;
            const float4 a0 = *(const float4 *)(src + ka * C::QS), a1 = *(const float4 *)(src + ka * C::QS + 4);
            const float4 b0 = *(const float4 *)(src + kb * C::QS), b1 = *(const float4 *)(src + kb * C::QS + 4);
            if (nn < T) {   /* pair products */
                w[0] = pack_bf16x2(a0.x * b0.x, a0.y * b0.y);
                w[1] = pack_bf16x2(a0.z * b0.z, a0.w * b0.w);
                w[2] = pack_bf16x2(a1.x * b1.x, a1.y * b1.y);
                w[3] = pack_bf16x2(a1.z * b1.z, a1.w * b1.w);
            } else {        /* the rounding residuals of the diagonal pair products */
                w[0] = pack_bf16x2_res(a0.x * b0.x, a0.y * b0.y);
                w[1] = pack_bf16x2_res(a0.z * b0.z, a0.w * b0.w);
                w[2] = pack_bf16x2_res(a1.x * b1.x, a1.y * b1.y);
                w[3] = pack_bf16x2_res(a1.z * b1.z, a1.w * b1.w);
            }
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
    /* qp ready, qp consumed (4 warps), A tiles written (4 warps), the chunk's MMAs done, package
     * landed [3], package read (4 warps, EM sums only) [3], first half of the A tiles written (4
     * warps), the first K-step's MMAs done */
    __shared__ uint64_t mbar[6 + 2 * MP_NPKG];
    __shared__ uint32_t tmem_holder;
    __shared__ volatile int abort_flag;
    uint64_t *bar_qp = &mbar[0], *bar_qfree = &mbar[1], *bar_afull = &mbar[2], *bar_h = &mbar[3], *bar_p = &mbar[4];
    uint64_t *bar_read = &mbar[4 + MP_NPKG], *bar_ahalf = &mbar[4 + 2 * MP_NPKG], *bar_h0 = &mbar[5 + 2 * MP_NPKG];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp < 4;
    const int64_t j = (int64_t)blockIdx.x * 128 + tid;
    const bool valid = producer && j < J;
    const int64_t ia = (int64_t)blockIdx.y * islice;    /* islice is a multiple of MP_IC */
    const int64_t ib = min(I, ia + islice);
    const int nchunk = (int)((ib - ia + MP_IC - 1) / MP_IC);
    const uint8_t *pk0 = pkg + (size_t)(ia / MP_IC) * C::PKG;
    uint8_t *At = sm + C::OFF_A;
    double diag_keep[K];   /* producers: the Hessian diagonal, kept for the epilogue */
#pragma unroll
    for (int k = 0; k < K; ++k) diag_keep[k] = 0.0;

    if (warp == 4) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        mbar_init(bar_qp, 1);
        mbar_init(bar_qfree, 4);
        mbar_init(bar_afull, 4);
        mbar_init(bar_h, 1);
        for (int b = 0; b < MP_NPKG; ++b) mbar_init(&bar_p[b], 1);
        for (int b = 0; b < MP_NPKG; ++b) mbar_init(&bar_read[b], 4);
        mbar_init(bar_ahalf, 4);
        mbar_init(bar_h0, 1);
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
        /* K-step ks of chunk c's Hessian and gradient MMAs (leader thread) */
        auto issue_ks = [&](int c, int ks) {
            const uint8_t *pk = sm + C::OFF_PKG + (c % MP_NPKG) * C::PKG;
            const uint32_t abase = smem_u32(At), bbase = smem_u32(pk);
            const uint64_t ad = umma_desc_kmajor(abase + ks * 2 * C::A_LBO, C::A_LBO, C::A_SBO);
            const uint64_t bd = umma_desc_kmajor(bbase + ks * 2 * C::B_LBO, C::B_LBO, C::B_SBO);
            tc_mma_bf16(tmem + C::COL_H, ad, bd, idesc, (c % MX_HBLOCK != 0 || ks > 0) ? 1u : 0u);
            issue_grad<K, C::A_BYTES, C::A_LBO, C::DGB_BYTES, C::DG_LBO>(tmem + C::COL_DG, abase + C::A_BYTES,
                                                                         bbase + C::PK_DG, ks, (c % MX_DRAIN != 0) ? 1u : 0u);
        };
        for (int c = 0; c < nchunk && ok; ++c) {
            if constexpr (!EMS) {   /* the first K-step (individuals 0-15) as soon as it is written */
                if (wait(bar_ahalf, (uint32_t)(c & 1)) && leader) {
                    tc_fence_after_sync();
                    issue_ks(c, 0);
                    tc_commit(bar_h0);
                }
            }
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
            /* the second K-step once the producers wrote the rest of the chunk's A tiles */
            if (wait(bar_afull, (uint32_t)(c & 1)) && leader) {
                tc_fence_after_sync();
                issue_ks(c, 1);
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
        /* gradient sum_i dz q_k (EM mode: sum_i nm g q_k / qp), Hessian diagonal, and the EM mode's
         * second sums */
        uint32_t dst = dither_seed(j, blockIdx.y);   /* rounding dither of this row's Hessian weights */
        double gd[K], dd[EMS ? 1 : K], hd[EMS ? K : 1];
#pragma unroll
        for (int k = 0; k < K; ++k) gd[k] = 0.0;
#pragma unroll
        for (int k = 0; k < (EMS ? 1 : K); ++k) dd[k] = 0.0;
#pragma unroll
        for (int k = 0; k < (EMS ? K : 1); ++k) hd[k] = 0.0;
        /* the last chunk whose MMAs completed: its Hessian diagonal (columns 0..K-1 of the Hessian
         * accumulator, cleared for the next chunk) and its gradient sums, into FP64 */
        auto drain_dg = [&]() {
            if constexpr (!EMS) drain_chunk<K, C::NDG>(tmem + lane_base, C::COL_H, C::COL_DG, dd, gd);
        };
        for (int c = 0; c < nchunk && ok; ++c) {
            const uint8_t *pk = sm + C::OFF_PKG + (c % MP_NPKG) * C::PKG;
            const float *Qf = (const float *)(pk + C::PK_QF);
            const float2 *Sres = (const float2 *)(pk + C::PK_S);
            if constexpr (!EMS) {   /* chunk c-1's first K-step MMAs are done: the A tiles' first half is free */
                if (c > 0 && !wait(bar_h0, (uint32_t)((c - 1) & 1))) break;
            }
            /* qp / om of the chunk's 32 individuals, read in two halves of 16 columns
             * (individuals 0-15, then 16-31) to keep the producer within its registers */
            uint32_t rq[16], ro[16];
            if (!wait(bar_qp, (uint32_t)(c & 1))) break;
            tc_fence_after_sync();
            tmem_ld16_raw(tmem + lane_base, rq);
            tmem_ld16_raw(tmem + lane_base + C::COL_OM, ro);
            tmem_wait_ld();
            if (!wait(&bar_p[c % MP_NPKG], (uint32_t)((c / MP_NPKG) & 1))) break;
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
                uint32_t cp[4], d0p[4], d1p[4];
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
                        const float2 dz = __ffma2_rn(z2, make_float2(-1.f, -1.f), z1);   /* nm (g/qp - (2-g)/(1-qp)) */
                        cp[e] = pack_bf16x2_dither(cw.x, cw.y, dither_step(dst));
                        /* dz = hi + lo in BF16: hi rounded to nearest, lo the BF16 of the remainder */
                        const uint32_t h = pack_bf16x2(dz.x, dz.y);
                        const float2 hf = make_float2(__uint_as_float(h << 16), __uint_as_float(h & 0xFFFF0000u));
                        const float2 lr = __fadd2_rn(dz, make_float2(-hf.x, -hf.y));
                        d0p[e] = h;
                        d1p[e] = pack_bf16x2(lr.x, lr.y);
                    }
                }
                if constexpr (!EMS) {
                    *(uint4 *)(At + kc * C::A_LBO + 16 * tid) = make_uint4(cp[0], cp[1], cp[2], cp[3]);
                    *(uint4 *)(At + C::A_BYTES + kc * C::A_LBO + 16 * tid) = make_uint4(d0p[0], d0p[1], d0p[2], d0p[3]);
                    *(uint4 *)(At + 2 * C::A_BYTES + kc * C::A_LBO + 16 * tid) = make_uint4(d1p[0], d1p[1], d1p[2], d1p[3]);
                    if (kc == 1) {   /* as on the Q side: drain chunk c-1, then release the first K-step */
                        if (c > 0 && wait(bar_h, (uint32_t)((c - 1) & 1))) {
                            if (c % MX_DRAIN == 0) drain_dg();
                            if (c % MX_HBLOCK == 0) {
                                tc_fence_after_sync();
                                hess_drain<K, N, T>(tmem + lane_base + C::COL_H,
                                                    out + ((size_t)blockIdx.y * J + (valid ? j : 0)) * E, c == MX_HBLOCK, valid);
                                tc_fence_before_sync();
                            }
                        }
                        fence_async_smem();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(bar_ahalf);
                    }
                } else {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    const float4 q0 = *(const float4 *)(Qf + k * C::QS + kc * 8);
                    const float4 q1 = *(const float4 *)(Qf + k * C::QS + kc * 8 + 4);
                    gk[k] = __ffma2_rn(zz[0], make_float2(q0.x, q0.y), gk[k]);
                    gk[k] = __ffma2_rn(zz[1], make_float2(q0.z, q0.w), gk[k]);
                    gk[k] = __ffma2_rn(zz[2], make_float2(q1.x, q1.y), gk[k]);
                    gk[k] = __ffma2_rn(zz[3], make_float2(q1.z, q1.w), gk[k]);
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
            if constexpr (EMS) {
#pragma unroll
                for (int k = 0; k < K; ++k) gd[k] += (double)gk[k].x + (double)gk[k].y;
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
            if (nchunk > 0 && wait(bar_h, (uint32_t)((nchunk - 1) & 1))) drain_dg();   /* the last chunk */
            if (valid) {
                double *o = out + ((size_t)blockIdx.y * J + j) * E;
#pragma unroll
                for (int k = 0; k < K; ++k) o[T + k] = ok ? gd[k] : __longlong_as_double(0x7ff8000000000000LL);
            }
        }
        if constexpr (!EMS) {   /* the epilogue below writes the diagonal from these */
#pragma unroll
            for (int k = 0; k < K; ++k) diag_keep[k] = dd[k];
        }
    }
    ok = __syncthreads_and(ok);
    if (!ok && tid == MP_THREADS) {
        if constexpr (!EMS) { mbar_wait_bounded(bar_h0, 0u, 1024u); mbar_wait_bounded(bar_h0, 1u, 1024u); }
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
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + lane_base + C::COL_H + (uint32_t)c0, v);
                if (valid) {   /* the last accumulation block, added to the drained ones */
                    double *o = out + ((size_t)blockIdx.y * J + j) * E;
                    const bool first = nchunk <= MX_HBLOCK;
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        if (c0 + e >= K && c0 + e < T + K) {
                            double &x = o[col_out(K, c0 + e)];
                            x = ok ? (first ? (double)v[e] : x + (double)v[e]) : __longlong_as_double(0x7ff8000000000000LL);
                        }
                }
            }
        } else if (valid) {
            double *o = out + ((size_t)blockIdx.y * J + j) * E;
            for (int e = 0; e < T; ++e) o[e] = 0.0;
        }
        if (valid && nchunk > 0) {   /* the diagonal: per-chunk sums (FP64 across chunks) plus the residual columns */
            double *o = out + ((size_t)blockIdx.y * J + j) * E;
#pragma unroll
            for (int k = 0; k < K; ++k)
                o[k * (k + 1) / 2 + k] = ok ? o[k * (k + 1) / 2 + k] + diag_keep[k] : __longlong_as_double(0x7ff8000000000000LL);
        }
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 4) tmem_dealloc_warp(tmem, C::NCOLS);
}

/* ===================================================================== loglik on the tensor cores
 * loglikelihood_loop_skipmissing (loops.jl:517-539) with qp from tcgen05 in exact pieces.
 *
 * Every q and p is split into three BF16 limbs on fixed grids: x0 = round(x 2^8) 2^-8,
 * x1 = round((x - x0) 2^16) 2^-16, x2 = round((x - x0 - x1) 2^24) 2^-24 (each an integer of at most
 * 8 bits times a power of two, so exact in BF16; |x - x0 - x1 - x2| <= 2^-25).  Two accumulators
 * per cell:
 *   L01 = sum_k q0 p0 + q0 p1 + q1 p0   a multiple of 2^-24 below 1,
 *   L2  = sum_k q0 p2 + q1 p1 + q2 p0   a multiple of 2^-32 below 2^-12,
 * so every product and partial sum of either accumulator is exactly representable in FP32 and
 * the tensor core's accumulation (which rounds toward zero when it has to round) never rounds.
 * On the CUDA cores qp = L01 + L2 and 1 - qp = (1 - L01) - L2 (1 - L01 exact) are then rounded
 * to nearest once each: unbiased, and 1 - qp keeps its relative accuracy as qp -> 1.  (A single
 * TF32 accumulation biases every qp low by about half an ulp, which moves the log-likelihood
 * by ~1e-7 relative.)  The limbs' own rounding (2^-25 absolute, to nearest) and the dropped
 * products q1 p2, q2 p1, q2 p2 are of random sign.
 *
 * Per cell the CUDA cores then form qp^g (1-qp)^(2-g) (1 when missing) and fold it into a
 * running product: four cells' factors multiplied in FP32 (with an exact 2^60 scale), one FP64
 * multiply per four cells, the exponent moved into an integer every 16 cells, one log per thread
 * at the end.
 *
 * Roles as in the sweeps: warps 0-3 producers (thread = SNP = TMEM lane), warp 4 controller
 * (bulk copies of the per-chunk individual packages, MMA issue).  TMEM holds two chunk buffers
 * of [L01 | L2] x 32 individuals, so the MMAs of chunk c+1 run while chunk c is consumed. */
constexpr int LT_IC = 32;          /* individuals per chunk (MMA N) */
constexpr int LT_NPKG = 4;         /* package buffers */

template <int K>
struct LT {
    static constexpr int KP = ((K + 7) / 8) * 8;                /* limb width (granules of 8) */
    static constexpr int R = ((3 * KP + 15) / 16) * 16;         /* reduction length of one accumulator */
    static constexpr int NG = R / 8;                            /* granules per row */
    static constexpr uint32_t A_BYTES = 128 * R * 2;            /* one P-limb tile (128 SNPs) */
    static constexpr uint32_t B_BYTES = LT_IC * R * 2;          /* one Q-limb tile (32 individuals) */
    static constexpr uint32_t PKG = 2 * B_BYTES;                /* [B01 | B2] */
    static constexpr uint32_t OFF_A = 0;                        /* A01, A2 */
    static constexpr uint32_t OFF_PKG = 2 * A_BYTES;
    static constexpr uint32_t SMEM = OFF_PKG + LT_NPKG * PKG + 1024;
    static constexpr uint32_t A_LBO = 128 * 16, B_LBO = LT_IC * 16, SBO = 128;
    static constexpr uint32_t NCOLS = 128;                      /* 2 buffers x [L01 | L2] x 32 */
    static_assert(PKG % 16 == 0 && OFF_PKG % 1024 == 0, "bulk copies and descriptors need alignment");
};

/* the three BF16 limbs of x in [0, 1] (exact conversions: each limb has at most 8 significant bits) */
__device__ __forceinline__ void limbs3(double x, uint16_t &l0, uint16_t &l1, uint16_t &l2)
{
    const double a = rint(x * 256.0) * (1.0 / 256.0);
    const double r = x - a;
    const double b = rint(r * 65536.0) * (1.0 / 65536.0);
    const double c = rint((r - b) * 16777216.0) * (1.0 / 16777216.0);
    l0 = (uint16_t)(pack_bf16x2((float)a, 0.f) & 0xFFFFu);
    l1 = (uint16_t)(pack_bf16x2((float)b, 0.f) & 0xFFFFu);
    l2 = (uint16_t)(pack_bf16x2((float)c, 0.f) & 0xFFFFu);
}

/* byte offset of row r's element e in a K-major BF16 tile whose granules (8 elements of every
 * row) are lbo bytes apart */
__device__ __forceinline__ uint32_t lt_off(int r, int e, uint32_t lbo) { return (uint32_t)(e >> 3) * lbo + 16u * (uint32_t)r + 2u * (uint32_t)(e & 7); }

/* Per-chunk packages of 32 individuals: B01 = [q0 | q0 | q1], B2 = [q0 | q1 | q2] (limb widths KP,
 * zero padding).  Individuals beyond I get q = 0; their genotypes read as missing. */
template <int K>
__global__ void __launch_bounds__(128)
k_ll_pack(const double *__restrict__ q, int64_t I, uint8_t *__restrict__ pkg)
{
    using C = LT<K>;
    __shared__ __align__(16) uint8_t buf[C::PKG];
    const int tid = threadIdx.x;
    const int64_t ic = (int64_t)blockIdx.x * LT_IC;
    for (uint32_t t = tid; t < C::PKG / 16; t += 128) ((uint4 *)buf)[t] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    for (int t = tid; t < K * LT_IC; t += 128) {
        const int ii = t / K, k = t - ii * K;
        const double v = (ic + ii < I) ? q[(size_t)K * ic + t] : 0.0;
        uint16_t l0, l1, l2;
        limbs3(v, l0, l1, l2);
        uint8_t *b01 = buf, *b2 = buf + C::B_BYTES;
        *(uint16_t *)(b01 + lt_off(ii, k, C::B_LBO)) = l0;
        *(uint16_t *)(b01 + lt_off(ii, C::KP + k, C::B_LBO)) = l0;
        *(uint16_t *)(b01 + lt_off(ii, 2 * C::KP + k, C::B_LBO)) = l1;
        *(uint16_t *)(b2 + lt_off(ii, k, C::B_LBO)) = l0;
        *(uint16_t *)(b2 + lt_off(ii, C::KP + k, C::B_LBO)) = l1;
        *(uint16_t *)(b2 + lt_off(ii, 2 * C::KP + k, C::B_LBO)) = l2;
    }
    __syncthreads();
    uint4 *dst = (uint4 *)(pkg + (size_t)blockIdx.x * C::PKG);
    for (uint32_t t = tid; t < C::PKG / 16; t += 128) dst[t] = ((const uint4 *)buf)[t];
}

constexpr int LT_CTA = 128 + 32;

template <int K>
__global__ void __launch_bounds__(LT_CTA, 4)
k_loglik_mixed(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
               const double *__restrict__ p, const uint8_t *__restrict__ pkg, int64_t islice,
               double *__restrict__ partial, int *__restrict__ err)
{
    using C = LT<K>;
    extern __shared__ __align__(1024) uint8_t smraw[];
    uint8_t *sm = (uint8_t *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    /* package landed [NPKG], MMAs of buffer b done [2], buffer b read (4 warps) [2] */
    __shared__ uint64_t mbar[LT_NPKG + 4];
    __shared__ uint32_t tmem_holder;
    __shared__ volatile int abort_flag;
    __shared__ double red[4];
    uint64_t *bar_p = &mbar[0], *bar_mma = &mbar[LT_NPKG], *bar_free = &mbar[LT_NPKG + 2];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp < 4;
    const int64_t j = (int64_t)blockIdx.x * 128 + tid;
    const bool valid = producer && j < J;
    const int64_t ia = (int64_t)blockIdx.y * islice;    /* islice is a multiple of LT_IC */
    const int64_t ib = min(I, ia + islice);
    const int nchunk = (int)((ib - ia + LT_IC - 1) / LT_IC);
    const uint8_t *pk0 = pkg + (size_t)(ia / LT_IC) * C::PKG;

    if (warp == 4) tmem_alloc_warp(&tmem_holder, C::NCOLS);
    if (tid == 0) {
        for (int b = 0; b < LT_NPKG; ++b) mbar_init(&bar_p[b], 1);
        mbar_init(&bar_mma[0], 1);
        mbar_init(&bar_mma[1], 1);
        mbar_init(&bar_free[0], 4);
        mbar_init(&bar_free[1], 4);
        abort_flag = 0;
        mbar_fence_init();
    }
    if (producer) {   /* this SNP's rows of A01 = [p0 | p1 | p0] and A2 = [p2 | p1 | p0] */
        uint8_t *a01 = sm + C::OFF_A, *a2 = a01 + C::A_BYTES;
        for (int g = 0; g < C::NG; ++g) {
            *(uint4 *)(a01 + g * C::A_LBO + 16 * tid) = make_uint4(0u, 0u, 0u, 0u);
            *(uint4 *)(a2 + g * C::A_LBO + 16 * tid) = make_uint4(0u, 0u, 0u, 0u);
        }
        for (int k = 0; k < K; ++k) {
            uint16_t l0, l1, l2;
            limbs3(valid ? p[(size_t)K * j + k] : 0.0, l0, l1, l2);
            *(uint16_t *)(a01 + lt_off(tid, k, C::A_LBO)) = l0;
            *(uint16_t *)(a01 + lt_off(tid, C::KP + k, C::A_LBO)) = l1;
            *(uint16_t *)(a01 + lt_off(tid, 2 * C::KP + k, C::A_LBO)) = l0;
            *(uint16_t *)(a2 + lt_off(tid, k, C::A_LBO)) = l2;
            *(uint16_t *)(a2 + lt_off(tid, C::KP + k, C::A_LBO)) = l1;
            *(uint16_t *)(a2 + lt_off(tid, 2 * C::KP + k, C::A_LBO)) = l0;
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
    double ll = 0.0;

    if (!producer) {
        /* ---------------------------------------------------------------- controller warp */
        const bool leader = lane == 0;
        auto copy_pkg = [&](int c) {
            if (leader) {
                mbar_arrive_expect_tx(&bar_p[c % LT_NPKG], C::PKG);
                bulk_g2s(sm + C::OFF_PKG + (c % LT_NPKG) * C::PKG, pk0 + (size_t)c * C::PKG, C::PKG, &bar_p[c % LT_NPKG]);
            }
        };
        for (int c = 0; c < min(nchunk, LT_NPKG); ++c) copy_pkg(c);
        constexpr uint32_t idesc = idesc_bf16_f32(128, LT_IC);
        const uint32_t a01 = smem_u32(sm + C::OFF_A), a2 = a01 + C::A_BYTES;
        for (int c = 0; c < nchunk && ok; ++c) {
            const int b = c & 1;
            if (!wait(&bar_p[c % LT_NPKG], (uint32_t)((c / LT_NPKG) & 1))) break;
            if (c >= 2 && !wait(&bar_free[b], (uint32_t)(((c - 2) >> 1) & 1))) break;   /* buffer b was read */
            if (leader) {
                tc_fence_after_sync();
                const uint32_t b01 = smem_u32(sm + C::OFF_PKG + (c % LT_NPKG) * C::PKG), b2 = b01 + C::B_BYTES;
                const uint32_t d = tmem + (uint32_t)(b * 2 * LT_IC);
#pragma unroll
                for (int s = 0; s < C::R / 16; ++s) {
                    tc_mma_bf16(d, umma_desc_kmajor(a01 + s * 2 * C::A_LBO, C::A_LBO, C::SBO),
                                umma_desc_kmajor(b01 + s * 2 * C::B_LBO, C::B_LBO, C::SBO), idesc, s > 0 ? 1u : 0u);
                    tc_mma_bf16(d + LT_IC, umma_desc_kmajor(a2 + s * 2 * C::A_LBO, C::A_LBO, C::SBO),
                                umma_desc_kmajor(b2 + s * 2 * C::B_LBO, C::B_LBO, C::SBO), idesc, s > 0 ? 1u : 0u);
                }
                tc_commit(&bar_mma[b]);
            }
            __syncwarp();
            /* the previous chunk's MMAs are done with its package: refill that slot */
            if (c >= 1 && c - 1 + LT_NPKG < nchunk) {
                if (!wait(&bar_mma[(c - 1) & 1], (uint32_t)(((c - 1) >> 1) & 1))) break;
                fence_async_smem();
                copy_pkg(c - 1 + LT_NPKG);
            }
        }
    } else {
        /* ---------------------------------------------------------------- producer warps */
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        auto gload = [&](int c) -> uint2 {
            return valid ? __ldg((const uint2 *)(bed + (size_t)j * pitch + (size_t)((ia + (int64_t)c * LT_IC) / 4)))
                         : make_uint2(0x55555555u, 0x55555555u);
        };
        uint2 gcur = make_uint2(0x55555555u, 0x55555555u), gnext = gcur;
        if (nchunk > 0) gcur = gload(0);
        if (nchunk > 1) gnext = gload(1);
        double prod = 1.0;
        int64_t ex = 0;
        for (int c = 0; c < nchunk && ok; ++c) {
            const int b = c & 1;
            if (!wait(&bar_mma[b], (uint32_t)((c >> 1) & 1))) break;
            tc_fence_after_sync();
#pragma unroll
            for (int h = 0; h < 2; ++h) {   /* individuals 16h .. 16h+15 of the chunk */
                uint32_t ra[16], rb[16];
                tmem_ld16_raw(tmem + lane_base + (uint32_t)(b * 2 * LT_IC + 16 * h), ra);
                tmem_ld16_raw(tmem + lane_base + (uint32_t)(b * 2 * LT_IC + LT_IC + 16 * h), rb);
                tmem_wait_ld();
                if (h == 1) {   /* buffer b is read: the controller may reuse it for chunk c+2 */
                    tc_fence_before_sync();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bar_free[b]);
                }
                const uint32_t w = h ? gcur.y : gcur.x;   /* 16 individuals' codes, 2 bits each */
#pragma unroll
                for (int m4 = 0; m4 < 4; ++m4) {   /* 4 cells per step: two pairs */
                    float f[4];
#pragma unroll
                    for (int hm = 0; hm < 2; ++hm) {
                        const int e = 4 * m4 + 2 * hm;   /* the pair's first individual in this half */
                        const float2 l01 = make_float2(__uint_as_float(ra[e]), __uint_as_float(ra[e + 1]));
                        const float2 l2 = make_float2(__uint_as_float(rb[e]), __uint_as_float(rb[e + 1]));
                        const float2 qp = __fadd2_rn(l01, l2);
                        /* (1 - L01) - L2: 1 - L01 is exact, the subtraction rounds once */
                        const float2 om = __ffma2_rn(l2, make_float2(-1.f, -1.f),
                                                     __ffma2_rn(l01, make_float2(-1.f, -1.f), make_float2(1.f, 1.f)));
                        const float2 oo = __fmul2_rn(om, om), qo = __fmul2_rn(qp, om), qq = __fmul2_rn(qp, qp);
                        const int bp = 2 * e;   /* this pair's 4 code bits in w */
                        const bool lo0 = (w >> bp) & 1u, hi0 = (w >> (bp + 1)) & 1u;
                        const bool lo1 = (w >> (bp + 2)) & 1u, hi1 = (w >> (bp + 3)) & 1u;
                        f[2 * hm] = hi0 ? (lo0 ? qq.x : qo.x) : (lo0 ? 1.f : oo.x);
                        f[2 * hm + 1] = hi1 ? (lo1 ? qq.y : qo.y) : (lo1 ? 1.f : oo.y);
                    }
                    /* each pair's product (factors >= 1e-10 inside the projections' bounds: in
                     * [1e-20, 1]), then the four cells' product scaled by 2^60 (exact) so that it
                     * stays normal in FP32 ([1e-22, 1.2e18]), then into the FP64 running product */
                    const float2 ff = __fmul2_rn(make_float2(f[0], f[2]), make_float2(f[1], f[3]));
                    prod *= (double)(ff.x * (ff.y * 1152921504606846976.0f));
                }
                /* 16 cells: the product stays in [1e-88, 1e73]; move its exponent (less the four
                 * 2^60 scales) into the integer */
                const int64_t bits = __double_as_longlong(prod);
                ex += ((bits >> 52) & 0x7FF) - 1023 - 240;
                prod = __longlong_as_double((bits & ~(0x7FFLL << 52)) | (1023LL << 52));
            }
            if (c + 1 < nchunk) {
                gcur = gnext;
                if (c + 2 < nchunk) gnext = gload(c + 2);
            }
        }
        if (valid) ll = log(prod) + (double)ex * 0.69314718055994530942;
    }
    /* every role is past its loop; after a failure give MMAs and copies in flight a bounded moment */
    ok = __syncthreads_and(ok);
    if (!ok && tid == 128) {
        for (int b = 0; b < 2; ++b) { mbar_wait_bounded(&bar_mma[b], 0u, 1024u); mbar_wait_bounded(&bar_mma[b], 1u, 1024u); }
        for (int b = 0; b < LT_NPKG; ++b) { mbar_wait_bounded(&bar_p[b], 0u, 1024u); mbar_wait_bounded(&bar_p[b], 1u, 1024u); }
    }
    if (producer) {
        for (int o = 16; o > 0; o >>= 1) ll += __shfl_down_sync(0xffffffffu, ll, o);
        if (lane == 0) red[warp] = ll;
    }
    tc_fence_before_sync();
    __syncthreads();
    if (tid == 0)
        partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] =
            ok ? (red[0] + red[1]) + (red[2] + red[3]) : __longlong_as_double(0x7ff8000000000000LL);
    if (warp == 4) tmem_dealloc_warp(tmem, C::NCOLS);
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
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_loglik_mixed<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LT<K>::SMEM);
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
    k_ll_pack<K><<<(unsigned)((I + LT_IC - 1) / LT_IC), 128, 0, st>>>(q, I, pkg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_loglik_mixed<K><<<grid, LT_CTA, LT<K>::SMEM, st>>>(bed, I, J, pitch, p, pkg, pl.slice, partial, err);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_sum_partials_mixed<<<1, 1024, 0, st>>>(partial, (int64_t)pl.gx * pl.S, out);
    return cudaGetLastError();
}

template <int K>
size_t ll_pkg_bytes_t(int64_t I)
{
    return (size_t)((I + LT_IC - 1) / LT_IC) * LT<K>::PKG;
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

/* Resident CTAs per SM of one kernel, from its registers (allocated per warp in units of 256),
 * its static and dynamic shared memory (plus the per-CTA reservation), its threads and its tensor
 * memory columns (512 per SM).  The occupancy query answered one CTA per SM for all three mixed
 * kernels on a B200 while three (sweeps) and four (log-likelihood) run, as ncu's active warps
 * show, so the plans use this count, or the query's if that is larger.  0 when the kernel's
 * attributes cannot be read. */
template <typename F>
int resident_est(F *kern, int threads, uint32_t dyn_smem, uint32_t tmem_cols)
{
    cudaFuncAttributes a;
    int dev = 0, regs_sm = 0, smem_sm = 0, thr_sm = 0, res_blk = 0;
    if (cudaFuncGetAttributes(&a, kern) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&res_blk, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const int warps = (threads + 31) / 32;
    const int regs_warp = (a.numRegs * 32 + 255) / 256 * 256;
    int n = thr_sm / threads;
    if (regs_warp > 0) n = std::min(n, regs_sm / regs_warp / warps);
    n = std::min(n, smem_sm / (int)(a.sharedSizeBytes + dyn_smem + (size_t)res_blk));
    n = std::min(n, (int)(512u / tmem_cols));
    return std::max(n, 0);
}

/* resident CTAs per SM of the mixed kernels (needs prepare_mixed(K) first), cached per kernel
 * and K; 0 when it cannot be determined */
template <int K>
int resident_t(int kind)
{
    int n = 0, est = 0;
    cudaError_t e;
    if (kind == 0) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_q_mixed<K>, MQ_CTA, MQ<K>::SMEM);
        est = resident_est(k_sweep_q_mixed<K>, MQ_CTA, MQ<K>::SMEM, MQ<K>::NCOLS);
    } else if (kind == 1) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_p_mixed<K, false>, MP_CTA, MP<K>::SMEM);
        est = resident_est(k_sweep_p_mixed<K, false>, MP_CTA, MP<K>::SMEM, MP<K>::NCOLS);
    } else {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_loglik_mixed<K>, LT_CTA, LT<K>::SMEM);
        est = resident_est(k_loglik_mixed<K>, LT_CTA, LT<K>::SMEM, LT<K>::NCOLS);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    return std::max(n, est);
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

/* One CTA per 128 individuals and SNP slice.  Slices are multiples of MX_DRAIN chunks, so the
 * chunks whose FP32 gradient and diagonal sums are drained together are the same pairs for every
 * split, and another split (batch autotuning) only regroups FP64 sums. */
SweepPlan plan_sweep_q_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax)
{
    return plan_rows(I, J, sms, resident(0, K, 3), (int64_t)MX_DRAIN * MQ_JC, smax);
}

/* One CTA per 128 SNPs and individual slice (slices are multiples of MX_DRAIN chunks, as above). */
SweepPlan plan_sweep_p_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax)
{
    return plan_rows(J, I, sms, resident(1, K, 3), (int64_t)MX_DRAIN * MP_IC, smax);
}

/* One CTA per 128 SNPs and individual slice (slices are multiples of 32 individuals). */
SweepPlan plan_loglik_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax)
{
    return plan_rows(J, I, sms, resident(2, K, 4), LT_IC, smax);
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

size_t loglik_mixed_pkg_bytes(int K, int64_t I)
{
    size_t b = 0;
    ADMIX_DISPATCH_K(K, b = ll_pkg_bytes_t<KK>(I));
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
