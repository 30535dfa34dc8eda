/*
 * skfr.cu -- SKFR AIM pre-selection on the device: sparse k-means via feature ranking on the
 * imputed, standardised genotype matrix, the step run_admixture runs before the likelihood engine
 * when `sparsity` is given (driver.jl:56-69; _filter_SKFR, driver.jl:80-101).  The reference calls
 * the third-party SparseKmeansFeatureRanking.jl (compat 0.1, not vendored); this is a restatement
 * of the published method (Zhang, Lange and Xu, NeurIPS 2020) with this project's own choices,
 * pinned exactly by the CPU oracle (oracle/skfr_oracle.py), whose header states them.
 *
 * Device work, all on the handle's padded genotypes (padding coded missing):
 *   - per-SNP class counts by popcount of the code bit planes (k_skfr_counts);
 *   - k-means++ seeding distances ||x_i - x_c||^2 over all SNPs: the squared difference of every
 *     (SNP, code) to the centre in a table (k_skfr_sqtab), then a thread owns 16 individuals (one
 *     32-bit word of a column) and a slice of SKFR_SLICE SNPs, adding table entries staged in
 *     shared memory in FP64, the slice sums added in slice order (k_skfr_dist, k_skfr_dist_sum);
 *   - per iteration, the cluster sums of every SNP as exact integers: membership bit masks per
 *     16-individual word and the cluster sizes (k_skfr_masks), then per SNP and cluster but the last
 *     one popcount of the dosage bits per word and one of the missing bits per two words under the
 *     masks (k_skfr_sums, one thread per SNP streaming its column, masks broadcast from shared
 *     memory); the last cluster's sums are the SNP's totals less the others'; centres and feature
 *     scores in FP64 (k_skfr_means);
 *   - the `sparsity` largest scores of each kept list (ties to the lower index) by a radix select
 *     on the scores' bit patterns and an index-order compaction, one block per list (k_skfr_select);
 *   - the reassignment scores of every individual on the kept SNPs: the terms of each two
 *     consecutive kept SNPs added for all 16 code pairs (k_skfr_pairs), then one thread per
 *     individual and slice of SKFR_ASLICE kept SNPs adds one pair entry per two SNPs in FP64, in SNP
 *     order, with the pair tables of a chunk in shared memory (k_skfr_assign_shared: one list for all
 *     clusters, each code read once; k_skfr_assign_own: each cluster's own list), the slice sums then
 *     added in order (k_skfr_assign_sum); the argmin over clusters and the count of changed
 *     assignments (k_skfr_argmin).
 * The host keeps the sequential k-means++ draws from a splitmix64 stream, reads one count per
 * iteration for the convergence test, and sums the objective in individual order at the end of a
 * try.  Every FP64 operation whose rounding the oracle reproduces is written with explicit
 * round-to-nearest intrinsics, so no multiply-add is contracted.
 */
#include <algorithm>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <vector>
#include "kernels.h"

namespace {

constexpr int SKFR_SLICE = 1024;     /* SNPs per partial sum of the seeding distances */
constexpr int SKFR_DCHUNK = 128;     /* SNPs whose squared differences are staged in shared memory at a time */
constexpr int SKFR_WCHUNK = 256;     /* 16-individual words of masks staged per shared-memory chunk */
constexpr int SKFR_ASLICE = 1024;    /* kept SNPs per partial sum of the reassignment scores */
constexpr int SKFR_ACHUNK = 32;      /* kept SNPs whose pair tables are staged in shared memory at a time */
constexpr int SKFR_SEL_THREADS = 1024;

__device__ __forceinline__ uint32_t col_word(const uint8_t *bed, int64_t pitch, int64_t l, int64_t w)
{
    return *(const uint32_t *)(bed + (size_t)l * pitch + (size_t)w * 4);
}

/* class counts of every SNP: n0 (code 00, dosage 0), n1 (10, dosage 1), n2 (11, dosage 2) */
__global__ void k_skfr_counts(const uint8_t *__restrict__ bed, int64_t pitch, int64_t nw, int64_t J,
                              int64_t *__restrict__ cnt)
{
    const int64_t l = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (l >= J) return;
    long long c0 = 0, c1 = 0, c2 = 0;
    for (int64_t w = lane; w < nw; w += 32) {
        const uint32_t x = col_word(bed, pitch, l, w);
        const uint32_t hi = (x >> 1) & 0x55555555u, lo = x & 0x55555555u;
        c0 += __popc(~hi & ~lo & 0x55555555u);
        c1 += __popc(hi & ~lo);
        c2 += __popc(hi & lo);
    }
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_down_sync(0xffffffffu, c0, o);
        c1 += __shfl_down_sync(0xffffffffu, c1, o);
        c2 += __shfl_down_sync(0xffffffffu, c2, o);
    }
    if (lane == 0) {
        cnt[3 * l] = c0;
        cnt[3 * l + 1] = c1;
        cnt[3 * l + 2] = c2;
    }
}

/* sq[l][c] = (x_lc - x_l,centre)^2 for every SNP l and code c, x from the table xt[l][code] */
__global__ void k_skfr_sqtab(const uint8_t *__restrict__ bed, int64_t pitch, int64_t J, const double *__restrict__ xt,
                             int64_t center, double *__restrict__ sq)
{
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= J) return;
    const double *t = xt + 4 * l;
    const double xc = t[(bed[(size_t)l * pitch + (size_t)(center >> 2)] >> ((center & 3) * 2)) & 3];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double d = __dsub_rn(t[c], xc);
        sq[4 * l + c] = __dmul_rn(d, d);
    }
}

/* partial[s][i] = sum over the SNPs l of slice s, in order, of sq[l][code_il] */
__global__ void __launch_bounds__(128)
k_skfr_dist(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I, int64_t J, const double *__restrict__ sq,
            double *__restrict__ partial)
{
    __shared__ double tab[SKFR_DCHUNK * 4];
    const int64_t w = (int64_t)blockIdx.x * 128 + threadIdx.x;   /* word = 16 individuals */
    const int64_t s = blockIdx.y;
    const bool live = w * 16 < I;
    const int64_t l0 = s * SKFR_SLICE, l1 = min(J, l0 + SKFR_SLICE);
    double part[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) part[j] = 0.0;
    for (int64_t c0 = l0; c0 < l1; c0 += SKFR_DCHUNK) {
        const int n = (int)min((int64_t)SKFR_DCHUNK, l1 - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < 4 * n; t += 128) tab[t] = sq[4 * c0 + t];
        __syncthreads();
        if (live) {
            const uint8_t *col = bed + (size_t)c0 * pitch + (size_t)w * 4;
            int u = 0;
            for (; u + 4 <= n; u += 4) {
                uint32_t x[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) x[v] = *(const uint32_t *)(col + (size_t)(u + v) * pitch);
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const double *tb = tab + (u + v) * 4;
#pragma unroll
                    for (int j = 0; j < 16; ++j) part[j] = __dadd_rn(part[j], tb[(x[v] >> (2 * j)) & 3u]);
                }
            }
            for (; u < n; ++u) {
                const uint32_t x = *(const uint32_t *)(col + (size_t)u * pitch);
                const double *tb = tab + u * 4;
#pragma unroll
                for (int j = 0; j < 16; ++j) part[j] = __dadd_rn(part[j], tb[(x >> (2 * j)) & 3u]);
            }
        }
    }
    if (live) {
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (w * 16 + j < I) partial[(size_t)s * I + w * 16 + j] = part[j];
    }
}

__global__ void k_skfr_dist_sum(const double *__restrict__ partial, int64_t I, int nslice, double *__restrict__ D)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= I) return;
    double t = 0.0;
    for (int s = 0; s < nslice; ++s) t = __dadd_rn(t, partial[(size_t)s * I + i]);
    D[i] = t;
}

/* membership masks (bit 2j of mask[k][w] set when individual 16w + j is in cluster k) and the
 * cluster sizes nk[k] (added to; zeroed before the launch) */
__global__ void k_skfr_masks(const int32_t *__restrict__ cl, int64_t I, int64_t nw, int K, uint32_t *__restrict__ mask,
                             int32_t *__restrict__ nk)
{
    __shared__ int cnt[16];
    if (threadIdx.x < 16) cnt[threadIdx.x] = 0;
    __syncthreads();
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w < nw) {
        uint32_t m[16];
        for (int k = 0; k < K; ++k) m[k] = 0u;
        for (int j = 0; j < 16; ++j) {
            const int64_t i = w * 16 + j;
            if (i < I) m[cl[i]] |= 1u << (2 * j);
        }
        for (int k = 0; k < K; ++k) {
            mask[(size_t)k * nw + w] = m[k];
            if (m[k]) atomicAdd(&cnt[k], __popc(m[k]));
        }
    }
    __syncthreads();
    if (threadIdx.x < K && cnt[threadIdx.x]) atomicAdd(&nk[threadIdx.x], cnt[threadIdx.x]);
}

/* one word of a column: dosage sums and missing counts under each cluster's mask */
template <int KC>
__device__ __forceinline__ void sums_word(uint32_t x, const uint32_t (*ms)[SKFR_WCHUNK], int w, int32_t *sg, int32_t *sm)
{
    const uint32_t hi = (x >> 1) & 0x55555555u, lo = x & 0x55555555u;
    const uint32_t h2 = hi & lo, mi = ~hi & lo;
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        /* dosage = hi + (hi & lo), both on the even bits: one count of (hi & m) | ((hi & lo & m) << 1) */
        const uint32_t m = ms[k][w];
        sg[k] += __popc((hi & m) | ((h2 & m) << 1));
        sm[k] += __popc(mi & m);
    }
}

/* two words: the missing bits (even bits only) of the second shifted onto the odd bits, one count */
template <int KC>
__device__ __forceinline__ void sums_pair(uint32_t x0, uint32_t x1, const uint32_t (*ms)[SKFR_WCHUNK], int w, int32_t *sg,
                                          int32_t *sm)
{
    const uint32_t hi0 = (x0 >> 1) & 0x55555555u, lo0 = x0 & 0x55555555u;
    const uint32_t hi1 = (x1 >> 1) & 0x55555555u, lo1 = x1 & 0x55555555u;
    const uint32_t h20 = hi0 & lo0, mi0 = ~hi0 & lo0, h21 = hi1 & lo1, mi1 = ~hi1 & lo1;
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        const uint32_t m0 = ms[k][w], m1 = ms[k][w + 1];
        sg[k] += __popc((hi0 & m0) | ((h20 & m0) << 1)) + __popc((hi1 & m1) | ((h21 & m1) << 1));
        sm[k] += __popc((mi0 & m0) | ((mi1 & m1) << 1));
    }
}

/* per SNP l and cluster k < KC (all clusters but the last): S = sum of the members' dosages,
 * M = members with a missing code (one thread per SNP, its column streamed 64 bytes at a time, masks
 * staged in shared memory) */
template <int KC>
__global__ void __launch_bounds__(128)
k_skfr_sums(const uint8_t *__restrict__ bed, int64_t pitch, int64_t nw, int64_t J, const uint32_t *__restrict__ mask,
            int32_t *__restrict__ S, int32_t *__restrict__ M)
{
    __shared__ uint32_t ms[KC][SKFR_WCHUNK];
    const int64_t l = (int64_t)blockIdx.x * 128 + threadIdx.x;
    int32_t sg[KC], sm[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k) sg[k] = sm[k] = 0;
    for (int64_t w0 = 0; w0 < nw; w0 += SKFR_WCHUNK) {
        const int nwc = (int)min((int64_t)SKFR_WCHUNK, nw - w0);
        __syncthreads();
        for (int t = threadIdx.x; t < KC * SKFR_WCHUNK; t += 128) {
            const int k = t / SKFR_WCHUNK, w = t - k * SKFR_WCHUNK;
            ms[k][w] = w < nwc ? mask[(size_t)k * nw + w0 + w] : 0u;
        }
        __syncthreads();
        if (l < J) {
            /* the column pitch is a multiple of 16 bytes and covers every word up to nw rounded up to 4 */
            const uint8_t *col = bed + (size_t)l * pitch + (size_t)w0 * 4;
            int w = 0;
            for (; w + 16 <= nwc; w += 16) {
                uint4 v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) v[u] = *(const uint4 *)(col + (size_t)(w + 4 * u) * 4);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    sums_pair<KC>(v[u].x, v[u].y, ms, w + 4 * u, sg, sm);
                    sums_pair<KC>(v[u].z, v[u].w, ms, w + 4 * u + 2, sg, sm);
                }
            }
            for (; w < nwc; w += 4) {
                const uint4 v = *(const uint4 *)(col + (size_t)w * 4);
                if (w + 1 < nwc) sums_pair<KC>(v.x, v.y, ms, w, sg, sm);
                else sums_word<KC>(v.x, ms, w, sg, sm);
                if (w + 3 < nwc) sums_pair<KC>(v.z, v.w, ms, w + 2, sg, sm);
                else if (w + 2 < nwc) sums_word<KC>(v.z, ms, w + 2, sg, sm);
            }
        }
    }
    if (l < J) {
#pragma unroll
        for (int k = 0; k < KC; ++k) {
            S[(size_t)k * J + l] = sg[k];
            M[(size_t)k * J + l] = sm[k];
        }
    }
}

/* theta_kl = (a_l S_kl - b_l n_kl) / N_k (n_kl = N_k - M_kl non-missing members) and the feature
 * scores: global r_l = sum_k N_k theta_kl^2, local r_kl = N_k theta_kl^2.  S and M hold clusters
 * 0..K-2; the last cluster's are the SNP's totals (class counts cnt) less theirs. */
__global__ void k_skfr_means(const int32_t *__restrict__ S, const int32_t *__restrict__ M, const int64_t *__restrict__ cnt,
                             int64_t I, const double *__restrict__ ab, const int32_t *__restrict__ Nk, int K, int64_t J,
                             int local, double *__restrict__ theta, double *__restrict__ score)
{
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= J) return;
    const double a = ab[2 * l], b = ab[2 * l + 1];
    int64_t s_last = cnt[3 * l + 1] + 2 * cnt[3 * l + 2];
    int64_t m_last = I - cnt[3 * l] - cnt[3 * l + 1] - cnt[3 * l + 2];
    double r = 0.0;
    for (int k = 0; k < K; ++k) {
        int64_t sk, mk;
        if (k < K - 1) {
            sk = S[(size_t)k * J + l];
            mk = M[(size_t)k * J + l];
            s_last -= sk;
            m_last -= mk;
        } else {
            sk = s_last;
            mk = m_last;
        }
        double t = 0.0;
        const double nk = (double)Nk[k];
        if (nk > 0.0) {
            const double n = nk - (double)mk;
            t = __ddiv_rn(__dsub_rn(__dmul_rn(a, (double)sk), __dmul_rn(b, n)), nk);
        }
        theta[(size_t)k * J + l] = t;
        const double rk = __dmul_rn(__dmul_rn(nk, t), t);
        if (local) score[(size_t)k * J + l] = rk;
        else r = k == 0 ? rk : __dadd_rn(r, rk);
    }
    if (!local) score[l] = r;
}

/* exclusive scan of v over a block of SKFR_SEL_THREADS threads; *total = the block's sum */
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *wsum, uint32_t *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t t = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        wsum[lane] = t;
    }
    __syncthreads();
    const uint32_t before = (wid ? wsum[wid - 1] : 0u) + x - v;
    *total = wsum[31];
    __syncthreads();
    return before;
}

/* The s largest of the J scores of list blockIdx.x (ties to the lower index), written to out in
 * increasing index order.  The scores are non-negative doubles, so their bit patterns order as the
 * values: eight radix passes of 8 bits find the s-th largest pattern T and how many copies of it
 * are needed; one pass in index order then keeps every score above T and the first `need` equal
 * to T, each thread taking 4 consecutive SNPs and one packed scan of (above, equal) counts giving
 * every kept SNP its output position. */
__global__ void __launch_bounds__(SKFR_SEL_THREADS)
k_skfr_select(const double *__restrict__ score, int64_t J, int64_t s, int32_t *__restrict__ out)
{
    __shared__ uint32_t hist[256];
    __shared__ uint32_t wsum[32];
    __shared__ unsigned long long s_prefix;
    __shared__ long long s_rank;
    const unsigned long long *key = (const unsigned long long *)(score + (size_t)blockIdx.x * J);
    int32_t *o = out + (size_t)blockIdx.x * s;
    const int tid = threadIdx.x, lane = tid & 31;
    unsigned long long prefix = 0ull, pmask = 0ull;
    long long rank = s;                     /* rank of the wanted pattern among those under the prefix */
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int t = tid; t < 256; t += SKFR_SEL_THREADS) hist[t] = 0u;
        __syncthreads();
        for (int64_t l0 = 0; l0 < J; l0 += 4 * SKFR_SEL_THREADS) {
            unsigned long long kv[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int64_t l = l0 + tid + (int64_t)v * SKFR_SEL_THREADS;
                kv[v] = l < J ? key[l] : 0ull;
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int64_t l = l0 + tid + (int64_t)v * SKFR_SEL_THREADS;
                const bool act = l < J && (kv[v] & pmask) == prefix;
                const uint32_t bin = act ? (uint32_t)((kv[v] >> shift) & 255u) : 256u;
                const uint32_t peers = __match_any_sync(0xffffffffu, bin);
                if (act && lane == __ffs(peers) - 1) atomicAdd(&hist[bin], (uint32_t)__popc(peers));
            }
        }
        __syncthreads();
        if (tid == 0) {
            long long acc = 0;
            int b = 255;
            for (; b > 0; --b) {
                if (acc + (long long)hist[b] >= rank) break;
                acc += hist[b];
            }
            s_prefix = prefix | ((unsigned long long)b << shift);
            s_rank = rank - acc;
        }
        __syncthreads();
        prefix = s_prefix;
        rank = s_rank;
        pmask |= 255ull << shift;
    }
    const unsigned long long T = prefix;
    const uint32_t need = (uint32_t)rank;   /* copies of T kept; s - need patterns lie above T */
    uint32_t base_gt = 0, base_eq = 0;
    for (int64_t l0 = 0; l0 < J; l0 += 4 * SKFR_SEL_THREADS) {
        const int64_t lb = l0 + 4 * (int64_t)tid;
        uint32_t gt = 0, eq = 0, gtm = 0, eqm = 0;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            if (lb + v < J) {
                const unsigned long long kv = key[lb + v];
                if (kv > T) { gt++; gtm |= 1u << v; }
                else if (kv == T) { eq++; eqm |= 1u << v; }
            }
        }
        uint32_t tot;
        const uint32_t pre = block_excl_scan((gt << 16) | eq, wsum, &tot);
        uint32_t g = base_gt + (pre >> 16), e = base_eq + (pre & 0xffffu);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            if (gtm & (1u << v)) {
                o[g + min(e, need)] = (int32_t)(lb + v);
                g++;
            } else if (eqm & (1u << v)) {
                if (e < need) o[g + e] = (int32_t)(lb + v);
                e++;
            }
        }
        base_gt += tot >> 16;
        base_eq += tot & 0xffffu;
    }
}

/* Pair tables of the reassignment terms.  For cluster k and pair r of its kept list (list k * kstride:
 * one shared list when kstride is 0; list positions q = 2r and q + 1) and codes c1, c2:
 * pt[k][r][4 c1 + c2] = T(q, c1) + T(q + 1, c2), with T(p, c) = theta_kl^2 - (2 x_l,c) theta_kl for l
 * the SNP at position p; an odd last position alone gives T(q, c1) for every c2. */
__global__ void k_skfr_pairs(const double *__restrict__ theta, const double *__restrict__ xt, const int32_t *__restrict__ kept,
                             int64_t nkept, int64_t kstride, int K, int64_t J, double *__restrict__ pt)
{
    const int64_t npair = (nkept + 1) / 2;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)K * npair) return;
    const int k = (int)(t / npair);
    const int64_t r = t - k * npair;
    const int32_t *kl = kept + k * kstride;
    const bool two = 2 * r + 1 < nkept;
    double a[4], b[4];
    {
        const int64_t l = kl[2 * r];
        const double th = theta[(size_t)k * J + l], tt = __dmul_rn(th, th);
#pragma unroll
        for (int c = 0; c < 4; ++c) a[c] = __dsub_rn(tt, __dmul_rn(__dmul_rn(2.0, xt[4 * l + c]), th));
    }
    if (two) {
        const int64_t l = kl[2 * r + 1];
        const double th = theta[(size_t)k * J + l], tt = __dmul_rn(th, th);
#pragma unroll
        for (int c = 0; c < 4; ++c) b[c] = __dsub_rn(tt, __dmul_rn(__dmul_rn(2.0, xt[4 * l + c]), th));
    }
    double *o = pt + (size_t)t * 16;
#pragma unroll
    for (int c1 = 0; c1 < 4; ++c1)
#pragma unroll
        for (int c2 = 0; c2 < 4; ++c2) o[4 * c1 + c2] = two ? __dadd_rn(a[c1], b[c2]) : a[c1];
}

/* The codes of a chunk's kept SNPs for a block's 128 individuals (32 bytes per SNP): thread t loads
 * the 8 bytes 8 (t & 3) .. 8 (t & 3) + 7 of list position t >> 2 (positions past the chunk's n repeat
 * its last SNP).  The 32 bytes from i0 / 4 stay inside the column's 16-byte pitch but for the last
 * block, whose overrun (at most 16 bytes, for individuals beyond I) falls in the next column or in
 * the 64 bytes after the last one. */
__device__ __forceinline__ uint2 load_codes(const uint8_t *__restrict__ bed, int64_t pitch, int64_t i0,
                                            const int32_t *__restrict__ kl, int64_t q0, int n)
{
    const int pos = min((int)(threadIdx.x >> 2), n - 1);
    return *(const uint2 *)(bed + (size_t)kl[q0 + pos] * pitch + (size_t)(i0 >> 2) + 8u * (threadIdx.x & 3u));
}

/* The loaded codes interleaved by pair: cp[r][2m] = byte m of position 2r, cp[r][2m + 1] = byte m of
 * position 2r + 1 (the partner thread t ^ 4 holds the other position of the pair).  Every thread of
 * the block calls it. */
__device__ __forceinline__ void store_codes(uint8_t (*cp)[64], uint2 v)
{
    const uint2 o = make_uint2(__shfl_xor_sync(0xffffffffu, v.x, 4), __shfl_xor_sync(0xffffffffu, v.y, 4));
    const int pos = threadIdx.x >> 2, seg = threadIdx.x & 3;
    const bool even = (pos & 1) == 0;
    const uint32_t a = even ? v.x : o.y, b = even ? o.x : v.y;   /* position 2r's and 2r+1's 4 bytes */
    *(uint2 *)&cp[pos >> 1][seg * 16 + (even ? 0 : 8)] = make_uint2(__byte_perm(a, b, 0x5140), __byte_perm(a, b, 0x7362));
}

/* Reassignment scores, one shared kept list (global mode): thread = individual i, blockIdx.y = slice
 * of SKFR_ASLICE list positions; part[y][i][k] = sum over the slice's pairs (list order, FP64 from 0)
 * of pt[k][pair][4 code_q + code_q+1].  Per chunk of SKFR_ACHUNK positions the block stages the pair
 * tables as [pair][code pair][k] with an odd row stride (the 16 code pairs of one pair fall in
 * different banks) and the chunk's codes interleaved by pair (one 16-bit load per pair and thread),
 * the codes of the next chunk loaded while this one is summed; each code is read once for all K
 * clusters. */
template <int K>
__global__ void __launch_bounds__(128)
k_skfr_assign_shared(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I, const int32_t *__restrict__ kept,
                     int64_t nkept, const double *__restrict__ pt, double *__restrict__ part)
{
    constexpr int KS = K | 1;
    __shared__ double ts[(SKFR_ACHUNK / 2) * 16 * KS];
    __shared__ __align__(16) uint8_t cp[SKFR_ACHUNK / 2][64];
    const int64_t npair = (nkept + 1) / 2;
    const int64_t i0 = (int64_t)blockIdx.x * 128, i = i0 + threadIdx.x;
    const int64_t p0 = (int64_t)blockIdx.y * SKFR_ASLICE, p1 = min(nkept, p0 + SKFR_ASLICE);
    const int sh = (int)(threadIdx.x & 3) * 2, cb = 2 * (int)(threadIdx.x >> 2);
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    uint2 cv = load_codes(bed, pitch, i0, kept, p0, (int)min((int64_t)SKFR_ACHUNK, p1 - p0));
    for (int64_t q0 = p0; q0 < p1; q0 += SKFR_ACHUNK) {          /* q0 is even */
        const int n = (int)min((int64_t)SKFR_ACHUNK, p1 - q0), np = (n + 1) / 2;
        const int64_t r0 = q0 / 2;
        __syncthreads();
        for (int t = threadIdx.x; t < np * 16 * K; t += 128) {
            const int k = t / (np * 16), e = t - k * (np * 16);       /* e = pair * 16 + code pair */
            ts[e * KS + k] = pt[((size_t)k * npair + r0) * 16 + e];
        }
        store_codes(cp, cv);
        if (q0 + SKFR_ACHUNK < p1)
            cv = load_codes(bed, pitch, i0, kept, q0 + SKFR_ACHUNK, (int)min((int64_t)SKFR_ACHUNK, p1 - q0 - SKFR_ACHUNK));
        __syncthreads();
        if (i < I) {
#pragma unroll 4
            for (int pp = 0; pp < np; ++pp) {
                /* an odd last position is paired with itself: its table ignores the second code */
                const uint32_t v = *(const uint16_t *)&cp[pp][cb];
                const double *tp = ts + (pp * 16 + (int)(((v >> sh) & 3u) * 4u + ((v >> (sh + 8)) & 3u))) * KS;
#pragma unroll
                for (int k = 0; k < K; ++k) acc[k] = __dadd_rn(acc[k], tp[k]);
            }
        }
    }
    if (i < I) {
        double *o = part + ((size_t)blockIdx.y * I + i) * K;
#pragma unroll
        for (int k = 0; k < K; ++k) o[k] = acc[k];
    }
}

/* Reassignment scores, each cluster its own kept list (local mode): as k_skfr_assign_shared with
 * blockIdx.z = cluster k, its list kept[k] and pair tables pt[k]. */
__global__ void __launch_bounds__(128)
k_skfr_assign_own(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I, const int32_t *__restrict__ kept,
                  int64_t nkept, int K, const double *__restrict__ pt, double *__restrict__ part)
{
    __shared__ double ts[(SKFR_ACHUNK / 2) * 16];
    __shared__ __align__(16) uint8_t cp[SKFR_ACHUNK / 2][64];
    const int k = blockIdx.z;
    const int64_t npair = (nkept + 1) / 2;
    const int64_t i0 = (int64_t)blockIdx.x * 128, i = i0 + threadIdx.x;
    const int64_t p0 = (int64_t)blockIdx.y * SKFR_ASLICE, p1 = min(nkept, p0 + SKFR_ASLICE);
    const int sh = (int)(threadIdx.x & 3) * 2, cb = 2 * (int)(threadIdx.x >> 2);
    const int32_t *kl = kept + (size_t)k * nkept;
    const double *tk = pt + (size_t)k * npair * 16;
    double acc = 0.0;
    uint2 cv = load_codes(bed, pitch, i0, kl, p0, (int)min((int64_t)SKFR_ACHUNK, p1 - p0));
    for (int64_t q0 = p0; q0 < p1; q0 += SKFR_ACHUNK) {
        const int n = (int)min((int64_t)SKFR_ACHUNK, p1 - q0), np = (n + 1) / 2;
        const int64_t r0 = q0 / 2;
        __syncthreads();
        for (int t = threadIdx.x; t < np * 16; t += 128) ts[t] = tk[r0 * 16 + t];
        store_codes(cp, cv);
        if (q0 + SKFR_ACHUNK < p1)
            cv = load_codes(bed, pitch, i0, kl, q0 + SKFR_ACHUNK, (int)min((int64_t)SKFR_ACHUNK, p1 - q0 - SKFR_ACHUNK));
        __syncthreads();
        if (i < I) {
#pragma unroll 4
            for (int pp = 0; pp < np; ++pp) {
                const uint32_t v = *(const uint16_t *)&cp[pp][cb];
                acc = __dadd_rn(acc, ts[pp * 16 + (int)(((v >> sh) & 3u) * 4u + ((v >> (sh + 8)) & 3u))]);
            }
        }
    }
    if (i < I) part[((size_t)blockIdx.y * I + i) * K + k] = acc;
}

/* sc[i][k] = the slice sums part[y][i][k] added in slice order (FP64 from 0) */
__global__ void k_skfr_assign_sum(const double *__restrict__ part, int64_t IK, int nslice, double *__restrict__ sc)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= IK) return;
    double v = 0.0;
    for (int y = 0; y < nslice; ++y) v = __dadd_rn(v, part[(size_t)y * IK + t]);
    sc[t] = v;
}

/* cl_new[i] = argmin_k sc[i][k] (ties to the lower cluster); *changed += individuals whose cluster moved */
__global__ void k_skfr_argmin(const double *__restrict__ sc, int64_t I, int K, const int32_t *__restrict__ cl,
                              int32_t *__restrict__ cl_new, int32_t *__restrict__ changed)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool moved = false;
    if (i < I) {
        const double *r = sc + (size_t)i * K;
        int best = 0;
        double rb = r[0];
        for (int k = 1; k < K; ++k)
            if (r[k] < rb) { best = k; rb = r[k]; }
        cl_new[i] = best;
        moved = best != cl[i];
    }
    const uint32_t b = __ballot_sync(0xffffffffu, moved);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(changed, __popc(b));
}

struct SplitMix64 {
    uint64_t s;
    uint64_t next()
    {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

/* the kernels templated on the cluster count, for one K */
template <int K>
struct SkfrK {
    /* sums of clusters 0..K-2 (none for one cluster: the totals are its sums) */
    static cudaError_t sums(const uint8_t *bed, int64_t pitch, int64_t nw, int64_t J, const uint32_t *mask, int32_t *S,
                            int32_t *M, cudaStream_t st)
    {
        if constexpr (K > 1) {
            k_skfr_sums<K - 1><<<(unsigned)((J + 127) / 128), 128, 0, st>>>(bed, pitch, nw, J, mask, S, M);
            return cudaGetLastError();
        }
        return cudaSuccess;
    }
    static cudaError_t assign_shared(const uint8_t *bed, int64_t pitch, int64_t I, const int32_t *kept, int64_t nkept,
                                     const double *pt, double *part, cudaStream_t st)
    {
        const dim3 grid((unsigned)((I + 127) / 128), (unsigned)((nkept + SKFR_ASLICE - 1) / SKFR_ASLICE));
        k_skfr_assign_shared<K><<<grid, 128, 0, st>>>(bed, pitch, I, kept, nkept, pt, part);
        return cudaGetLastError();
    }
};

#define SKFR_DISPATCH(K, CALL)                                                                              \
    switch (K) {                                                                                            \
    case 1: return SkfrK<1>::CALL; case 2: return SkfrK<2>::CALL; case 3: return SkfrK<3>::CALL;             \
    case 4: return SkfrK<4>::CALL; case 5: return SkfrK<5>::CALL; case 6: return SkfrK<6>::CALL;             \
    case 7: return SkfrK<7>::CALL; case 8: return SkfrK<8>::CALL; case 9: return SkfrK<9>::CALL;             \
    case 10: return SkfrK<10>::CALL; case 11: return SkfrK<11>::CALL; case 12: return SkfrK<12>::CALL;       \
    case 13: return SkfrK<13>::CALL; case 14: return SkfrK<14>::CALL; case 15: return SkfrK<15>::CALL;       \
    case 16: return SkfrK<16>::CALL;                                                                        \
    }                                                                                                       \
    return cudaErrorInvalidValue;

cudaError_t sums_for_k(int K, const uint8_t *bed, int64_t pitch, int64_t nw, int64_t J, const uint32_t *mask, int32_t *S,
                       int32_t *M, cudaStream_t st)
{
    SKFR_DISPATCH(K, sums(bed, pitch, nw, J, mask, S, M, st))
}

cudaError_t assign_shared_for_k(int K, const uint8_t *bed, int64_t pitch, int64_t I, const int32_t *kept, int64_t nkept,
                                const double *pt, double *part, cudaStream_t st)
{
    SKFR_DISPATCH(K, assign_shared(bed, pitch, I, kept, nkept, pt, part, st))
}
#undef SKFR_DISPATCH

template <class T>
struct DevBuf {
    T *p = nullptr;
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)); }
    ~DevBuf() { if (p) cudaFree(p); }
};

#define SK_TRY(x)                                                                                           \
    do {                                                                                                    \
        const cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) return e_;                                                                   \
    } while (0)

}  // namespace

cudaError_t skfr_run(const uint8_t *bed, int64_t pitch, int64_t I, int64_t J, int K, int64_t sparsity, int local,
                     int max_iter, int tries, uint64_t seed, cudaStream_t st, int32_t *clusters_out, int32_t *aims_out,
                     int64_t aims_capacity, int64_t *n_aims, double *objective_out, int32_t *iters_out)
{
    if (K < 1 || K > 16 || I < 1 || J < 1 || sparsity < 1 || max_iter < 1 || tries < 1) return cudaErrorInvalidValue;
    const int64_t nw = (I + 15) / 16;                 /* 16-individual words per column (within the pitch) */
    const int nslice = (int)((J + SKFR_SLICE - 1) / SKFR_SLICE);
    const int64_t s = std::min(sparsity, J);
    const int naslice = (int)((s + SKFR_ASLICE - 1) / SKFR_ASLICE);
    const int nlists = local ? K : 1;                 /* kept lists: one for all clusters, or one per cluster */
    if ((int64_t)nslice > 65535 || (int64_t)naslice > 65535 || J > INT32_MAX) return cudaErrorInvalidValue;
    DevBuf<int64_t> d_cnt;
    DevBuf<double> d_xt, d_ab, d_sq, d_partial, d_D, d_theta, d_score, d_pt, d_apart, d_sc;
    DevBuf<uint32_t> d_mask;
    DevBuf<int32_t> d_cl, d_cl2, d_nk, d_changed, d_S, d_M, d_kept;
    SK_TRY(d_cnt.alloc(3 * J));
    SK_TRY(d_xt.alloc(4 * J));
    SK_TRY(d_ab.alloc(2 * J));
    SK_TRY(d_sq.alloc(4 * J));
    SK_TRY(d_partial.alloc((size_t)nslice * I));
    SK_TRY(d_D.alloc(I));
    SK_TRY(d_theta.alloc((size_t)K * J));
    SK_TRY(d_score.alloc((size_t)nlists * J));
    const int64_t npair = (s + 1) / 2;                /* kept-list pairs */
    SK_TRY(d_pt.alloc((size_t)K * npair * 16));
    SK_TRY(d_apart.alloc((size_t)naslice * I * K));
    SK_TRY(d_sc.alloc((size_t)I * K));
    SK_TRY(d_mask.alloc((size_t)K * nw));
    SK_TRY(d_cl.alloc(I));
    SK_TRY(d_cl2.alloc(I));
    SK_TRY(d_nk.alloc(K));
    SK_TRY(d_changed.alloc(1));
    SK_TRY(d_S.alloc((size_t)K * J));
    SK_TRY(d_M.alloc((size_t)K * J));
    SK_TRY(d_kept.alloc((size_t)nlists * s));

    /* per-SNP standardisation from the class counts (host FP64, as the oracle) */
    k_skfr_counts<<<(unsigned)((J + 3) / 4), 128, 0, st>>>(bed, pitch, nw, J, d_cnt.p);
    SK_TRY(cudaGetLastError());
    std::vector<int64_t> cnt((size_t)3 * J);
    SK_TRY(cudaMemcpyAsync(cnt.data(), d_cnt.p, sizeof(int64_t) * 3 * J, cudaMemcpyDeviceToHost, st));
    SK_TRY(cudaStreamSynchronize(st));
    std::vector<double> xt((size_t)4 * J), ab((size_t)2 * J);
    double x2_total = 0.0;
    for (int64_t l = 0; l < J; ++l) {
        const double n0 = (double)cnt[3 * l], n1 = (double)cnt[3 * l + 1], n2 = (double)cnt[3 * l + 2];
        const double n = n0 + n1 + n2;
        double a = 0.0, b = 0.0;
        if (n > 0.0) {
            const double mu = (n1 + 2.0 * n2) / n;
            const double var = (n1 + 4.0 * n2) / n - mu * mu;
            if (var > 0.0) {
                a = 1.0 / sqrt(var);
                b = mu * a;
                x2_total += n;
            }
        }
        ab[2 * l] = a;
        ab[2 * l + 1] = b;
        xt[4 * l] = -b;
        xt[4 * l + 1] = 0.0;
        xt[4 * l + 2] = a - b;
        xt[4 * l + 3] = 2.0 * a - b;
    }
    SK_TRY(cudaMemcpyAsync(d_xt.p, xt.data(), sizeof(double) * 4 * J, cudaMemcpyHostToDevice, st));
    SK_TRY(cudaMemcpyAsync(d_ab.p, ab.data(), sizeof(double) * 2 * J, cudaMemcpyHostToDevice, st));

    SplitMix64 rng{seed};
    std::vector<double> D((size_t)I), dk((size_t)I * K), sc((size_t)I * K);
    std::vector<int32_t> cl((size_t)I), kept((size_t)nlists * s);
    double best_obj = 0.0;
    bool have_best = false;

    /* squared distances of every individual to individual `center` over all SNPs, into out (host) */
    auto dist = [&](int64_t center, double *out) -> cudaError_t {
        k_skfr_sqtab<<<(unsigned)((J + 255) / 256), 256, 0, st>>>(bed, pitch, J, d_xt.p, center, d_sq.p);
        SK_TRY(cudaGetLastError());
        const dim3 grid((unsigned)((nw + 127) / 128), (unsigned)nslice);
        k_skfr_dist<<<grid, 128, 0, st>>>(bed, pitch, I, J, d_sq.p, d_partial.p);
        SK_TRY(cudaGetLastError());
        k_skfr_dist_sum<<<(unsigned)((I + 255) / 256), 256, 0, st>>>(d_partial.p, I, nslice, d_D.p);
        SK_TRY(cudaGetLastError());
        SK_TRY(cudaMemcpyAsync(out, d_D.p, sizeof(double) * I, cudaMemcpyDeviceToHost, st));
        return cudaStreamSynchronize(st);
    };
    /* for the assignment dcl: cluster sizes, centres, scores, kept lists, pair tables and sc[i][k] (no sync) */
    auto pass = [&](const int32_t *dcl) -> cudaError_t {
        SK_TRY(cudaMemsetAsync(d_nk.p, 0, sizeof(int32_t) * K, st));
        k_skfr_masks<<<(unsigned)((nw + 127) / 128), 128, 0, st>>>(dcl, I, nw, K, d_mask.p, d_nk.p);
        SK_TRY(cudaGetLastError());
        SK_TRY(sums_for_k(K, bed, pitch, nw, J, d_mask.p, d_S.p, d_M.p, st));
        k_skfr_means<<<(unsigned)((J + 255) / 256), 256, 0, st>>>(d_S.p, d_M.p, d_cnt.p, I, d_ab.p, d_nk.p, K, J, local,
                                                                d_theta.p, d_score.p);
        SK_TRY(cudaGetLastError());
        k_skfr_select<<<(unsigned)nlists, SKFR_SEL_THREADS, 0, st>>>(d_score.p, J, s, d_kept.p);
        SK_TRY(cudaGetLastError());
        k_skfr_pairs<<<(unsigned)((K * npair + 255) / 256), 256, 0, st>>>(d_theta.p, d_xt.p, d_kept.p, s, local ? s : 0, K,
                                                                         J, d_pt.p);
        SK_TRY(cudaGetLastError());
        if (local) {
            const dim3 grid((unsigned)((I + 127) / 128), (unsigned)naslice, (unsigned)K);
            k_skfr_assign_own<<<grid, 128, 0, st>>>(bed, pitch, I, d_kept.p, s, K, d_pt.p, d_apart.p);
            SK_TRY(cudaGetLastError());
        } else {
            SK_TRY(assign_shared_for_k(K, bed, pitch, I, d_kept.p, s, d_pt.p, d_apart.p, st));
        }
        k_skfr_assign_sum<<<(unsigned)((I * K + 255) / 256), 256, 0, st>>>(d_apart.p, I * K, naslice, d_sc.p);
        return cudaGetLastError();
    };

    for (int t = 0; t < tries; ++t) {
        /* k-means++ seeding */
        const int64_t c0 = std::min((int64_t)(rng.uniform() * (double)I), I - 1);
        SK_TRY(dist(c0, dk.data()));                                     /* row 0 of dk: centre 0 */
        std::copy(dk.begin(), dk.begin() + I, D.begin());
        for (int k = 1; k < K; ++k) {
            double tot = 0.0;
            for (int64_t i = 0; i < I; ++i) tot += D[i];
            const double u = rng.uniform();
            int64_t pick = I - 1;
            if (tot > 0.0) {
                const double r = u * tot;
                double acc = 0.0;
                for (int64_t i = 0; i < I; ++i) {
                    acc += D[i];
                    if (acc > r) { pick = i; break; }
                }
            } else {
                pick = std::min((int64_t)(u * (double)I), I - 1);
            }
            SK_TRY(dist(pick, dk.data() + (size_t)k * I));
            for (int64_t i = 0; i < I; ++i) D[i] = std::min(D[i], dk[(size_t)k * I + i]);
        }
        for (int64_t i = 0; i < I; ++i) {
            int best = 0;
            for (int k = 1; k < K; ++k)
                if (dk[(size_t)k * I + i] < dk[(size_t)best * I + i]) best = k;
            cl[i] = best;
        }
        int32_t *cur = d_cl.p, *nxt = d_cl2.p;
        SK_TRY(cudaMemcpyAsync(cur, cl.data(), sizeof(int32_t) * I, cudaMemcpyHostToDevice, st));
        /* iterations: the host reads one count per iteration */
        int it = 0;
        bool converged = false;
        for (it = 1; it <= max_iter; ++it) {
            SK_TRY(pass(cur));
            SK_TRY(cudaMemsetAsync(d_changed.p, 0, sizeof(int32_t), st));
            k_skfr_argmin<<<(unsigned)((I + 255) / 256), 256, 0, st>>>(d_sc.p, I, K, cur, nxt, d_changed.p);
            SK_TRY(cudaGetLastError());
            int32_t changed = 0;
            SK_TRY(cudaMemcpyAsync(&changed, d_changed.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            SK_TRY(cudaStreamSynchronize(st));
            if (changed == 0) {
                converged = true;
                break;
            }
            std::swap(cur, nxt);
        }
        if (it > max_iter) it = max_iter;
        /* the objective of the final assignment with its sparse centres: at convergence the last pass
         * was already of this assignment */
        if (!converged) SK_TRY(pass(cur));
        SK_TRY(cudaMemcpyAsync(sc.data(), d_sc.p, sizeof(double) * I * K, cudaMemcpyDeviceToHost, st));
        SK_TRY(cudaMemcpyAsync(cl.data(), cur, sizeof(int32_t) * I, cudaMemcpyDeviceToHost, st));
        SK_TRY(cudaMemcpyAsync(kept.data(), d_kept.p, sizeof(int32_t) * nlists * s, cudaMemcpyDeviceToHost, st));
        SK_TRY(cudaStreamSynchronize(st));
        double obj = x2_total;
        for (int64_t i = 0; i < I; ++i) obj += sc[(size_t)i * K + cl[i]];
        if (!have_best || obj < best_obj) {
            have_best = true;
            best_obj = obj;
            std::copy(cl.begin(), cl.end(), clusters_out);
            std::vector<int32_t> u(kept.begin(), kept.end());
            std::sort(u.begin(), u.end());
            u.erase(std::unique(u.begin(), u.end()), u.end());
            *n_aims = (int64_t)u.size();
            std::copy(u.begin(), u.begin() + std::min<int64_t>((int64_t)u.size(), aims_capacity), aims_out);
            *iters_out = it;
        }
    }
    *objective_out = best_obj;
    return cudaSuccess;
}
