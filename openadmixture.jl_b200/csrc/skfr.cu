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
 *   - k-means++ seeding distances ||x_i - x_c||^2 over all SNPs: a thread owns 16 individuals (one
 *     32-bit word of a column) and a slice of SKFR_SLICE SNPs, FP64 sums per slice added in slice
 *     order (k_skfr_dist, k_skfr_dist_sum);
 *   - per iteration, the cluster sums of every SNP as exact integers: membership bit masks per
 *     16-individual word (k_skfr_masks), then per SNP and cluster popc(h & m) + popc(h & l & m)
 *     dosage sums and popc(~h & l & m) missing counts over the column (k_skfr_sums, one thread per
 *     SNP streaming its column, masks broadcast from shared memory); centres and feature scores in
 *     FP64 (k_skfr_means);
 *   - the reassignment scores of every individual on the kept SNPs, FP64 in SNP order
 *     (k_skfr_assign, one thread per individual).
 * The host keeps the small sequential steps: the k-means++ draws from a splitmix64 stream, the
 * choice of the `sparsity` largest scores, the argmin over clusters and the convergence test.
 * Every FP64 operation whose rounding the oracle reproduces is written with explicit
 * round-to-nearest intrinsics, so no multiply-add is contracted.
 */
#include <algorithm>
#include <cuda_runtime.h>
#include <numeric>
#include <stdint.h>
#include <stdio.h>
#include <vector>
#include "kernels.h"

namespace {

constexpr int SKFR_SLICE = 4096;     /* SNPs per partial sum of the seeding distances */
constexpr int SKFR_WCHUNK = 256;     /* 16-individual words of masks staged per shared-memory chunk */

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

/* partial[s][i] = sum over SNPs l of slice s of (x_il - x_cl)^2, x from the per-SNP table xt[l][code] */
__global__ void k_skfr_dist(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I, int64_t J,
                            const double *__restrict__ xt, int64_t center, double *__restrict__ partial)
{
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   /* word = 16 individuals */
    const int64_t s = blockIdx.y;
    if (w * 16 >= I) return;
    const int64_t l0 = s * SKFR_SLICE, l1 = min(J, l0 + SKFR_SLICE);
    double part[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) part[j] = 0.0;
    const int cs = (int)(center & 3) * 2;
    for (int64_t l = l0; l < l1; ++l) {
        const uint32_t x = col_word(bed, pitch, l, w);
        const double *t = xt + 4 * l;
        const double xc = __ldg(t + ((bed[(size_t)l * pitch + (size_t)(center >> 2)] >> cs) & 3));
        const double t0 = __ldg(t), t1 = __ldg(t + 1), t2 = __ldg(t + 2), t3 = __ldg(t + 3);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint32_t c = (x >> (2 * j)) & 3u;
            const double xi = c == 0 ? t0 : (c == 1 ? t1 : (c == 2 ? t2 : t3));
            const double d = __dsub_rn(xi, xc);
            part[j] = __dadd_rn(part[j], __dmul_rn(d, d));
        }
    }
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (w * 16 + j < I) partial[(size_t)s * I + w * 16 + j] = part[j];
}

__global__ void k_skfr_dist_sum(const double *__restrict__ partial, int64_t I, int nslice, double *__restrict__ D)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= I) return;
    double t = 0.0;
    for (int s = 0; s < nslice; ++s) t = __dadd_rn(t, partial[(size_t)s * I + i]);
    D[i] = t;
}

/* membership masks: bit 2j of mask[k][w] is set when individual 16w + j is in cluster k */
__global__ void k_skfr_masks(const int32_t *__restrict__ cl, int64_t I, int64_t nw, int K, uint32_t *__restrict__ mask)
{
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nw) return;
    uint32_t m[16];
    for (int k = 0; k < K; ++k) m[k] = 0u;
    for (int j = 0; j < 16; ++j) {
        const int64_t i = w * 16 + j;
        if (i < I) m[cl[i]] |= 1u << (2 * j);
    }
    for (int k = 0; k < K; ++k) mask[(size_t)k * nw + w] = m[k];
}

/* per SNP l and cluster k: S = sum of the members' dosages, M = members with a missing code
 * (one thread per SNP, its column streamed in 16-byte loads, masks staged in shared memory) */
template <int K>
__global__ void __launch_bounds__(128)
k_skfr_sums(const uint8_t *__restrict__ bed, int64_t pitch, int64_t nw, int64_t J, const uint32_t *__restrict__ mask,
            int32_t *__restrict__ S, int32_t *__restrict__ M)
{
    __shared__ uint32_t ms[K][SKFR_WCHUNK];
    const int64_t l = (int64_t)blockIdx.x * 128 + threadIdx.x;
    int32_t sg[K], sm[K];
#pragma unroll
    for (int k = 0; k < K; ++k) sg[k] = sm[k] = 0;
    for (int64_t w0 = 0; w0 < nw; w0 += SKFR_WCHUNK) {
        const int nwc = (int)min((int64_t)SKFR_WCHUNK, nw - w0);
        __syncthreads();
        for (int t = threadIdx.x; t < K * SKFR_WCHUNK; t += 128) {
            const int k = t / SKFR_WCHUNK, w = t - k * SKFR_WCHUNK;
            ms[k][w] = w < nwc ? mask[(size_t)k * nw + w0 + w] : 0u;
        }
        __syncthreads();
        if (l < J) {
            const uint8_t *col = bed + (size_t)l * pitch + (size_t)w0 * 4;
            for (int w = 0; w < nwc; w += 4) {   /* the column pitch is a multiple of 16 bytes */
                const uint4 v = *(const uint4 *)(col + (size_t)w * 4);
                const uint32_t xs[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (w + q >= nwc) break;
                    const uint32_t x = xs[q];
                    const uint32_t hi = (x >> 1) & 0x55555555u, lo = x & 0x55555555u;
                    const uint32_t h1 = hi, h2 = hi & lo, mi = ~hi & lo;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const uint32_t m = ms[k][w + q];
                        sg[k] += __popc(h1 & m) + __popc(h2 & m);
                        sm[k] += __popc(mi & m);
                    }
                }
            }
        }
    }
    if (l < J) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            S[(size_t)k * J + l] = sg[k];
            M[(size_t)k * J + l] = sm[k];
        }
    }
}

/* theta_kl = (a_l S_kl - b_l n_kl) / N_k (n_kl = N_k - M_kl non-missing members) and the feature
 * scores: global r_l = sum_k N_k theta_kl^2, local r_kl = N_k theta_kl^2 */
__global__ void k_skfr_means(const int32_t *__restrict__ S, const int32_t *__restrict__ M, const double *__restrict__ ab,
                             const double *__restrict__ Nk, int K, int64_t J, int local, double *__restrict__ theta,
                             double *__restrict__ score)
{
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= J) return;
    const double a = ab[2 * l], b = ab[2 * l + 1];
    double r = 0.0;
    for (int k = 0; k < K; ++k) {
        double t = 0.0;
        const double nk = Nk[k];
        if (nk > 0.0) {
            const double n = nk - (double)M[(size_t)k * J + l];
            t = __ddiv_rn(__dsub_rn(__dmul_rn(a, (double)S[(size_t)k * J + l]), __dmul_rn(b, n)), nk);
        }
        theta[(size_t)k * J + l] = t;
        const double rk = __dmul_rn(__dmul_rn(nk, t), t);
        if (local) score[(size_t)k * J + l] = rk;
        else r = k == 0 ? rk : __dadd_rn(r, rk);
    }
    if (!local) score[l] = r;
}

/* per kept SNP (cluster k's list position p) and code: theta^2 - (2 x) theta, x = xt[l][code] */
__global__ void k_skfr_terms(const double *__restrict__ theta, const double *__restrict__ xt, const int32_t *__restrict__ kept,
                             int64_t nkept, int K, int64_t J, double *__restrict__ terms)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)K * nkept) return;
    const int k = (int)(t / nkept);
    const int64_t l = kept[t];
    const double th = theta[(size_t)k * J + l], tt = __dmul_rn(th, th);
    for (int c = 0; c < 4; ++c)
        terms[4 * t + c] = __dsub_rn(tt, __dmul_rn(__dmul_rn(2.0, xt[4 * l + c]), th));
}

/* sc[i][k] = sum over cluster k's kept SNPs (in list order) of terms[k][p][code_il] */
__global__ void k_skfr_assign(const uint8_t *__restrict__ bed, int64_t pitch, int64_t I, const int32_t *__restrict__ kept,
                              int64_t nkept, int K, const double *__restrict__ terms, double *__restrict__ sc)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= I) return;
    const int sh = (int)(i & 3) * 2;
    for (int k = 0; k < K; ++k) {
        const int32_t *kl = kept + (size_t)k * nkept;
        const double *tk = terms + (size_t)k * nkept * 4;
        double acc = 0.0;
        for (int64_t p = 0; p < nkept; ++p) {
            const int c = (bed[(size_t)kl[p] * pitch + (size_t)(i >> 2)] >> sh) & 3;
            acc = __dadd_rn(acc, tk[4 * p + c]);
        }
        sc[(size_t)i * K + k] = acc;
    }
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

/* the s largest scores, ties to the lower index, in increasing index order */
void top_s(const double *score, int64_t J, int64_t s, int32_t *out)
{
    std::vector<int32_t> idx((size_t)J);
    std::iota(idx.begin(), idx.end(), 0);
    const int64_t n = std::min(s, J);
    auto better = [&](int32_t x, int32_t y) { return score[x] > score[y] || (score[x] == score[y] && x < y); };
    std::nth_element(idx.begin(), idx.begin() + (n - 1), idx.end(), better);
    std::sort(idx.begin(), idx.begin() + n, better);
    std::vector<int32_t> pick(idx.begin(), idx.begin() + n);
    std::sort(pick.begin(), pick.end());
    std::copy(pick.begin(), pick.end(), out);
}

template <int K>
cudaError_t launch_sums(const uint8_t *bed, int64_t pitch, int64_t nw, int64_t J, const uint32_t *mask, int32_t *S,
                        int32_t *M, cudaStream_t st)
{
    k_skfr_sums<K><<<(unsigned)((J + 127) / 128), 128, 0, st>>>(bed, pitch, nw, J, mask, S, M);
    return cudaGetLastError();
}

cudaError_t sums_for_k(int K, const uint8_t *bed, int64_t pitch, int64_t nw, int64_t J, const uint32_t *mask, int32_t *S,
                       int32_t *M, cudaStream_t st)
{
    switch (K) {
#define SK_CASE(k) case k: return launch_sums<k>(bed, pitch, nw, J, mask, S, M, st);
        SK_CASE(1) SK_CASE(2) SK_CASE(3) SK_CASE(4) SK_CASE(5) SK_CASE(6) SK_CASE(7) SK_CASE(8)
        SK_CASE(9) SK_CASE(10) SK_CASE(11) SK_CASE(12) SK_CASE(13) SK_CASE(14) SK_CASE(15) SK_CASE(16)
#undef SK_CASE
    }
    return cudaErrorInvalidValue;
}

template <class T>
struct DevBuf {
    T *p = nullptr;
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)); }
    ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

cudaError_t skfr_run(const uint8_t *bed, int64_t pitch, int64_t I, int64_t J, int K, int64_t sparsity, int local,
                     int max_iter, int tries, uint64_t seed, cudaStream_t st, int32_t *clusters_out, int32_t *aims_out,
                     int64_t aims_capacity, int64_t *n_aims, double *objective_out, int32_t *iters_out)
{
    if (K < 1 || K > 16 || I < 1 || J < 1 || sparsity < 1 || max_iter < 1 || tries < 1) return cudaErrorInvalidValue;
    const int64_t nw = (I + 15) / 16;                 /* 16-individual words per column (within the pitch) */
    const int nslice = (int)((J + SKFR_SLICE - 1) / SKFR_SLICE);
    const int64_t s = std::min(sparsity, J);
    cudaError_t e = cudaSuccess;
    DevBuf<int64_t> d_cnt;
    DevBuf<double> d_xt, d_ab, d_partial, d_D, d_theta, d_score, d_Nk, d_terms, d_sc;
    DevBuf<uint32_t> d_mask;
    DevBuf<int32_t> d_cl, d_S, d_M, d_kept;
    if ((e = d_cnt.alloc(3 * J)) || (e = d_xt.alloc(4 * J)) || (e = d_ab.alloc(2 * J)) ||
        (e = d_partial.alloc((size_t)nslice * I)) || (e = d_D.alloc(I)) || (e = d_theta.alloc((size_t)K * J)) ||
        (e = d_score.alloc((size_t)K * J)) || (e = d_Nk.alloc(K)) || (e = d_terms.alloc((size_t)K * s * 4)) ||
        (e = d_sc.alloc((size_t)I * K)) || (e = d_mask.alloc((size_t)K * nw)) || (e = d_cl.alloc(I)) ||
        (e = d_S.alloc((size_t)K * J)) || (e = d_M.alloc((size_t)K * J)) || (e = d_kept.alloc((size_t)K * s)))
        return e;

    /* per-SNP standardisation from the class counts (host FP64, as the oracle) */
    k_skfr_counts<<<(unsigned)((J + 3) / 4), 128, 0, st>>>(bed, pitch, nw, J, d_cnt.p);
    std::vector<int64_t> cnt((size_t)3 * J);
    if ((e = cudaGetLastError()) || (e = cudaMemcpyAsync(cnt.data(), d_cnt.p, sizeof(int64_t) * 3 * J, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaStreamSynchronize(st)))
        return e;
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
    if ((e = cudaMemcpyAsync(d_xt.p, xt.data(), sizeof(double) * 4 * J, cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(d_ab.p, ab.data(), sizeof(double) * 2 * J, cudaMemcpyHostToDevice, st)))
        return e;

    SplitMix64 rng{seed};
    std::vector<double> D((size_t)I), dk((size_t)I * K), sc((size_t)I * K), score((size_t)K * J);
    std::vector<int32_t> cl((size_t)I), cl_new((size_t)I), kept((size_t)K * s);
    std::vector<double> Nk((size_t)K);
    double best_obj = 0.0;
    bool have_best = false;

    auto dist = [&](int64_t center, double *out) -> cudaError_t {
        dim3 grid((unsigned)((nw + 127) / 128), (unsigned)nslice);
        k_skfr_dist<<<grid, 128, 0, st>>>(bed, pitch, I, J, d_xt.p, center, d_partial.p);
        cudaError_t r = cudaGetLastError();
        if (r == cudaSuccess) {
            k_skfr_dist_sum<<<(unsigned)((I + 255) / 256), 256, 0, st>>>(d_partial.p, I, nslice, d_D.p);
            r = cudaGetLastError();
        }
        if (r == cudaSuccess) r = cudaMemcpyAsync(out, d_D.p, sizeof(double) * I, cudaMemcpyDeviceToHost, st);
        if (r == cudaSuccess) r = cudaStreamSynchronize(st);
        return r;
    };
    /* centres, scores and the kept SNP lists of the assignment cl; then sc[i][k] */
    auto pass = [&]() -> cudaError_t {
        std::fill(Nk.begin(), Nk.end(), 0.0);
        for (int64_t i = 0; i < I; ++i) Nk[cl[i]] += 1.0;
        cudaError_t r = cudaMemcpyAsync(d_cl.p, cl.data(), sizeof(int32_t) * I, cudaMemcpyHostToDevice, st);
        if (r == cudaSuccess) r = cudaMemcpyAsync(d_Nk.p, Nk.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st);
        if (r == cudaSuccess) {
            k_skfr_masks<<<(unsigned)((nw + 127) / 128), 128, 0, st>>>(d_cl.p, I, nw, K, d_mask.p);
            r = cudaGetLastError();
        }
        if (r == cudaSuccess) r = sums_for_k(K, bed, pitch, nw, J, d_mask.p, d_S.p, d_M.p, st);
        if (r == cudaSuccess) {
            k_skfr_means<<<(unsigned)((J + 255) / 256), 256, 0, st>>>(d_S.p, d_M.p, d_ab.p, d_Nk.p, K, J, local, d_theta.p,
                                                                    d_score.p);
            r = cudaGetLastError();
        }
        if (r == cudaSuccess)
            r = cudaMemcpyAsync(score.data(), d_score.p, sizeof(double) * (local ? K : 1) * J, cudaMemcpyDeviceToHost, st);
        if (r == cudaSuccess) r = cudaStreamSynchronize(st);
        if (r != cudaSuccess) return r;
        for (int k = 0; k < K; ++k) top_s(score.data() + (local ? (size_t)k * J : 0), J, s, kept.data() + (size_t)k * s);
        r = cudaMemcpyAsync(d_kept.p, kept.data(), sizeof(int32_t) * K * s, cudaMemcpyHostToDevice, st);
        if (r == cudaSuccess) {
            k_skfr_terms<<<(unsigned)((K * s + 255) / 256), 256, 0, st>>>(d_theta.p, d_xt.p, d_kept.p, s, K, J, d_terms.p);
            r = cudaGetLastError();
        }
        if (r == cudaSuccess) {
            k_skfr_assign<<<(unsigned)((I + 127) / 128), 128, 0, st>>>(bed, pitch, I, d_kept.p, s, K, d_terms.p, d_sc.p);
            r = cudaGetLastError();
        }
        if (r == cudaSuccess) r = cudaMemcpyAsync(sc.data(), d_sc.p, sizeof(double) * I * K, cudaMemcpyDeviceToHost, st);
        if (r == cudaSuccess) r = cudaStreamSynchronize(st);
        return r;
    };

    for (int t = 0; t < tries; ++t) {
        /* k-means++ seeding */
        int64_t c0 = std::min((int64_t)(rng.uniform() * (double)I), I - 1);
        if ((e = dist(c0, dk.data()))) return e;                      /* column 0 of dk: centre 0 */
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
            if ((e = dist(pick, dk.data() + (size_t)k * I))) return e;
            for (int64_t i = 0; i < I; ++i) D[i] = std::min(D[i], dk[(size_t)k * I + i]);
        }
        for (int64_t i = 0; i < I; ++i) {
            int best = 0;
            for (int k = 1; k < K; ++k)
                if (dk[(size_t)k * I + i] < dk[(size_t)best * I + i]) best = k;
            cl[i] = best;
        }
        /* iterations */
        int it = 0;
        for (it = 1; it <= max_iter; ++it) {
            if ((e = pass())) return e;
            bool same = true;
            for (int64_t i = 0; i < I; ++i) {
                const double *r = sc.data() + (size_t)i * K;
                int best = 0;
                for (int k = 1; k < K; ++k)
                    if (r[k] < r[best]) best = k;
                cl_new[i] = best;
                same = same && best == cl[i];
            }
            if (same) break;
            cl.swap(cl_new);
        }
        if (it > max_iter) it = max_iter;
        /* the objective of the final assignment with its sparse centres */
        if ((e = pass())) return e;
        double obj = x2_total;
        for (int64_t i = 0; i < I; ++i) obj += sc[(size_t)i * K + cl[i]];
        if (!have_best || obj < best_obj) {
            have_best = true;
            best_obj = obj;
            std::copy(cl.begin(), cl.end(), clusters_out);
            std::vector<int32_t> u(kept.begin(), kept.begin() + (local ? (size_t)K * s : (size_t)s));
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
