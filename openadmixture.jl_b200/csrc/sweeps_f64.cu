/*
 * sweeps_f64.cu -- the FP64 ("plain") decode-fused sweeps over the packed genotype matrix.
 *
 * Every kernel decodes the 2-bit PLINK codes in place (loops.jl:529-534), recomputes
 * qp = sum_k q_ki p_kj (qp_block!, loops.jl:303-314) and accumulates in FP64.  Unlike the
 * reference's CUDA.jl kernels (cuda/kernels.jl), which add every cell's contribution into
 * global memory with FP64 atomics, each accumulator here has one owner thread; a sweep that
 * needs more parallelism than its owners provide is split into S slices whose partial sums
 * the consumer kernel adds in a fixed order.  Results are deterministic run to run.
 */
#include "common.cuh"
#include "kernels.h"

/* ===================================================================== loglik */

/* loglikelihood_kernel (cuda/kernels.jl:2-32) / loglikelihood_loop_skipmissing
 * (loops.jl:517-539); with mu != NULL the non-skipmissing loglikelihood_loop (loops.jl:493-514),
 * whose missing cells count with the SNP's mean dosage mu_j.  Thread = one genotype byte (4
 * individuals) of a column range;
 * q of its 4 individuals lives in registers, p of a 64-SNP chunk in shared memory.
 * Each cell adds nm * log(qp^g (1-qp)^(2-g)): one log per cell instead of two (equal to
 * the reference's g log qp + (2-g) log(1-qp) up to rounding). */
template <int K>
__global__ void __launch_bounds__(256)
k_loglik_f64(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t Ib, int64_t pitch,
             const double *__restrict__ q, const double *__restrict__ p,
             int64_t jslice, double *__restrict__ partial, const double *__restrict__ mu)
{
    constexpr int JC = 64;
    __shared__ double ps[JC * K];
    __shared__ double red[8];
    const int64_t b = (int64_t)blockIdx.x * 256 + threadIdx.x;
    const int64_t j0 = (int64_t)blockIdx.y * jslice;
    const int64_t j1 = min(J, j0 + jslice);
    double qr[4][K];
    bool valid[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int64_t i = 4 * b + s;
        valid[s] = (b < Ib) && (i < I);
#pragma unroll
        for (int k = 0; k < K; ++k) qr[s][k] = valid[s] ? q[(size_t)K * i + k] : 0.5 / K;
    }
    double acc = 0.0;
    for (int64_t jc = j0; jc < j1; jc += JC) {
        const int n = (int)min((int64_t)JC, j1 - jc);
        __syncthreads();
        for (int t = threadIdx.x; t < n * K; t += blockDim.x) ps[t] = p[(size_t)K * jc + t];
        __syncthreads();
        if (b < Ib) {
            const uint8_t *col = bed + (size_t)jc * pitch + b;
            for (int jj = 0; jj < n; ++jj) {
                const unsigned byte = __ldg(col + (size_t)jj * pitch);
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int c = (byte >> (2 * s)) & 3;
                    double qp = 0.0;
#pragma unroll
                    for (int k = 0; k < K; ++k) qp = fma(qr[s][k], ps[jj * K + k], qp);
                    const double om = 1.0 - qp;
                    double v = 0.0;
                    if (c != 1) {
                        const double arg = (c == 3) ? qp * qp : ((c == 2) ? qp * om : om * om);
                        v = log(arg);
                    } else if (mu) {   /* loglikelihood_loop: the missing dosage imputed by mu_j */
                        const double gm = __ldg(mu + jc + jj);
                        v = gm * log(qp) + (2.0 - gm) * log(om);
                    }
                    acc += valid[s] ? v : 0.0;
                }
            }
        }
    }
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

/* Fixed-order sum of n partials into *out (one block of 1024 threads). */
__global__ void __launch_bounds__(1024)
k_sum_partials(const double *__restrict__ partial, int64_t n, double *__restrict__ out)
{
    __shared__ double red[32];
    double v = 0.0;
    for (int64_t t = threadIdx.x; t < n; t += blockDim.x) v += partial[t];
    const double s = block_sum(v, red);
    if (threadIdx.x == 0) *out = s;
}

/* ===================================================================== Q side */

/* With mu != NULL every kernel below runs the reference's non-skipmissing twin (update_q_loop!,
 * em_q_loop!, update_p_loop!, em_p_loop!, loops.jl:589-608,679-698,840-865,896-921): a missing
 * cell counts with g = mu_j, the SNP's mean dosage, and weight 1.
 *
 * Per-individual accumulators over SNPs j.  MODE 0 (update_q_loop_skipmissing!,
 * loops.jl:867-894; update_q_kernel!, cuda/kernels.jl:102-137): entries e < T are the
 * packed upper triangle of XtX_q (T = K(K+1)/2), entries T..T+K-1 are Xtz_q.
 * MODE 1 (em_q_loop_skipmissing!, loops.jl:610-632): E = K entries sum_j (z1 p_k + z2 (1-p_k)),
 * finalised into q_next by k_emq_finalize.
 *   z1 = nm g / qp, z2 = nm (2-g) / (1-qp), w1 = z1 / qp, w2 = z2 / (1-qp)
 *   XtX[k,k2] += w1 p_k p_k2 + w2 (1-p_k)(1-p_k2),   Xtz[k] += z1 p_k + z2 (1-p_k)
 * Shared tables A[jj][e], B[jj][e] hold the SNP-side factors of each entry for a chunk of
 * JC SNPs, so the inner loop is two FMAs per entry.  Thread (i, sub) owns entries
 * [sub*L, sub*L + L) of individual i. */
template <int K, int MODE>
struct QSide {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int E = MODE == 0 ? T + K : K;
    static constexpr int NS = ns_for_k(K);
    static constexpr int L = (E + NS - 1) / NS;
    static constexpr int IPB = 128 / NS;
    static constexpr int JC = (E > 64) ? 16 : 32;
    static constexpr size_t smem = sizeof(double) * (size_t)JC * (2 * E + K);
};

template <int K, int MODE>
__global__ void __launch_bounds__(128)
k_sweep_q_f64(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
              const double *__restrict__ q, const double *__restrict__ p,
              int64_t jslice, double *__restrict__ out, const double *__restrict__ mu)
{
    using C = QSide<K, MODE>;
    constexpr int T = C::T, E = C::E, NS = C::NS, L = C::L, JC = C::JC;
    extern __shared__ double sm[];
    double *A = sm, *B = sm + JC * E, *P = sm + 2 * JC * E;
    const int sub = threadIdx.x % NS;
    const int64_t i = (int64_t)blockIdx.x * C::IPB + threadIdx.x / NS;
    const bool valid = i < I;
    const int64_t j0 = (int64_t)blockIdx.y * jslice;
    const int64_t j1 = min(J, j0 + jslice);
    double qi[K];
#pragma unroll
    for (int k = 0; k < K; ++k) qi[k] = valid ? q[(size_t)K * i + k] : 0.5 / K;
    double acc[L];
#pragma unroll
    for (int l = 0; l < L; ++l) acc[l] = 0.0;
    const int ebase = sub * L;
    const uint8_t *colbase = bed + (valid ? (i >> 2) : 0);
    const int sh = (int)(i & 3) * 2;

    for (int64_t jc = j0; jc < j1; jc += JC) {
        const int n = (int)min((int64_t)JC, j1 - jc);
        __syncthreads();
        for (int t = threadIdx.x; t < n * K; t += blockDim.x) P[t] = p[(size_t)K * jc + t];
        __syncthreads();
        for (int t = threadIdx.x; t < n * E; t += blockDim.x) {
            const int jj = t / E, e = t - jj * E;
            const double *pj = P + jj * K;
            double a, bb;
            if (MODE == 0 && e < T) {
                int k, k2;
                tri_pair(e, k, k2);
                a = pj[k] * pj[k2];
                bb = (1.0 - pj[k]) * (1.0 - pj[k2]);
            } else {
                const int k = (MODE == 0) ? e - T : e;
                a = pj[k];
                bb = 1.0 - pj[k];
            }
            A[t] = a;
            B[t] = bb;
        }
        __syncthreads();
        for (int jj = 0; jj < n; ++jj) {
            const int c = valid ? ((__ldg(colbase + (size_t)(jc + jj) * pitch) >> sh) & 3) : 1;
            double qp = 0.0;
#pragma unroll
            for (int k = 0; k < K; ++k) qp = fma(qi[k], P[jj * K + k], qp);
            double g = gval(c);
            bool nm = (c != 1);
            if (!nm && mu && valid) { g = __ldg(mu + jc + jj); nm = true; }   /* mean-imputed loops */
            const double r1 = 1.0 / qp, r2 = 1.0 / (1.0 - qp);
            const double z1 = (nm && g != 0.0) ? g * r1 : 0.0;
            const double z2 = (nm && g != 2.0) ? (2.0 - g) * r2 : 0.0;
            const double w1 = z1 * r1, w2 = z2 * r2;
            const double *Aj = A + jj * E, *Bj = B + jj * E;
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const int e = ebase + l;
                if (e < E) {
                    const bool hess = (MODE == 0) && (e < T);
                    const double c1 = hess ? w1 : z1, c2 = hess ? w2 : z2;
                    acc[l] = fma(c1, Aj[e], fma(c2, Bj[e], acc[l]));
                }
            }
        }
    }
    if (valid) {
        double *o = out + ((size_t)blockIdx.y * I + i) * E;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const int e = ebase + l;
            if (e < E) o[e] = acc[l];
        }
    }
}

/* em_q! finalisation (algorithms_inner.jl:89): q_next[k,i] = q[k,i] * sum_s acc / (2J). */
/* q_next[k,i] = q[k,i] sum_j (z1 p_k + z2 (1-p_k)) / 2J from S slices of per-individual rows of E
 * entries whose sums start at entry off (E = K, off = 0 for the EM sweep; E = T + K, off = T for
 * the gradient entries of a gradient / Hessian sweep, which are the same sums) */
__global__ void k_emq_finalize(int64_t I, int K, int64_t J, int S, int E, int off, const double *__restrict__ parts,
                               const double *__restrict__ q, double *__restrict__ q_next)
{
    const int64_t n = (int64_t)K * I;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / K, k = t - i * K;
        double s = 0.0;
        for (int sl = 0; sl < S; ++sl) s += parts[((size_t)sl * I + i) * E + off + k];
        q_next[t] = q[t] * s / (double)(2 * J);
    }
}

/* ===================================================================== P side */

/* Per-SNP accumulators over individuals i.  MODE 0 (update_p_loop_skipmissing!,
 * loops.jl:923-950; update_p_kernel!, cuda/kernels.jl:139-174): e < T packed XtX_p,
 * T..T+K-1 Xtz_p, with
 *   XtX[k,k2] += nm (g/qp^2 + (2-g)/(1-qp)^2) q_k q_k2,  Xtz[k] += nm (g/qp - (2-g)/(1-qp)) q_k.
 * MODE 1 (em_p_loop_skipmissing!, loops.jl:700-721): E = 2K entries sum_i z1 q_k and
 * sum_i z2 q_k, finalised by k_emp_finalize.  Thread (j, sub) owns entries of SNP j;
 * individuals are staged IC at a time with their q and q_k q_k2 products in shared memory.
 * Slices over i start on a byte boundary (islice is a multiple of 4). */
template <int K, int MODE>
struct PSide {
    static constexpr int T = K * (K + 1) / 2;
    static constexpr int E = MODE == 0 ? T + K : 2 * K;
    static constexpr int NS = ns_for_k(K);
    static constexpr int L = (E + NS - 1) / NS;
    static constexpr int JPB = 128 / NS;
    static constexpr int IC = (E > 64) ? 32 : 64;
    static constexpr size_t smem = sizeof(double) * (size_t)IC * (E + K);
};

template <int K, int MODE>
__global__ void __launch_bounds__(128)
k_sweep_p_f64(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch,
              const double *__restrict__ q, const double *__restrict__ p,
              int64_t islice, double *__restrict__ out, const double *__restrict__ mu)
{
    using C = PSide<K, MODE>;
    constexpr int T = C::T, E = C::E, NS = C::NS, L = C::L, IC = C::IC;
    extern __shared__ double sm[];
    double *Tab = sm, *Qc = sm + IC * E;
    const int sub = threadIdx.x % NS;
    const int64_t j = (int64_t)blockIdx.x * C::JPB + threadIdx.x / NS;
    const bool valid = j < J;
    const int64_t i0 = (int64_t)blockIdx.y * islice;
    const int64_t i1 = min(I, i0 + islice);
    double pj[K];
#pragma unroll
    for (int k = 0; k < K; ++k) pj[k] = valid ? p[(size_t)K * j + k] : 0.5;
    const double muj = (mu && valid) ? mu[j] : 0.0;
    double acc[L];
#pragma unroll
    for (int l = 0; l < L; ++l) acc[l] = 0.0;
    const int ebase = sub * L;
    const uint8_t *col = bed + (size_t)(valid ? j : 0) * pitch;

    for (int64_t ic = i0; ic < i1; ic += IC) {
        const int n = (int)min((int64_t)IC, i1 - ic);
        __syncthreads();
        for (int t = threadIdx.x; t < n * K; t += blockDim.x) Qc[t] = q[(size_t)K * ic + t];
        __syncthreads();
        if (MODE == 0) {
            for (int t = threadIdx.x; t < n * E; t += blockDim.x) {
                const int ii = t / E, e = t - ii * E;
                const double *qq = Qc + ii * K;
                double v;
                if (e < T) { int k, k2; tri_pair(e, k, k2); v = qq[k] * qq[k2]; }
                else v = qq[e - T];
                Tab[t] = v;
            }
            __syncthreads();
        }
        for (int ii = 0; ii < n; ii += 4) {
            const unsigned byte = valid ? __ldg(col + ((ic + ii) >> 2)) : 0x55u;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (ii + s >= n) break;
                const int c = (byte >> (2 * s)) & 3;
                const double *qq = Qc + (ii + s) * K;
                double qp = 0.0;
#pragma unroll
                for (int k = 0; k < K; ++k) qp = fma(qq[k], pj[k], qp);
                double g = gval(c);
                bool nm = (c != 1);
                if (!nm && mu && valid) { g = muj; nm = true; }   /* mean-imputed loops */
                const double r1 = 1.0 / qp, r2 = 1.0 / (1.0 - qp);
                const double z1 = (nm && g != 0.0) ? g * r1 : 0.0;
                const double z2 = (nm && g != 2.0) ? (2.0 - g) * r2 : 0.0;
                if (MODE == 0) {
                    const double ch = fma(z1, r1, z2 * r2);   /* nm (g/qp^2 + (2-g)/(1-qp)^2) */
                    const double cg = z1 - z2;                /* nm (g/qp - (2-g)/(1-qp)) */
                    const double *tb = Tab + (ii + s) * E;
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const int e = ebase + l;
                        if (e < E) acc[l] = fma(e < T ? ch : cg, tb[e], acc[l]);
                    }
                } else {
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const int e = ebase + l;
                        if (e < E) acc[l] = fma(e < K ? z1 : z2, qq[e < K ? e : e - K], acc[l]);
                    }
                }
            }
        }
    }
    if (valid) {
        double *o = out + ((size_t)blockIdx.y * J + j) * E;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const int e = ebase + l;
            if (e < E) o[e] = acc[l];
        }
    }
}

/* em_p! finalisation (algorithms_inner.jl:133-137): A = p sum z1 q, B = (1-p) sum z2 q,
 * p_next = A / (A + B). */
__global__ void k_emp_finalize(int64_t J, int K, int S, const double *__restrict__ parts,
                               const double *__restrict__ p, double *__restrict__ p_next)
{
    const int64_t n = (int64_t)K * J;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / K;
        const int k = (int)(t - j * K);
        double a = 0.0, b = 0.0;
        for (int sl = 0; sl < S; ++sl) {
            const double *o = parts + ((size_t)sl * J + j) * (2 * K);
            a += o[k];
            b += o[K + k];
        }
        const double pk = p[t];
        const double A = pk * a, B = (1.0 - pk) * b;
        p_next[t] = A / (A + B);
    }
}

/* Sum S slices of packed accumulators (E = T + K per problem) and expand to the
 * reference's K x K x n / K x n layout (for host dumps). */
__global__ void k_expand_hess(int64_t nprob, int K, int S, const double *__restrict__ parts,
                              double *__restrict__ XtX, double *__restrict__ Xtz)
{
    const int T = K * (K + 1) / 2, E = T + K;
    const int64_t n = nprob * (int64_t)E;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pr = t / E;
        const int e = (int)(t - pr * E);
        double s = 0.0;
        for (int sl = 0; sl < S; ++sl) s += parts[(size_t)sl * n + t];
        if (e < T) {
            int k, k2;
            tri_pair(e, k, k2);
            XtX[(size_t)K * K * pr + k2 + (size_t)K * k] = s;
            XtX[(size_t)K * K * pr + k + (size_t)K * k2] = s;
        } else {
            Xtz[(size_t)K * pr + (e - T)] = s;
        }
    }
}

/* ===================================================================== decode counts */

/* Missing-code counts, bit-exact: code 01 <=> low bit 1, high bit 0.  Thread = one byte
 * column position b over a slice of SNPs; padding bits of the last byte are masked. */
__global__ void __launch_bounds__(256)
k_decode_counts(const uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t Ib, int64_t pitch, int64_t jslice,
                unsigned long long *__restrict__ miss_snp, unsigned long long *__restrict__ miss_ind)
{
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j0 = (int64_t)blockIdx.y * jslice, j1 = min(J, j0 + jslice);
    const bool valid = b < Ib;
    unsigned mask = 0x55u;
    if (valid && b == Ib - 1 && (I & 3)) mask = 0x55u >> (2 * (4 - (I & 3)));
    unsigned c[4] = {0, 0, 0, 0};
    for (int64_t j = j0; j < j1; ++j) {
        unsigned m = 0;
        if (valid) {
            const unsigned byte = __ldg(bed + (size_t)j * pitch + b);
            m = byte & ~(byte >> 1) & mask;
            c[0] += m & 1u; c[1] += (m >> 2) & 1u; c[2] += (m >> 4) & 1u; c[3] += (m >> 6) & 1u;
        }
        unsigned cnt = __popc(m);
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(miss_snp + j, (unsigned long long)cnt);
    }
    if (valid)
        for (int s = 0; s < 4; ++s) {
            const int64_t i = 4 * b + s;
            if (i < I && c[s]) atomicAdd(miss_ind + i, (unsigned long long)c[s]);
        }
}

/* ===================================================================== SNP means */

/* g.mu of the SnpLinAlg (additive model): per SNP the mean dosage over its non-missing
 * individuals, NaN when all are missing.  One block per SNP over its padded column (padding is
 * coded missing, so it never counts).  Per byte: codes 10 and 11 have the high bit, 11 also the
 * low bit, so sum g = popc(hi) + popc(hi & lo) and the missing count is popc(lo & ~hi). */
__global__ void __launch_bounds__(256)
k_snp_means(const uint8_t *__restrict__ bed, int64_t J, int64_t pitch, double *__restrict__ mu)
{
    __shared__ double red[8];
    const int64_t j = blockIdx.x;
    if (j >= J) return;
    const uint8_t *col = bed + (size_t)j * pitch;
    long long gs = 0, nn = 0;
    for (int64_t b = threadIdx.x; b < pitch; b += blockDim.x) {
        const unsigned v = col[b];
        const unsigned lo = v & 0x55u, hi = (v >> 1) & 0x55u;
        gs += __popc(hi) + __popc(hi & lo);
        nn += 4 - __popc(lo & ~hi);
    }
    const double sg = block_sum((double)gs, red);
    const double sn = block_sum((double)nn, red);
    if (threadIdx.x == 0) mu[j] = sn > 0.0 ? sg / sn : __longlong_as_double(0x7ff8000000000000LL);
}

cudaError_t launch_snp_means(const uint8_t *bed, int64_t J, int64_t pitch, double *mu, cudaStream_t st)
{
    k_snp_means<<<(unsigned)J, 256, 0, st>>>(bed, J, pitch, mu);
    return cudaGetLastError();
}

/* ===================================================================== launchers */

template <int K>
static cudaError_t launch_loglik_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                   const double *p, const LoglikPlan &pl, double *partial, double *out,
                                   cudaStream_t st, const double *mu)
{
    const int64_t Ib = (I + 3) / 4;
    dim3 grid((unsigned)pl.gx, (unsigned)pl.gy);
    k_loglik_f64<K><<<grid, 256, 0, st>>>(bed, I, J, Ib, pitch, q, p, pl.jslice, partial, mu);
    k_sum_partials<<<1, 1024, 0, st>>>(partial, (int64_t)pl.gx * pl.gy, out);
    return cudaGetLastError();
}

LoglikPlan plan_loglik(int64_t I, int64_t J, int sms)
{
    LoglikPlan pl;
    const int64_t Ib = (I + 3) / 4;
    pl.gx = (int)((Ib + 255) / 256);
    const int64_t target = (int64_t)sms * 8;
    int64_t gy = (target + pl.gx - 1) / pl.gx;
    gy = std::max<int64_t>(1, std::min<int64_t>(gy, (J + 63) / 64));
    pl.jslice = (J + gy - 1) / gy;
    pl.gy = (int)((J + pl.jslice - 1) / pl.jslice);
    if (J == 0) { pl.gy = 1; pl.jslice = 1; }
    return pl;
}

cudaError_t launch_loglik_f64(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                              const double *p, const LoglikPlan &pl, double *partial, double *out,
                              cudaStream_t st, const double *mu)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = launch_loglik_t<KK>(bed, I, J, pitch, q, p, pl, partial, out, st, mu));
    return e;
}

SweepPlan plan_sweep_q(int K, int64_t I, int64_t J, int sms)
{
    SweepPlan pl;
    const int NS = ns_for_k(K);
    pl.gx = (int)((I + 128 / NS - 1) / (128 / NS));
    const int64_t target = (int64_t)sms * 6;
    int64_t S = (target + pl.gx - 1) / pl.gx;
    S = std::max<int64_t>(1, std::min<int64_t>(S, (J + 127) / 128));
    pl.slice = (J + S - 1) / S;
    pl.S = (int)((J + pl.slice - 1) / pl.slice);
    if (J == 0) { pl.S = 1; pl.slice = 1; }
    return pl;
}

SweepPlan plan_sweep_p(int K, int64_t I, int64_t J, int sms)
{
    SweepPlan pl;
    const int NS = ns_for_k(K);
    pl.gx = (int)((J + 128 / NS - 1) / (128 / NS));
    const int64_t target = (int64_t)sms * 6;
    int64_t S = (target + pl.gx - 1) / pl.gx;
    S = std::max<int64_t>(1, std::min<int64_t>(S, (I + 127) / 128));
    int64_t slice = (I + S - 1) / S;
    slice = (slice + 3) / 4 * 4;
    pl.slice = slice;
    pl.S = (int)((I + slice - 1) / slice);
    if (I == 0) { pl.S = 1; pl.slice = 4; }
    return pl;
}

template <int K, int MODE>
static cudaError_t launch_sweep_q_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                    const double *p, const SweepPlan &pl, double *out, cudaStream_t st,
                                    const double *mu)
{
    using C = QSide<K, MODE>;
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_sweep_q_f64<K, MODE><<<grid, 128, C::smem, st>>>(bed, I, J, pitch, q, p, pl.slice, out, mu);
    return cudaGetLastError();
}

cudaError_t launch_sweep_q_f64(int K, int mode, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                               const double *q, const double *p, const SweepPlan &pl, double *out,
                               cudaStream_t st, const double *mu)
{
    cudaError_t e = cudaErrorInvalidValue;
    if (mode == 0) { ADMIX_DISPATCH_K(K, (e = launch_sweep_q_t<KK, 0>(bed, I, J, pitch, q, p, pl, out, st, mu))); }
    else { ADMIX_DISPATCH_K(K, (e = launch_sweep_q_t<KK, 1>(bed, I, J, pitch, q, p, pl, out, st, mu))); }
    return e;
}

template <int K, int MODE>
static cudaError_t launch_sweep_p_t(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                    const double *p, const SweepPlan &pl, double *out, cudaStream_t st,
                                    const double *mu)
{
    using C = PSide<K, MODE>;
    dim3 grid((unsigned)pl.gx, (unsigned)pl.S);
    k_sweep_p_f64<K, MODE><<<grid, 128, C::smem, st>>>(bed, I, J, pitch, q, p, pl.slice, out, mu);
    return cudaGetLastError();
}

cudaError_t launch_sweep_p_f64(int K, int mode, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                               const double *q, const double *p, const SweepPlan &pl, double *out,
                               cudaStream_t st, const double *mu)
{
    cudaError_t e = cudaErrorInvalidValue;
    if (mode == 0) { ADMIX_DISPATCH_K(K, (e = launch_sweep_p_t<KK, 0>(bed, I, J, pitch, q, p, pl, out, st, mu))); }
    else { ADMIX_DISPATCH_K(K, (e = launch_sweep_p_t<KK, 1>(bed, I, J, pitch, q, p, pl, out, st, mu))); }
    return e;
}

static int grid_for(int64_t n, int sms)
{
    int64_t b = (n + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sms * 16));
}

cudaError_t launch_emq_finalize(int64_t I, int K, int64_t J, int S, const double *parts,
                                const double *q, double *q_next, int sms, cudaStream_t st, int E, int off)
{
    k_emq_finalize<<<grid_for((int64_t)K * I, sms), 256, 0, st>>>(I, K, J, S, E > 0 ? E : K, off, parts, q, q_next);
    return cudaGetLastError();
}

cudaError_t launch_emp_finalize(int64_t J, int K, int S, const double *parts, const double *p,
                                double *p_next, int sms, cudaStream_t st)
{
    k_emp_finalize<<<grid_for((int64_t)K * J, sms), 256, 0, st>>>(J, K, S, parts, p, p_next);
    return cudaGetLastError();
}

cudaError_t launch_expand_hess(int64_t nprob, int K, int S, const double *parts, double *XtX,
                               double *Xtz, int sms, cudaStream_t st)
{
    const int E = K * (K + 1) / 2 + K;
    k_expand_hess<<<grid_for(nprob * E, sms), 256, 0, st>>>(nprob, K, S, parts, XtX, Xtz);
    return cudaGetLastError();
}

cudaError_t launch_sum_doubles(const double *src, int64_t n, double *dst, cudaStream_t st)
{
    k_sum_partials<<<1, 1024, 0, st>>>(src, n, dst);
    return cudaGetLastError();
}

cudaError_t launch_decode_counts(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                                 unsigned long long *miss_snp, unsigned long long *miss_ind,
                                 int sms, cudaStream_t st)
{
    const int64_t Ib = (I + 3) / 4;
    const int gx = (int)((Ib + 255) / 256);
    int64_t gy = std::max<int64_t>(1, std::min<int64_t>(((int64_t)sms * 8 + gx - 1) / gx, J));
    const int64_t jslice = (J + gy - 1) / gy;
    gy = (J + jslice - 1) / jslice;
    k_decode_counts<<<dim3(gx, (unsigned)gy), 256, 0, st>>>(bed, I, J, Ib, pitch, jslice, miss_snp, miss_ind);
    return cudaGetLastError();
}

template <int K>
static cudaError_t prepare_sweeps_t()
{
    cudaError_t e = cudaFuncSetAttribute(k_sweep_q_f64<K, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QSide<K, 0>::smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sweep_q_f64<K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)QSide<K, 1>::smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sweep_p_f64<K, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PSide<K, 0>::smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sweep_p_f64<K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PSide<K, 1>::smem);
    return e;
}

/* Dynamic shared-memory limits of the sweep kernels for this K; called once per handle
 * before any launch (and so before any stream capture). */
cudaError_t prepare_sweeps(int K)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = prepare_sweeps_t<KK>());
    return e;
}

/* Padding of the last genotype byte of every column (individuals >= I) set to the missing code
 * 01, so kernels that read whole 16-byte groups need no per-individual bound checks.  The
 * reference never reads those bits (its loops stop at I), so this changes no result. */
__global__ void k_mask_tail(uint8_t *__restrict__ bed, int64_t I, int64_t J, int64_t pitch)
{
    const int64_t Ib = (I + 3) / 4;
    const int r = (int)(I & 3);
    const unsigned keep = (1u << (2 * r)) - 1u;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < J; j += (int64_t)gridDim.x * blockDim.x) {
        uint8_t *b = bed + (size_t)j * pitch + (Ib - 1);
        *b = (uint8_t)((*b & keep) | (0x55u & ~keep));
    }
}

cudaError_t launch_mask_tail(uint8_t *bed, int64_t I, int64_t J, int64_t pitch, int sms, cudaStream_t st)
{
    if ((I & 3) == 0) return cudaSuccess;
    k_mask_tail<<<grid_for(J, sms), 256, 0, st>>>(bed, I, J, pitch);
    return cudaGetLastError();
}
