/*
 * qp_batch.cu -- batched per-individual simplex QPs and per-SNP box QPs of the block SQP
 * updates (update_q! / update_p!, algorithms_inner.jl:199-228 and 275-306), fused with the
 * x + delta step and the projection (projections.jl).
 *
 * One thread solves one problem; its (K+2)^2 or (K+1)^2 tableau lives in shared memory in
 * a [element][thread] layout so a warp's accesses to the same element are consecutive.
 * The solver is the Jennrich-Sampson sweep / active-set method of qp.jl:171-317, step for
 * step.  Products feeding a sum are rounded separately (__dmul_rn / __dadd_rn), as in the
 * reference's plain Julia loops, so the tableau arithmetic is the same IEEE sequence as the
 * oracle's; only the accumulated XtX / Xtz inputs differ in their last bits.
 */
#include "common.cuh"
#include "kernels.h"

namespace {

constexpr int QB = 32;   /* problems (threads) per block */

template <int N>
struct Tab {
    double *base;
    int tid;
    __device__ __forceinline__ double &operator()(int r, int c) const { return base[((r) * N + (c)) * QB + tid]; }
};

/* sweep! (qp.jl:297-317) */
template <int N>
__device__ __noinline__ void sweep(const Tab<N> &A, double *tmp, int k, bool inverse)
{
    const double piv = 1.0 / A(k, k);
#pragma unroll
    for (int i = 0; i < N; ++i) {
        tmp[i * QB] = A(i, k);
        A(i, k) = 0.0;
        A(k, i) = 0.0;
    }
    tmp[k * QB] = inverse ? 1.0 : -1.0;
#pragma unroll 1
    for (int i = 0; i < N; ++i) {
        const double pv = __dmul_rn(piv, tmp[i * QB]);
#pragma unroll
        for (int j = 0; j < N; ++j) A(j, i) = __dsub_rn(A(j, i), __dmul_rn(pv, tmp[j * QB]));
    }
}

/* quadratic_program! (qp.jl:171-292) with pmin = 0, pmax = 1.  Returns the iteration count
 * or 0 on failure; delta is left as the reference leaves it. */
template <int K, int C>
__device__ int quadratic_program(const Tab<K + C + 1> &A, double *tmp, double *d,
                                 const double (&par)[K], double (&delta)[K])
{
    constexpr int N = K + C + 1, E = N - 1;
    const double small = 1e-5, tol = 1e-8;
#pragma unroll
    for (int i = 0; i < K; ++i) delta[i] = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) d[i * QB] = A(i, i);
#pragma unroll 1
    for (int i = 0; i < K; ++i) {
        const double di = d[i * QB];
        if (di <= 0.0 || A(i, i) < __dmul_rn(di, tol)) return 0;
        sweep<N>(A, tmp, i, false);
    }
    uint32_t swept = (K >= 32) ? 0xffffffffu : ((1u << K) - 1u);
#pragma unroll 1
    for (int i = K; i < K + C; ++i) {
        if (A(i, i) >= 0.0) return 0;
        sweep<N>(A, tmp, i, false);
    }
    for (int iteration = 1; iteration <= 1000; ++iteration) {
        double a = 1.0;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (swept & (1u << i)) {
                const double ui = A(i, E);
                const double ai = (ui > 0.0) ? (1.0 - par[i] - delta[i]) : (0.0 - par[i] - delta[i]);
                if (fabs(ui) > 1e-10) a = fmin(a, ai / ui);
            }
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (swept & (1u << i)) {
                const double ui = A(i, E);
                delta[i] = __dadd_rn(delta[i], __dmul_rn(a, ui));
                A(i, E) = __dmul_rn(1.0 - a, ui);
                A(E, i) = A(i, E);
            }
        }
        int pick = -1;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (pick < 0) {
                const double xi = par[i] + delta[i];
                const bool critical = (0.0 >= xi - small) || (1.0 <= xi + small);
                if ((swept & (1u << i)) && fabs(A(i, i)) > 1e-10 && critical) pick = i;
            }
        }
        if (pick >= 0) {
            sweep<N>(A, tmp, pick, true);
            swept &= ~(1u << pick);
            continue;
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (pick < 0) {
                const double ui = A(i, E);
                const double xi = par[i] + delta[i];
                bool violation = ui > 0.0 && 0.0 >= xi - small;
                violation = violation || (ui < 0.0 && 1.0 <= xi + small);
                if (!(swept & (1u << i)) && violation) pick = i;
            }
        }
        if (pick >= 0) {
            sweep<N>(A, tmp, pick, false);
            swept |= (1u << pick);
            continue;
        }
        return iteration;
    }
    return 0;
}

/* project_q! (projections.jl:27-59) on K values held in registers; s is scratch. */
template <int K>
__device__ __forceinline__ void project_simplex(double (&b)[K], double *s)
{
    const double pc = 1e-5;
    const double tau = 1.0 - __dmul_rn((double)K, pc);
#pragma unroll
    for (int i = 0; i < K; ++i) b[i] -= pc;
    /* descending insertion sort of the values (order of equal values is immaterial) */
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const double v = b[i];
        int k = i;
        while (k > 0 && s[(k - 1) * QB] < v) { s[k * QB] = s[(k - 1) * QB]; --k; }
        s[k * QB] = v;
    }
    double tsum = 0.0, tmax = 0.0;
    bool bget = false;
    for (int i = 0; i < K - 1; ++i) {
        tsum += s[i * QB];
        tmax = (tsum - tau) / (double)(i + 1);
        if (tmax >= s[(i + 1) * QB]) { bget = true; break; }
    }
    if (!bget) tmax = (tsum + s[(K - 1) * QB] - tau) / (double)K;
#pragma unroll
    for (int i = 0; i < K; ++i) b[i] = fmax(b[i] - tmax, 0.0) + pc;
}

/* damp_retry (the mixed-precision form only): a problem whose QP fails is solved once more with
 * the Hessian's diagonal scaled by 1 + K/512.  A BF16 Hessian rounds every pair product p_k p_k'
 * on its own, so a problem whose exact Hessian is nearly singular can come out slightly
 * indefinite and fail the reference's pivot tests; the scaling covers that rounding (K * 2^-9
 * per row, Gershgorin) and only shortens the Newton step -- the fixed point is set by the
 * gradient.  The FP64 form never retries: a failed QP leaves the reference's zero step. */
template <int K, bool SIMPLEX>
__global__ void __launch_bounds__(QB)
k_qp(int64_t nprob, const double *__restrict__ parts, int S, const double *__restrict__ x,
     double *__restrict__ x_next, int32_t *__restrict__ status, int32_t *__restrict__ fail_count,
     const double *__restrict__ vt, int mu_mode, int damp_retry)
{
    constexpr int C = SIMPLEX ? 1 : 0;
    constexpr int N = K + C + 1;
    constexpr int T = K * (K + 1) / 2, E = T + K;
    extern __shared__ double sm[];
    const int tid = threadIdx.x;
    const int64_t pr = (int64_t)blockIdx.x * QB + tid;
    if (pr >= nprob) return;           /* no block-level synchronisation below */
    Tab<N> A{sm, tid};
    double *tmp = sm + N * N * QB + tid;
    double *d = tmp + N * QB;

    double par[K], delta[K];
#pragma unroll
    for (int k = 0; k < K; ++k) par[k] = x[(size_t)K * pr + k];

    /* create_tableau! (qp.jl:8-76): H, border -r = Xtz (r = -Xtz, algorithms_inner.jl:201) */
    const int64_t stride = nprob * (int64_t)E;
    const double *src = parts + (size_t)pr * E;
    int st = 0;
    for (int attempt = 0; attempt < (damp_retry ? 2 : 1) && st == 0; ++attempt) {
    const double dscale = attempt ? 1.0 + (double)K / 512.0 : 1.0;
#pragma unroll 1
    for (int k2 = 0; k2 < K; ++k2) {
#pragma unroll 1
        for (int k = 0; k <= k2; ++k) {
            const int e = tri_index(k, k2);
            double s = 0.0;
            for (int sl = 0; sl < S; ++sl) s += src[(size_t)sl * stride + e];
            if (k == k2) s *= dscale;
            A(k, k2) = s;
            A(k2, k) = s;
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int sl = 0; sl < S; ++sl) s += src[(size_t)sl * stride + T + k];
        A(N - 1, k) = s;
        A(k, N - 1) = s;
    }
    A(N - 1, N - 1) = 0.0;
    if (SIMPLEX) {
        double mu = 0.0;
        if (mu_mode == 1) {
            /* tmp_k = H v[:,1]; tmp_k = V' tmp_k; mu = 2 (|tmp_k|_1 - 2 tmp_k[1]) / K */
            /* t1 is staged in the d column (free until quadratic_program fills it) */
#pragma unroll 1
            for (int i = 0; i < K; ++i) {
                double s = 0.0;
#pragma unroll 1
                for (int j = 0; j < K; ++j) s = __dadd_rn(s, __dmul_rn(A(i, j), vt[j]));
                d[i * QB] = s;
            }
            double n1 = 0.0, first = 0.0;
#pragma unroll 1
            for (int i = 0; i < K; ++i) {
                double s = 0.0;
#pragma unroll 1
                for (int j = 0; j < K; ++j) s = __dadd_rn(s, __dmul_rn(vt[i + K * j], d[j * QB]));
                n1 += fabs(s);
                if (i == 0) first = s;
            }
            mu = (n1 - __dmul_rn(2.0, first)) / (double)K;
            mu = __dmul_rn(2.0, mu);
        }
#pragma unroll
        for (int j = 0; j < K; ++j)
#pragma unroll
            for (int i = 0; i < K; ++i) A(i, j) += mu;
#pragma unroll
        for (int i = 0; i < K; ++i) { A(K, i) = 1.0; A(i, K) = 1.0; }
        A(K, K) = 0.0;
        double sx = 0.0;
#pragma unroll
        for (int i = 0; i < K; ++i) sx += par[i];
        A(K + 1, K) = 1.0 - sx;
        A(K, K + 1) = 1.0 - sx;
        A(K + 1, K + 1) = 0.0;
    }

    st = quadratic_program<K, C>(A, tmp, d, par, delta);
    }   /* attempts */
    if (status) status[pr] = st;
    if (st == 0 && fail_count) atomicAdd(fail_count, 1);

    double b[K];
#pragma unroll
    for (int k = 0; k < K; ++k) b[k] = par[k] + delta[k];
    if (SIMPLEX) {
        project_simplex<K>(b, tmp);
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) b[k] = fmin(fmax(b[k], 1e-5), 1.0 - 1e-5);   /* project_p! */
    }
#pragma unroll
    for (int k = 0; k < K; ++k) x_next[(size_t)K * pr + k] = b[k];
}

template <int K, bool SIMPLEX>
constexpr size_t qp_smem()
{
    constexpr int N = K + (SIMPLEX ? 1 : 0) + 1;
    return sizeof(double) * (size_t)QB * (N * N + 2 * N);
}

template <int K>
cudaError_t prepare_qp_t()
{
    cudaError_t e = cudaFuncSetAttribute(k_qp<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)qp_smem<K, true>());
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_qp<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)qp_smem<K, false>());
    return e;
}

template <int K, bool SIMPLEX>
cudaError_t launch_qp_t(int64_t nprob, const double *parts, int S, const double *x, double *x_next,
                        int32_t *status, int32_t *fail_count, const double *vt, int mu_mode, int damp_retry,
                        cudaStream_t st)
{
    const size_t smem = qp_smem<K, SIMPLEX>();
    if (nprob <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((nprob + QB - 1) / QB);
    k_qp<K, SIMPLEX><<<grid, QB, smem, st>>>(nprob, parts, S, x, x_next, status, fail_count, vt, mu_mode, damp_retry);
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_qp(int K, bool simplex, int64_t nprob, const double *parts, int S,
                      const double *x, double *x_next, int32_t *status, int32_t *fail_count,
                      const double *vt, int mu_mode, int damp_retry, cudaStream_t st)
{
    cudaError_t e = cudaErrorInvalidValue;
    if (simplex) { ADMIX_DISPATCH_K(K, (e = launch_qp_t<KK, true>(nprob, parts, S, x, x_next, status, fail_count, vt, mu_mode, damp_retry, st))); }
    else { ADMIX_DISPATCH_K(K, (e = launch_qp_t<KK, false>(nprob, parts, S, x, x_next, status, fail_count, vt, mu_mode, damp_retry, st))); }
    return e;
}

/* Dynamic shared-memory limits of the QP kernels for this K (once per handle, before capture). */
cudaError_t prepare_qp(int K)
{
    cudaError_t e = cudaErrorInvalidValue;
    ADMIX_DISPATCH_K(K, e = prepare_qp_t<KK>());
    return e;
}
