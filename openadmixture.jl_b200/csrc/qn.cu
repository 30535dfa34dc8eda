/*
 * qn.cu -- ZAL quasi-Newton extrapolation (quasi_newton.jl:5-9, 29-31) and the
 * accept / reject step of admixture_qn! (algorithms_outer.jl:126-159) as device kernels.
 *
 *   U[:,c] = x1 - x0, V[:,c] = x2 - x1            c = (i-1) % Q
 *   x_tmp  = x1 - V inv(U'(U-V)) U'(x0-x1)          over the first m = min(i, Q) columns
 *   project_p!(p_tmp), project_q!(q_tmp); accept x_tmp if ll_qn > ll_prev else x_next2.
 *
 * The iteration number i is read from DevScalars so one captured sequence of launches
 * serves every iteration.  The LBQN mode of admixture_qn! (quasi_newton.jl:15-58) follows the
 * ZAL kernels below.
 */
#include "common.cuh"
#include "kernels.h"

namespace {

/* secant columns + the m x m system U'(U-V) and right side U'(x0-x1): per-block partials */
template <int Q>
__global__ void __launch_bounds__(256)
k_qn_dots(int64_t n, const double *__restrict__ x0, const double *__restrict__ x1,
          const double *__restrict__ x2, double *__restrict__ U, double *__restrict__ V,
          const DevScalars *__restrict__ sc, double *__restrict__ partial)
{
    __shared__ double red[8];
    const int iter = sc->iter;
    const int col = (iter - 1) % Q;
    double M[Q][Q], b[Q];
#pragma unroll
    for (int r = 0; r < Q; ++r) {
        b[r] = 0.0;
#pragma unroll
        for (int c = 0; c < Q; ++c) M[r][c] = 0.0;
    }
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += (int64_t)gridDim.x * blockDim.x) {
        const double xa0 = x0[a], xa1 = x1[a];
        const double un = xa1 - xa0, vn = x2[a] - xa1;
        double u[Q], w[Q];
#pragma unroll
        for (int r = 0; r < Q; ++r) {
            double ur, vr;
            if (r == col) { ur = un; vr = vn; U[a + n * r] = un; V[a + n * r] = vn; }
            else { ur = U[a + n * r]; vr = V[a + n * r]; }
            u[r] = ur;
            w[r] = ur - vr;
        }
        const double dx = xa0 - xa1;
#pragma unroll
        for (int r = 0; r < Q; ++r) {
            b[r] = fma(u[r], dx, b[r]);
#pragma unroll
            for (int c = 0; c < Q; ++c) M[r][c] = fma(u[r], w[c], M[r][c]);
        }
    }
    constexpr int NV = Q * Q + Q;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double val = (v < Q * Q) ? M[v / Q][v % Q] : b[v - Q * Q];
        const double s = block_sum(val, red);
        if (threadIdx.x == 0) partial[(size_t)blockIdx.x * NV + v] = s;
    }
}

/* Fixed-order reduction of the partials, then cf = inv(M) b by Gauss-Jordan with partial
 * pivoting (the reference calls LAPACK's inv; both are LU-based).  A singular M gives
 * non-finite coefficients, so the QN point is rejected by the ll comparison. */
template <int Q>
__global__ void k_qn_solve(int nblocks, const double *__restrict__ partial, DevScalars *__restrict__ sc)
{
    constexpr int NV = Q * Q + Q;
    __shared__ double tot[NV];
    for (int v = threadIdx.x; v < NV; v += blockDim.x) {
        double s = 0.0;
        for (int bl = 0; bl < nblocks; ++bl) s += partial[(size_t)bl * NV + v];
        tot[v] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int iter = sc->iter;
    const int m = iter < Q ? iter : Q;
    double a[Q][2 * Q];
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < 2 * m; ++j)
            a[i][j] = (j < m) ? tot[i * Q + j] : (j - m == i ? 1.0 : 0.0);
    bool singular = false;
    for (int c = 0; c < m && !singular; ++c) {
        int piv = c;
        for (int r = c + 1; r < m; ++r)
            if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
        if (a[piv][c] == 0.0) { singular = true; break; }
        if (piv != c)
            for (int j = 0; j < 2 * m; ++j) { const double t = a[c][j]; a[c][j] = a[piv][j]; a[piv][j] = t; }
        const double dv = a[c][c];
        for (int j = 0; j < 2 * m; ++j) a[c][j] /= dv;
        for (int r = 0; r < m; ++r) {
            if (r == c) continue;
            const double f = a[r][c];
            if (f != 0.0)
                for (int j = 0; j < 2 * m; ++j) a[r][j] = __dsub_rn(a[r][j], __dmul_rn(f, a[c][j]));
        }
    }
    for (int r = 0; r < Q; ++r) {
        double acc = 0.0;
        if (r < m) {
            if (singular) acc = __longlong_as_double(0x7ff8000000000000LL);
            else
                for (int c = 0; c < m; ++c) acc = __dadd_rn(acc, __dmul_rn(a[r][m + c], tot[Q * Q + c]));
        }
        sc->qn_cf[r] = acc;
    }
    sc->qn_singular = singular ? 1 : 0;
}

/* x_tmp = x1 - V cf, then project_q! on Q columns and project_p! on P columns.
 * One thread per column of x (K values). */
template <int K, int Q>
__global__ void __launch_bounds__(256)
k_qn_extrap(int64_t I, int64_t J, const double *__restrict__ x1, const double *__restrict__ V,
            const DevScalars *__restrict__ sc, double *__restrict__ x_tmp)
{
    const int64_t ncol = I + J, n = ncol * K;
    const int iter = sc->iter;
    const int m = iter < Q ? iter : Q;
    double cf[Q];
#pragma unroll
    for (int r = 0; r < Q; ++r) cf[r] = sc->qn_cf[r];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += (int64_t)gridDim.x * blockDim.x) {
        double b[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int64_t a = c * K + k;
            double s = 0.0;
#pragma unroll
            for (int r = 0; r < Q; ++r)
                if (r < m) s = fma(V[a + n * r], cf[r], s);
            b[k] = x1[a] - s;
        }
        if (c < I) {
            project_simplex_local<K>(b);
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) b[k] = fmin(fmax(b[k], 1e-5), 1.0 - 1e-5);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) x_tmp[c * K + k] = b[k];
    }
}

/* ------------------------------------------------------------------------------------------
 * LBQN mode (update_UV_LBQN!, quasi_newton.jl:15-23; update_QN_LBQN!, quasi_newton.jl:38-58):
 *   shift the secant columns right, U[:,1] = x1 - x0, V[:,1] = (x2 - x1) - U[:,1];
 *   gamma = u'v / v'v;  x_q = u;  for i = 1..m: alpha_i = (V_i' x_q) / (V_i' V_i), x_q -= alpha_i V_i;
 *   x_tmp = x0 - (gamma x_q + sum_i alpha_i U_i)       (u = U[:,1], v = V[:,1], m = min(iter, Q))
 * The column shift is an index change: logical column l (1 = newest) of iteration i is physical
 * slot (i - l) mod Q.  Because x_q = u - sum_{l<i} alpha_l V_l, every dot product the loop takes is
 * a combination of the Gram matrix V_l' V_l' and of V_l' u, so one pass over the vectors collects
 * them all (per-block partials, reduced in a fixed order) and one thread runs the recurrence. */
template <int Q>
__global__ void __launch_bounds__(256)
k_lbqn_dots(int64_t n, const double *__restrict__ x0, const double *__restrict__ x1,
            const double *__restrict__ x2, double *__restrict__ U, double *__restrict__ V,
            const DevScalars *__restrict__ sc, double *__restrict__ partial)
{
    __shared__ double red[8];
    const int iter = sc->iter;
    const int m = iter < Q ? iter : Q;
    const int slot = (iter - 1) % Q;
    double G[Q][Q], c[Q];
#pragma unroll
    for (int r = 0; r < Q; ++r) {
        c[r] = 0.0;
#pragma unroll
        for (int t = 0; t < Q; ++t) G[r][t] = 0.0;
    }
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += (int64_t)gridDim.x * blockDim.x) {
        const double xa1 = x1[a];
        const double un = xa1 - x0[a];
        const double vn = (x2[a] - xa1) - un;
        U[a + n * slot] = un;
        V[a + n * slot] = vn;
        double v[Q];
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            v[l] = 0.0;
            if (l < m) v[l] = (l == 0) ? vn : V[a + n * ((iter - 1 - l) % Q)];
        }
#pragma unroll
        for (int l = 0; l < Q; ++l) {
            c[l] = fma(v[l], un, c[l]);
#pragma unroll
            for (int t = 0; t < Q; ++t) G[l][t] = fma(v[l], v[t], G[l][t]);
        }
    }
    constexpr int NV = Q * Q + Q;
#pragma unroll
    for (int w = 0; w < NV; ++w) {
        const double val = (w < Q * Q) ? G[w / Q][w % Q] : c[w - Q * Q];
        const double s = block_sum(val, red);
        if (threadIdx.x == 0) partial[(size_t)blockIdx.x * NV + w] = s;
    }
}

template <int Q>
__global__ void k_lbqn_solve(int nblocks, const double *__restrict__ partial, DevScalars *__restrict__ sc)
{
    constexpr int NV = Q * Q + Q;
    __shared__ double tot[NV];
    for (int w = threadIdx.x; w < NV; w += blockDim.x) {
        double s = 0.0;
        for (int bl = 0; bl < nblocks; ++bl) s += partial[(size_t)bl * NV + w];
        tot[w] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int iter = sc->iter;
    const int m = iter < Q ? iter : Q;
    double alpha[Q];
    for (int i = 0; i < m; ++i) {
        double d = tot[Q * Q + i];                       /* V_i' x_q with x_q = u - sum_{l<i} alpha_l V_l */
        for (int l = 0; l < i; ++l) d = __dsub_rn(d, __dmul_rn(alpha[l], tot[i * Q + l]));
        const double rho = 1.0 / tot[i * Q + i];
        alpha[i] = __dmul_rn(rho, d);
    }
    for (int r = 0; r < Q; ++r) sc->qn_cf[r] = r < m ? alpha[r] : 0.0;
    sc->qn_gamma = tot[Q * Q] / tot[0];                 /* u'v / v'v, v = V_1 */
    sc->qn_singular = (tot[0] == 0.0) ? 1 : 0;
}

/* x_tmp = x0 - (gamma (u - sum_l alpha_l V_l) + sum_l alpha_l U_l) in the reference's order of
 * operations per element, then project_q! on Q columns and project_p! on P columns. */
template <int K, int Q>
__global__ void __launch_bounds__(256)
k_lbqn_extrap(int64_t I, int64_t J, const double *__restrict__ x0, const double *__restrict__ U,
              const double *__restrict__ V, const DevScalars *__restrict__ sc, double *__restrict__ x_tmp)
{
    const int64_t ncol = I + J, n = ncol * K;
    const int iter = sc->iter;
    const int m = iter < Q ? iter : Q;
    const double gamma = sc->qn_gamma;
    double al[Q];
    int64_t off[Q];
#pragma unroll
    for (int l = 0; l < Q; ++l) {
        al[l] = sc->qn_cf[l];
        off[l] = n * (int64_t)((iter - 1 - (l < m ? l : 0)) % Q);
    }
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += (int64_t)gridDim.x * blockDim.x) {
        double b[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int64_t a = c * K + k;
            double xq = U[a + off[0]];
#pragma unroll
            for (int l = 0; l < Q; ++l)
                if (l < m) xq = __dsub_rn(xq, __dmul_rn(al[l], V[a + off[l]]));
            double xr = __dmul_rn(gamma, xq);
#pragma unroll
            for (int l = 0; l < Q; ++l)
                if (l < m) xr = __dadd_rn(xr, __dmul_rn(al[l], U[a + off[l]]));
            b[k] = x0[a] - xr;
        }
        if (c < I) {
            project_simplex_local<K>(b);
        } else {
#pragma unroll
            for (int k = 0; k < K; ++k) b[k] = fmin(fmax(b[k], 1e-5), 1.0 - 1e-5);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) x_tmp[c * K + k] = b[k];
    }
}

__global__ void k_iter_begin(DevScalars *sc)
{
    sc->ll_prev = sc->ll_new;
    sc->fail_q = 0;
    sc->fail_p = 0;
    sc->qn_singular = 0;
}

/* algorithms_outer.jl:150-158: keep x_tmp when ll_prev < ll_qn, else x_next2. */
__global__ void __launch_bounds__(256)
k_accept(int64_t n, const double *__restrict__ x_tmp, const double *__restrict__ x_next2,
         double *__restrict__ x, DevScalars *__restrict__ sc)
{
    const double ll_prev = sc->ll_prev, ll_qn = sc->ll_qn, ll_basic = sc->ll_basic;
    const bool acc = ll_prev < ll_qn;
    const double *src = acc ? x_tmp : x_next2;
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += (int64_t)gridDim.x * blockDim.x)
        x[a] = src[a];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const double ll_new = acc ? ll_qn : ll_basic;
        sc->ll_new = ll_new;
        sc->reldiff = fabs((ll_new - ll_prev) / ll_prev);
        sc->accepted = acc ? 1 : 0;
    }
}

__global__ void __launch_bounds__(256)
k_copy(int64_t n, const double *__restrict__ src, double *__restrict__ dst)
{
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += (int64_t)gridDim.x * blockDim.x)
        dst[a] = src[a];
}

template <int Q>
cudaError_t launch_qn_q(int64_t I, int64_t J, int K, const double *x0, const double *x1,
                        const double *x2, double *U, double *V, double *x_tmp, double *partial,
                        const QNPlan &pl, DevScalars *sc, int sms, cudaStream_t st)
{
    const int64_t n = (int64_t)K * (I + J);
    k_qn_dots<Q><<<pl.blocks, 256, 0, st>>>(n, x0, x1, x2, U, V, sc, partial);
    k_qn_solve<Q><<<1, 128, 0, st>>>(pl.blocks, partial, sc);
    const int64_t ncol = I + J;
    const int gb = (int)std::max<int64_t>(1, std::min<int64_t>((ncol + 255) / 256, (int64_t)sms * 16));
    cudaError_t e = cudaSuccess;
    ADMIX_DISPATCH_K(K, (k_qn_extrap<KK, Q><<<gb, 256, 0, st>>>(I, J, x1, V, sc, x_tmp)));
    e = cudaGetLastError();
    return e;
}

template <int Q>
cudaError_t launch_lbqn_q(int64_t I, int64_t J, int K, const double *x0, const double *x1,
                          const double *x2, double *U, double *V, double *x_tmp, double *partial,
                          const QNPlan &pl, DevScalars *sc, int sms, cudaStream_t st)
{
    const int64_t n = (int64_t)K * (I + J);
    k_lbqn_dots<Q><<<pl.blocks, 256, 0, st>>>(n, x0, x1, x2, U, V, sc, partial);
    k_lbqn_solve<Q><<<1, 128, 0, st>>>(pl.blocks, partial, sc);
    const int64_t ncol = I + J;
    const int gb = (int)std::max<int64_t>(1, std::min<int64_t>((ncol + 255) / 256, (int64_t)sms * 16));
    ADMIX_DISPATCH_K(K, (k_lbqn_extrap<KK, Q><<<gb, 256, 0, st>>>(I, J, x0, U, V, sc, x_tmp)));
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_lbqn(int Q, int64_t I, int64_t J, int K, const double *x0, const double *x1,
                        const double *x2, double *U, double *V, double *x_tmp, double *partial,
                        const QNPlan &pl, DevScalars *sc, int sms, cudaStream_t st)
{
    switch (Q) {
    case 1: return launch_lbqn_q<1>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 2: return launch_lbqn_q<2>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 3: return launch_lbqn_q<3>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 4: return launch_lbqn_q<4>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 5: return launch_lbqn_q<5>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 6: return launch_lbqn_q<6>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 7: return launch_lbqn_q<7>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 8: return launch_lbqn_q<8>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    default: return cudaErrorInvalidValue;
    }
}

QNPlan plan_qn(int64_t n, int sms)
{
    QNPlan pl;
    pl.blocks = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 4));
    return pl;
}

cudaError_t launch_qn(int Q, int64_t I, int64_t J, int K, const double *x0, const double *x1,
                      const double *x2, double *U, double *V, double *x_tmp, double *partial,
                      const QNPlan &pl, DevScalars *sc, int sms, cudaStream_t st)
{
    switch (Q) {
    case 1: return launch_qn_q<1>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 2: return launch_qn_q<2>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 3: return launch_qn_q<3>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 4: return launch_qn_q<4>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 5: return launch_qn_q<5>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 6: return launch_qn_q<6>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 7: return launch_qn_q<7>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    case 8: return launch_qn_q<8>(I, J, K, x0, x1, x2, U, V, x_tmp, partial, pl, sc, sms, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_iter_begin(DevScalars *sc, cudaStream_t st)
{
    k_iter_begin<<<1, 1, 0, st>>>(sc);
    return cudaGetLastError();
}

cudaError_t launch_accept(int64_t n, const double *x_tmp, const double *x_next2, double *x,
                          DevScalars *sc, int sms, cudaStream_t st)
{
    const int gb = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
    k_accept<<<gb, 256, 0, st>>>(n, x_tmp, x_next2, x, sc);
    return cudaGetLastError();
}

cudaError_t launch_copy(int64_t n, const double *src, double *dst, int sms, cudaStream_t st)
{
    const int gb = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8));
    k_copy<<<gb, 256, 0, st>>>(n, src, dst);
    return cudaGetLastError();
}
