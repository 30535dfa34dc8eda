/*
 * admix_oracle.c -- CPU restatement of OpenADMIXTURE.jl's likelihood / gradient /
 * Hessian sweeps, block SQP updates and ZAL quasi-Newton outer loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA library
 * and the timed CPU baseline ("port" kind).  Nothing in the product path links it.
 *
 * PARITY UNPINNED: the reference is Julia (not installed here) and its only golden
 * values (test/runtests.jl:8,11) need SnpArrays' EUR_subset.bed plus Julia's
 * StableRNG stream, neither of which exists in this environment.  This file follows
 * the reference source line by line (citations below) and is checked by the test
 * suite against mathematical known-answer properties (finite-difference gradients,
 * KKT conditions of the QP, projection optimality, EM monotonicity).
 *
 * Layout follows the reference (Julia column-major):
 *   bed   : uint8 [Ib = ceil(I/4)] x J, SNP-major (SnpArray.data without the 3-byte magic)
 *   q     : K x I      p : K x J      x = [q p] : K x (I+J), flat K*(I+J)
 *   XtX_q : K x K x I  Xtz_q : K x I  XtX_p : K x K x J  Xtz_p : K x J
 *   U, V  : K(I+J) x Q
 *
 * Numerical precision: Float64 throughout, as the reference's default T=Float64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MU_AS_EXECUTED 0   /* mu = 0: what the aliased mul! in qp.jl:54-55 produces */
#define ORC_MU_GERSHGORIN  1   /* mu = 2(|V'Hv1|_1 - 2(V'Hv1)_1)/K, qp.jl:54-58 as written */

/* 2-bit PLINK codes -> genotype value / non-missing indicator.
 * loops.jl:2-5 (g_map_Float64 = [0,0,1,2], nonmissing_map_Float64 = [1,0,1,1]). */
static const double G_MAP[4]  = {0.0, 0.0, 1.0, 2.0};
static const double NM_MAP[4] = {1.0, 0.0, 1.0, 1.0};

/* The non-skipmissing loops (AdmixData(...; skipmissing=false): loglikelihood_loop,
 * em_q_loop!, em_p_loop!, update_q_loop!, update_p_loop!, loops.jl:365-383,493-514,589-608,
 * 679-698,840-865,896-921) use gij = g_map[code] + (code == 01) mu_j -- the missing genotype
 * imputed by the SNP's mean dosage g.mu[j] of the SnpLinAlg -- and no non-missing factor.
 * g_mu = NULL selects the skipmissing loops (the driver's choice, driver.jl:149). */
static const double *g_mu = NULL;

void orc_set_mean_impute(const double *mu) { g_mu = mu; }

/* g.mu of a SnpLinAlg with the additive model: the mean dosage over the non-missing
 * individuals of each SNP (NaN when every genotype is missing, the mean of nothing). */
void orc_snp_means(const uint8_t *bed, int64_t I, int64_t J, double *mu)
{
    const int64_t Ib = (I + 3) / 4;
    #pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < J; ++j) {
        double s = 0.0;
        int64_t n = 0;
        for (int64_t i = 0; i < I; ++i) {
            const uint8_t blk = bed[j * Ib + (i >> 2)];
            const int c = (blk >> ((i & 3) << 1)) & 3;
            if (c != 1) { s += G_MAP[c]; ++n; }
        }
        mu[j] = n > 0 ? s / (double)n : NAN;
    }
}

/* genotype value and non-missing weight of a cell (both loop families) */
static inline void cell_gnm(int c, int64_t j, double *g, double *nm)
{
    if (g_mu) { *g = G_MAP[c] + (c == 1 ? g_mu[j] : 0.0); *nm = 1.0; }
    else { *g = G_MAP[c]; *nm = NM_MAP[c]; }
}

static inline int code_at(const uint8_t *bed, int64_t Ib, int64_t i, int64_t j)
{
    /* loops.jl:529-532: blk = gmat[(i-1)>>2+1, j]; re = (i-1)%4; (blk >> (re<<1)) & 3 */
    uint8_t blk = bed[j * Ib + (i >> 2)];
    return (blk >> ((i & 3) << 1)) & 3;
}

/* qp_block! (loops.jl:303-314): qp = sum_k q[k,i] p[k,j], accumulated from zero in k order. */
static inline double qp_cell(const double *qi, const double *pj, int K)
{
    double s = 0.0;
    for (int k = 0; k < K; ++k) s = fma(qi[k], pj[k], s);
    return s;
}

/* ------------------------------------------------------------------ decode */

/* Missing-genotype counts per SNP and per individual (code 01), bit-exact integers.
 * Decode rule: loops.jl:529-534. */
void orc_decode_counts(const uint8_t *bed, int64_t I, int64_t J,
                       int64_t *miss_per_snp, int64_t *miss_per_ind)
{
    const int64_t Ib = (I + 3) / 4;
    if (miss_per_ind) memset(miss_per_ind, 0, sizeof(int64_t) * (size_t)I);
    #pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < J; ++j) {
        int64_t c = 0;
        for (int64_t i = 0; i < I; ++i) c += (code_at(bed, Ib, i, j) == 1);
        if (miss_per_snp) miss_per_snp[j] = c;
    }
    if (miss_per_ind) {
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < I; ++i) {
            int64_t c = 0;
            for (int64_t j = 0; j < J; ++j) c += (code_at(bed, Ib, i, j) == 1);
            miss_per_ind[i] = c;
        }
    }
}

/* ------------------------------------------------------------------ loglik */

/* loglikelihood_loop_skipmissing (loops.jl:517-539) on one tile: j outer, i inner,
 * Float64 accumulator starting from zero. */
static double loglik_tile(const uint8_t *bed, int64_t Ib, const double *q, const double *p,
                          int K, int64_t i0, int64_t i1, int64_t j0, int64_t j1)
{
    double r = 0.0;
    for (int64_t j = j0; j < j1; ++j) {
        const double *pj = p + (size_t)K * j;
        for (int64_t i = i0; i < i1; ++i) {
            int c = code_at(bed, Ib, i, j);
            double g, nm;
            cell_gnm(c, j, &g, &nm);
            double qp = qp_cell(q + (size_t)K * i, pj, K);
            r += nm * ((g * log(qp)) + ((2.0 - g) * log(1.0 - qp)));
        }
    }
    return r;
}

/* findcleft / cleave (loops.jl:16-28): split point of a 0-based half-open range. */
static int64_t cleft_len(int64_t len, int64_t step)
{
    if (len >= 2 * step) return step * (len / (step * 2));
    return (int64_t)llround((double)len / 2.0);   /* round(Int, len/2), ties to even */
}

typedef struct { int64_t i0, i1, j0, j1; } tile_t;

/* threader_scalar (loops.jl:223-258) recursion: split the longer side with cleave(.,4)
 * until both sides are <= 64 (tile_maxiter(Float64) = 512/8). */
static int64_t count_leaves(int64_t i0, int64_t i1, int64_t j0, int64_t j1)
{
    int64_t il = i1 - i0, jl = j1 - j0;
    if (il > 64 || jl > 64) {
        if (il > jl) { int64_t c = i0 + cleft_len(il, 4);
            return count_leaves(i0, c, j0, j1) + count_leaves(c, i1, j0, j1); }
        int64_t c = j0 + cleft_len(jl, 4);
        return count_leaves(i0, i1, j0, c) + count_leaves(i0, i1, c, j1);
    }
    return 1;
}

static void list_leaves(int64_t i0, int64_t i1, int64_t j0, int64_t j1, tile_t *out, int64_t *n)
{
    int64_t il = i1 - i0, jl = j1 - j0;
    if (il > 64 || jl > 64) {
        if (il > jl) { int64_t c = i0 + cleft_len(il, 4);
            list_leaves(i0, c, j0, j1, out, n); list_leaves(c, i1, j0, j1, out, n); return; }
        int64_t c = j0 + cleft_len(jl, 4);
        list_leaves(i0, i1, j0, c, out, n); list_leaves(i0, i1, c, j1, out, n); return;
    }
    out[(*n)++] = (tile_t){i0, i1, j0, j1};
}

/* Combine leaf sums along the same binary tree.  In the reference every node adds its
 * two children into an Atomic initialised to zero; 0+r1+r2 == 0+r2+r1 exactly, so the
 * node value is r1 + r2 whatever the task order. */
static double combine_leaves(int64_t i0, int64_t i1, int64_t j0, int64_t j1,
                             const double *sums, int64_t *n)
{
    int64_t il = i1 - i0, jl = j1 - j0;
    if (il > 64 || jl > 64) {
        double r1, r2;
        if (il > jl) { int64_t c = i0 + cleft_len(il, 4);
            r1 = combine_leaves(i0, c, j0, j1, sums, n); r2 = combine_leaves(c, i1, j0, j1, sums, n); }
        else { int64_t c = j0 + cleft_len(jl, 4);
            r1 = combine_leaves(i0, i1, j0, c, sums, n); r2 = combine_leaves(i0, i1, c, j1, sums, n); }
        return (0.0 + r1) + r2;
    }
    return sums[(*n)++];
}

/* loglikelihood(g::SnpLinAlg, q, p, ...) (algorithms_inner.jl:27-35). */
double orc_loglik(const uint8_t *bed, int64_t I, int64_t J, int K, const double *q, const double *p)
{
    const int64_t Ib = (I + 3) / 4;
    if (I == 0 || J == 0) return 0.0;
    int64_t nl = count_leaves(0, I, 0, J);
    tile_t *tiles = (tile_t *)malloc(sizeof(tile_t) * (size_t)nl);
    double *sums = (double *)malloc(sizeof(double) * (size_t)nl);
    int64_t n = 0;
    list_leaves(0, I, 0, J, tiles, &n);
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t t = 0; t < nl; ++t)
        sums[t] = loglik_tile(bed, Ib, q, p, K, tiles[t].i0, tiles[t].i1, tiles[t].j0, tiles[t].j1);
    n = 0;
    double r = combine_leaves(0, I, 0, J, sums, &n);
    free(tiles); free(sums);
    return r;
}

/* ------------------------------------------------------------------ EM */

/* em_q! (algorithms_inner.jl:68-92) + em_q_loop_skipmissing! (loops.jl:610-632):
 * q_next[k,i] = (1/2J) sum_j nm (g q p / qp + (2-g) q (1-p) / (1-qp)). */
void orc_em_q(const uint8_t *bed, int64_t I, int64_t J, int K,
              const double *q, const double *p, double *q_next)
{
    const int64_t Ib = (I + 3) / 4;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < I; ++i) {
        const double *qi = q + (size_t)K * i;
        double *out = q_next + (size_t)K * i;
        for (int k = 0; k < K; ++k) out[k] = 0.0;
        for (int64_t j = 0; j < J; ++j) {
            const double *pj = p + (size_t)K * j;
            int c = code_at(bed, Ib, i, j);
            double g, nm;
            cell_gnm(c, j, &g, &nm);
            double qp = qp_cell(qi, pj, K);
            for (int k = 0; k < K; ++k) {
                double tmp = (g * qi[k] * pj[k] / qp + (2.0 - g) * qi[k] * (1.0 - pj[k]) / (1.0 - qp));
                out[k] += nm * tmp;
            }
        }
        for (int k = 0; k < K; ++k) out[k] /= (double)(2 * J);
    }
}

/* em_p! (algorithms_inner.jl:108-141) + em_p_loop_skipmissing! (loops.jl:700-721):
 * A = sum_i nm g q p / qp, B = sum_i nm (2-g) q (1-p) / (1-qp), p_next = A / (A + B). */
void orc_em_p(const uint8_t *bed, int64_t I, int64_t J, int K,
              const double *q, const double *p, double *p_next)
{
    const int64_t Ib = (I + 3) / 4;
    #pragma omp parallel
    {
        double *A = (double *)malloc(sizeof(double) * (size_t)K);
        double *B = (double *)malloc(sizeof(double) * (size_t)K);
        #pragma omp for schedule(static)
        for (int64_t j = 0; j < J; ++j) {
            const double *pj = p + (size_t)K * j;
            for (int k = 0; k < K; ++k) { A[k] = 0.0; B[k] = 0.0; }
            for (int64_t i = 0; i < I; ++i) {
                const double *qi = q + (size_t)K * i;
                int c = code_at(bed, Ib, i, j);
                double g, nm;
                cell_gnm(c, j, &g, &nm);
                double qp = qp_cell(qi, pj, K);
                for (int k = 0; k < K; ++k) {
                    A[k] += nm * (g * qi[k] * pj[k] / qp);
                    B[k] += nm * ((2.0 - g) * qi[k] * (1.0 - pj[k]) / (1.0 - qp));
                }
            }
            for (int k = 0; k < K; ++k) p_next[(size_t)K * j + k] = A[k] / (A[k] + B[k]);
        }
        free(A); free(B);
    }
}

/* ------------------------------------------------------------------ gradient / Hessian */

/* update_q_loop_skipmissing! (loops.jl:867-894), summed over all j in increasing order
 * for each individual i (the order threader!/tiler! visit j for a fixed i). */
void orc_grad_hess_q(const uint8_t *bed, int64_t I, int64_t J, int K,
                     const double *q, const double *p, double *XtX, double *Xtz)
{
    const int64_t Ib = (I + 3) / 4;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < I; ++i) {
        const double *qi = q + (size_t)K * i;
        double *H = XtX + (size_t)K * K * i;
        double *z = Xtz + (size_t)K * i;
        for (int a = 0; a < K * K; ++a) H[a] = 0.0;
        for (int k = 0; k < K; ++k) z[k] = 0.0;
        for (int64_t j = 0; j < J; ++j) {
            const double *pj = p + (size_t)K * j;
            int c = code_at(bed, Ib, i, j);
            double g, nm;
            cell_gnm(c, j, &g, &nm);
            double qp = qp_cell(qi, pj, K);
            double oq = 1.0 - qp;
            for (int k = 0; k < K; ++k) {
                z[k] += nm * (g * pj[k] / qp + (2.0 - g) * (1.0 - pj[k]) / oq);
                for (int k2 = 0; k2 < K; ++k2)
                    H[k2 + K * k] += nm * (g / (qp * qp) * pj[k] * pj[k2] +
                                           (2.0 - g) / (oq * oq) * (1.0 - pj[k]) * (1.0 - pj[k2]));
            }
        }
    }
}

/* update_p_loop_skipmissing! (loops.jl:923-950), summed over i in increasing order. */
void orc_grad_hess_p(const uint8_t *bed, int64_t I, int64_t J, int K,
                     const double *q, const double *p, double *XtX, double *Xtz)
{
    const int64_t Ib = (I + 3) / 4;
    #pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < J; ++j) {
        const double *pj = p + (size_t)K * j;
        double *H = XtX + (size_t)K * K * j;
        double *z = Xtz + (size_t)K * j;
        for (int a = 0; a < K * K; ++a) H[a] = 0.0;
        for (int k = 0; k < K; ++k) z[k] = 0.0;
        for (int64_t i = 0; i < I; ++i) {
            const double *qi = q + (size_t)K * i;
            int c = code_at(bed, Ib, i, j);
            double g, nm;
            cell_gnm(c, j, &g, &nm);
            double qp = qp_cell(qi, pj, K);
            double oq = 1.0 - qp;
            for (int k = 0; k < K; ++k) {
                z[k] += nm * (g * qi[k] / qp - (2.0 - g) * qi[k] / oq);
                for (int k2 = 0; k2 < K; ++k2)
                    H[k2 + K * k] += nm * (g / (qp * qp) * qi[k] * qi[k2] +
                                           (2.0 - g) / (oq * oq) * qi[k] * qi[k2]);
            }
        }
    }
}

/* ------------------------------------------------------------------ QP (qp.jl) */

/* V' of svd(ones(1,K), full=true) (structs.jl:180).  LAPACK's gesdd reduces a 1xK row by
 * one Householder reflector H = I - tau v v' (dlarfg on ones(K)) and returns V' = H as
 * generated by dorgl2; the 1x1 bidiagonal SVD puts the sign into U.  Written column-major. */
void orc_vt_ones(int K, double *vt)
{
    for (int a = 0; a < K * K; ++a) vt[a] = 0.0;
    if (K == 1) { vt[0] = 1.0; return; }
    double alpha = 1.0, xnorm = sqrt((double)(K - 1));
    double w = fmax(fabs(alpha), fabs(xnorm)), z = fmin(fabs(alpha), fabs(xnorm));
    double nrm = w * sqrt(1.0 + (z / w) * (z / w));
    double beta = -copysign(nrm, alpha);
    double tau = (beta - alpha) / beta;
    double vs = 1.0 / (alpha - beta);            /* v(2:K) = ones * (1/(alpha-beta)) */
    /* row 1 */
    vt[0] = 1.0 - tau;
    for (int c = 1; c < K; ++c) vt[0 + K * c] = -tau * vs;
    /* rows 2..K: e_r - tau v_r v' (dger: A += x * (alpha*y)) */
    for (int r = 1; r < K; ++r) {
        double vr = vs;
        for (int c = 0; c < K; ++c) {
            double vc = (c == 0) ? 1.0 : vs;
            vt[r + K * c] = ((r == c) ? 1.0 : 0.0) + vr * (-tau * vc);
        }
    }
}

/* sweep! (qp.jl:297-317): sweep (inverse=0) or inverse-sweep (inverse=1) the n x n
 * symmetric tableau on diagonal entry k (0-based). */
void orc_sweep(double *A, int n, int k, double *tmp, int inverse)
{
    double piv = 1.0 / A[k + n * k];
    for (int i = 0; i < n; ++i) {
        tmp[i] = A[i + n * k];
        A[i + n * k] = 0.0;
        A[k + n * i] = 0.0;
    }
    tmp[k] = inverse ? 1.0 : -1.0;
    for (int i = 0; i < n; ++i) {
        double pv = piv * tmp[i];
        for (int j = 0; j < n; ++j) A[j + n * i] = A[j + n * i] - pv * tmp[j];
    }
}

/* create_tableau! (qp.jl:8-76) for the simplex (n = K+2) and box (n = K+1) cases.
 * H is the K x K matrix_q, r the linear term (already negated gradient), x the current
 * parameter.  mu_mode selects the mu constant of the simplex branch. */
void orc_create_tableau(double *tab, const double *H, const double *r, const double *x,
                        const double *vt, int K, int simplex, int mu_mode, double *tmp_k)
{
    int n = simplex ? K + 2 : K + 1;
    for (int a = 0; a < n * n; ++a) tab[a] = 0.0;
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i) tab[i + n * j] = H[i + K * j];
    for (int i = 0; i < K; ++i) { tab[(n - 1) + n * i] = -r[i]; tab[i + n * (n - 1)] = -r[i]; }
    tab[(n - 1) + n * (n - 1)] = 0.0;
    if (!simplex) return;
    double mu = 0.0;
    if (mu_mode == ORC_MU_GERSHGORIN) {
        /* tmp_k = H * vt[:,1]; tmp_k = vt * tmp_k; mu = 2 (|tmp|_1 - 2 tmp[1]) / K */
        double *t1 = tmp_k, t2[64];
        for (int i = 0; i < K; ++i) { double s = 0.0; for (int j = 0; j < K; ++j) s += H[i + K * j] * vt[j]; t1[i] = s; }
        for (int i = 0; i < K; ++i) { double s = 0.0; for (int j = 0; j < K; ++j) s += vt[i + K * j] * t1[j]; t2[i] = s; }
        double n1 = 0.0;
        for (int i = 0; i < K; ++i) n1 += fabs(t2[i]);
        mu = (n1 - 2.0 * t2[0]) / K;
        mu = 2.0 * mu;
    }
    /* mu_mode == ORC_MU_AS_EXECUTED: mul!(tmp_k, v, tmp_k) aliases output and input; BLAS
     * gemv with beta = 0 clears y (== x) before accumulating, so tmp_k == 0 and mu == 0. */
    for (int j = 0; j < K; ++j)
        for (int i = 0; i < K; ++i) tab[i + n * j] += mu;
    for (int i = 0; i < K; ++i) { tab[(K) + n * i] = 1.0; tab[i + n * K] = 1.0; }
    tab[K + n * K] = 0.0;
    double sx = 0.0;
    for (int i = 0; i < K; ++i) sx += x[i];
    tab[(K + 1) + n * K] = tab[K + n * (K + 1)] = 1.0 - sx;
    tab[(K + 1) + n * (K + 1)] = 0.0;
}

/* quadratic_program! (qp.jl:171-292): Jennrich-Sampson active-set sweep solver.
 * Returns the iteration at which it stopped (>0) or 0 on failure, like the reference.
 * n = p + c + 1 is the tableau order; d, tmp have length n, swept length p. */
int orc_quadratic_program(double *delta, double *tab, const double *par,
                          const double *pmin, const double *pmax, int p, int c,
                          double *d, double *tmp, int *swept)
{
    const int n = p + c + 1;
    const double small = 1e-5, tol = 1e-8;
    for (int i = 0; i < p; ++i) delta[i] = 0.0;
    for (int i = 0; i < n; ++i) d[i] = tab[i + n * i];
    for (int i = 0; i < p; ++i) {
        if (d[i] <= 0.0 || tab[i + n * i] < d[i] * tol) return 0;
        orc_sweep(tab, n, i, tmp, 0);
    }
    for (int i = 0; i < p; ++i) swept[i] = 1;
    for (int i = p; i < p + c; ++i) {
        if (tab[i + n * i] >= 0.0) return 0;
        orc_sweep(tab, n, i, tmp, 0);
    }
    const int e = n - 1;
    for (int iteration = 1; iteration <= 1000; ++iteration) {
        double a = 1.0;
        for (int i = 0; i < p; ++i) {
            if (swept[i]) {
                double ui = tab[i + n * e], ai;
                if (ui > 0.0) ai = pmax[i] - par[i] - delta[i];
                else          ai = pmin[i] - par[i] - delta[i];
                if (fabs(ui) > 1e-10) a = fmin(a, ai / ui);
            }
        }
        for (int i = 0; i < p; ++i) {
            if (swept[i]) {
                double ui = tab[i + n * e];
                delta[i] = delta[i] + a * ui;
                tab[i + n * e] = (1.0 - a) * ui;
                tab[e + n * i] = tab[i + n * e];
            }
        }
        int cycle = 0;
        for (int i = 0; i < p; ++i) {
            int critical = pmin[i] >= par[i] + delta[i] - small;
            critical = critical || pmax[i] <= par[i] + delta[i] + small;
            if (swept[i] && fabs(tab[i + n * i]) > 1e-10 && critical) {
                orc_sweep(tab, n, i, tmp, 1);
                swept[i] = 0;
                cycle = 1;
                break;
            }
        }
        if (cycle) continue;
        for (int i = 0; i < p; ++i) {
            double ui = tab[i + n * e];
            int violation = ui > 0.0 && pmin[i] >= par[i] + delta[i] - small;
            violation = violation || (ui < 0.0 && pmax[i] <= par[i] + delta[i] + small);
            if (!swept[i] && violation) {
                orc_sweep(tab, n, i, tmp, 0);
                swept[i] = 1;
                cycle = 1;
                break;
            }
        }
        if (cycle) continue;
        return iteration;
    }
    return 0;
}

/* ------------------------------------------------------------------ projections */

/* project_q! (projections.jl:27-59): Euclidean projection of b - pc onto the simplex of
 * mass 1 - n pc, plus pc.  The reference sorts with a hand-written quicksort (qsortperm!);
 * only the sorted VALUES enter the arithmetic and equal values are interchangeable, so any
 * descending sort gives the same bits.  This uses insertion sort. */
void orc_project_q1(double *b, int n, double pseudocount)
{
    double tau = 1.0 - n * pseudocount;
    double s[64];
    for (int i = 0; i < n; ++i) b[i] -= pseudocount;
    for (int i = 0; i < n; ++i) {
        double v = b[i]; int k = i;
        while (k > 0 && s[k - 1] < v) { s[k] = s[k - 1]; --k; }
        s[k] = v;
    }
    double tsum = 0.0, tmax = 0.0;
    int bget = 0;
    for (int i = 0; i < n - 1; ++i) {
        tsum += s[i];
        tmax = (tsum - tau) / (i + 1);
        if (tmax >= s[i + 1]) { bget = 1; break; }
    }
    if (!bget) tmax = (tsum + s[n - 1] - tau) / n;
    for (int i = 0; i < n; ++i) b[i] = fmax(b[i] - tmax, 0.0);
    for (int i = 0; i < n; ++i) b[i] += pseudocount;
}

void orc_project_q(double *q, int64_t I, int K)
{
    for (int64_t i = 0; i < I; ++i) orc_project_q1(q + (size_t)K * i, K, 1e-5);
}

/* project_p! (projections.jl:69-74): clamp to [pc, 1 - pc]. */
void orc_project_p(double *p, int64_t n)
{
    const double pc = 1e-5;
    for (int64_t i = 0; i < n; ++i) p[i] = fmin(fmax(p[i], pc), 1.0 - pc);
}

/* ------------------------------------------------------------------ state + outer loop */

typedef struct {
    int64_t I, J;
    int32_t K, Q;
    const uint8_t *bed;
    double *x, *x_next, *x_next2, *x_tmp;      /* K*(I+J) each */
    double *XtX_q, *Xtz_q, *XtX_p, *Xtz_p;
    double *U, *V;                              /* K(I+J) x Q */
    double *vt;                                 /* K x K */
    double ll_prev, ll_new;
    int32_t mu_mode;
    int32_t fix;                                /* bit 0: fix_q, bit 1: fix_p (algorithms_outer.jl:98-116) */
    int32_t mode;                               /* 0 = :ZAL, 1 = :LBQN (algorithms_outer.jl:126-137) */
    double *x_q, *x_r;                          /* LBQN work vectors, K*(I+J) each (structs.jl x_qq, x_rr) */
} orc_state;

static double *Qof(orc_state *s, double *x) { (void)s; return x; }
static double *Pof(orc_state *s, double *x) { return x + (size_t)s->K * s->I; }

/* update_q! (algorithms_inner.jl:167-231), CPU branch. */
/* The per-problem QP loop of update_q! / update_p! (algorithms_inner.jl:205-221, 281-298):
 * for each of n problems, the tableau of (XtX, r = -Xtz, x) (simplex form for the Q block, box
 * form for the P block) and quadratic_program!; delta (K x n) receives the steps and status (n,
 * may be NULL) the return values.  Exported on its own so a test can run the QPs on sums that
 * came from elsewhere (the engine's). */
void orc_qp_batch(const double *XtX, const double *r, const double *x, const double *vt, int K, int64_t n,
                  int simplex, int mu_mode, double *delta, int32_t *status)
{
    #pragma omp parallel
    {
        int m = simplex ? K + 2 : K + 1;
        double *tab = (double *)malloc(sizeof(double) * m * m);
        double *tk = (double *)malloc(sizeof(double) * (K + 2));
        double *d = (double *)malloc(sizeof(double) * m);
        double *tmp = (double *)malloc(sizeof(double) * m);
        double *pmin = (double *)calloc(K, sizeof(double));
        double *pmax = (double *)malloc(sizeof(double) * K);
        int *swept = (int *)malloc(sizeof(int) * K);
        for (int k = 0; k < K; ++k) pmax[k] = 1.0;
        #pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < n; ++i) {
            orc_create_tableau(tab, XtX + (size_t)K * K * i, r + (size_t)K * i, x + (size_t)K * i, vt, K,
                               simplex, mu_mode, tk);
            int st = orc_quadratic_program(delta + (size_t)K * i, tab, x + (size_t)K * i, pmin, pmax, K,
                                           simplex ? 1 : 0, d, tmp, swept);
            if (status) status[i] = st;
        }
        free(tab); free(tk); free(d); free(tmp); free(pmin); free(pmax); free(swept);
    }
}

void orc_update_q(orc_state *s, int update2, int32_t *status)
{
    const int K = s->K;
    const int64_t I = s->I, J = s->J;
    double *q_next = update2 ? Qof(s, s->x_next2) : Qof(s, s->x_next);
    double *q      = update2 ? Qof(s, s->x_next)  : Qof(s, s->x);
    double *p      = update2 ? Pof(s, s->x_next)  : Pof(s, s->x);
    double *qdiff  = Qof(s, s->x_tmp);
    s->ll_prev = s->ll_new;
    orc_grad_hess_q(s->bed, I, J, K, q, p, s->XtX_q, s->Xtz_q);
    for (int64_t a = 0; a < (int64_t)K * I; ++a) s->Xtz_q[a] *= -1.0;
    orc_qp_batch(s->XtX_q, s->Xtz_q, q, s->vt, K, I, 1, s->mu_mode, qdiff, status);
    for (int64_t a = 0; a < (int64_t)K * I; ++a) q_next[a] = q[a] + qdiff[a];
    orc_project_q(q_next, I, K);
}

/* update_p! (algorithms_inner.jl:245-310), CPU branch.  Note q is q_next / q_next2. */
void orc_update_p(orc_state *s, int update2, int32_t *status)
{
    const int K = s->K;
    const int64_t I = s->I, J = s->J;
    double *p_next = update2 ? Pof(s, s->x_next2) : Pof(s, s->x_next);
    double *q      = update2 ? Qof(s, s->x_next2) : Qof(s, s->x_next);
    double *p      = update2 ? Pof(s, s->x_next)  : Pof(s, s->x);
    double *pdiff  = Pof(s, s->x_tmp);
    s->ll_prev = s->ll_new;
    orc_grad_hess_p(s->bed, I, J, K, q, p, s->XtX_p, s->Xtz_p);
    for (int64_t a = 0; a < (int64_t)K * J; ++a) s->Xtz_p[a] *= -1.0;
    orc_qp_batch(s->XtX_p, s->Xtz_p, p, s->vt, K, J, 0, s->mu_mode, pdiff, status);
    for (int64_t a = 0; a < (int64_t)K * J; ++a) p_next[a] = p[a] + pdiff[a];
    orc_project_p(p_next, (int64_t)K * J);
}

double orc_loglik_x(orc_state *s, const double *x)
{
    return orc_loglik(s->bed, s->I, s->J, s->K, x, x + (size_t)s->K * s->I);
}

/* init_em! (algorithms_outer.jl:12-45), CPU branch.  ll_hist[it] receives the
 * log-likelihood printed after each EM iteration; s->ll_new the final one. */
void orc_init_em(orc_state *s, int iters, double *ll_hist)
{
    const int K = s->K;
    const int64_t I = s->I, J = s->J;
    double *q = Qof(s, s->x), *p = Pof(s, s->x);
    double *q_next = Qof(s, s->x_next), *p_next = Pof(s, s->x_next);
    for (int it = 0; it < iters; ++it) {
        orc_em_q(s->bed, I, J, K, q, p, q_next);
        orc_em_p(s->bed, I, J, K, q, p, p_next);
        memcpy(p, p_next, sizeof(double) * (size_t)K * J);
        memcpy(q, q_next, sizeof(double) * (size_t)K * I);
        double ll = orc_loglik(s->bed, I, J, K, q, p);
        if (ll_hist) ll_hist[it] = ll;
    }
    s->ll_new = orc_loglik(s->bed, I, J, K, q, p);
}

/* inv(M) for a small m x m matrix by Gauss-Jordan with partial pivoting. */
static int small_inv(double *M, int m, double *out)
{
    double a[8 * 16];
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < 2 * m; ++j)
            a[i * 2 * m + j] = (j < m) ? M[i + m * j] : (j - m == i ? 1.0 : 0.0);
    for (int c = 0; c < m; ++c) {
        int piv = c;
        for (int r = c + 1; r < m; ++r)
            if (fabs(a[r * 2 * m + c]) > fabs(a[piv * 2 * m + c])) piv = r;
        if (a[piv * 2 * m + c] == 0.0) return -1;
        if (piv != c)
            for (int j = 0; j < 2 * m; ++j) {
                double t = a[c * 2 * m + j]; a[c * 2 * m + j] = a[piv * 2 * m + j]; a[piv * 2 * m + j] = t;
            }
        double d = a[c * 2 * m + c];
        for (int j = 0; j < 2 * m; ++j) a[c * 2 * m + j] /= d;
        for (int r = 0; r < m; ++r) {
            if (r == c) continue;
            double f = a[r * 2 * m + c];
            if (f != 0.0) for (int j = 0; j < 2 * m; ++j) a[r * 2 * m + j] -= f * a[c * 2 * m + j];
        }
    }
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) out[i + m * j] = a[i * 2 * m + m + j];
    return 0;
}

/* update_UV! (quasi_newton.jl:5-9) and update_QN! (quasi_newton.jl:29-31):
 * U[:,c] = x1 - x0, V[:,c] = x2 - x1, c = (iter-1)%Q; x_tmp = x1 - V inv(U'(U-V)) U'(x0-x1)
 * over the first min(iter, Q) columns. */
void orc_qn_step(orc_state *s, int iter)
{
    const int64_t n = (int64_t)s->K * (s->I + s->J);
    const int Q = s->Q;
    int col = (iter - 1) % Q;
    double *U = s->U, *V = s->V;
    for (int64_t a = 0; a < n; ++a) {
        V[a + n * col] = s->x_next2[a] - s->x_next[a];
        U[a + n * col] = s->x_next[a] - s->x[a];
    }
    int m = iter < Q ? iter : Q;
    double M[64], Mi[64], b[8], cf[8];
    for (int r = 0; r < m; ++r) {
        for (int c2 = 0; c2 < m; ++c2) {
            double acc = 0.0;
            for (int64_t a = 0; a < n; ++a) acc += U[a + n * r] * (U[a + n * c2] - V[a + n * c2]);
            M[r + m * c2] = acc;
        }
        double acc = 0.0;
        for (int64_t a = 0; a < n; ++a) acc += U[a + n * r] * (s->x[a] - s->x_next[a]);
        b[r] = acc;
    }
    if (small_inv(M, m, Mi) != 0) {
        for (int r = 0; r < m * m; ++r) Mi[r] = NAN;   /* inv of a singular matrix: non-finite */
    }
    for (int r = 0; r < m; ++r) {
        double acc = 0.0;
        for (int c2 = 0; c2 < m; ++c2) acc += Mi[r + m * c2] * b[c2];
        cf[r] = acc;
    }
    for (int64_t a = 0; a < n; ++a) {
        double acc = 0.0;
        for (int r = 0; r < m; ++r) acc += V[a + n * r] * cf[r];
        s->x_tmp[a] = s->x_next[a] - acc;
    }
}

/* update_UV_LBQN! (quasi_newton.jl:15-23) then update_QN_LBQN! (quasi_newton.jl:38-58) on the
 * first m = min(iter, Q) columns, written out as the reference's vector operations. */
static double orc_dot(const double *a, const double *b, int64_t n)
{
    double acc = 0.0;
    for (int64_t t = 0; t < n; ++t) acc += a[t] * b[t];
    return acc;
}

void orc_qn_step_lbqn(orc_state *s, int iter)
{
    const int64_t n = (int64_t)s->K * (s->I + s->J);
    const int Q = s->Q;
    double *U = s->U, *V = s->V;
    for (int c = (iter < Q ? iter : Q) - 1; c >= 1; --c) {          /* for i in min(iter, Q):-1:2 */
        memcpy(U + n * c, U + n * (c - 1), sizeof(double) * (size_t)n);
        memcpy(V + n * c, V + n * (c - 1), sizeof(double) * (size_t)n);
    }
    for (int64_t a = 0; a < n; ++a) {
        U[a] = s->x_next[a] - s->x[a];
        V[a] = s->x_next2[a] - s->x_next[a];
        V[a] = V[a] - U[a];                                           /* x2 - 2x1 + x0 */
    }
    const int m = iter < Q ? iter : Q;
    const double gamma = orc_dot(U, V, n) / orc_dot(V, V, n);
    double alpha[8];
    memcpy(s->x_q, U, sizeof(double) * (size_t)n);
    for (int i = 0; i < m; ++i) {
        const double *Vi = V + n * i;
        const double rho = 1.0 / orc_dot(Vi, Vi, n);
        alpha[i] = rho * orc_dot(Vi, s->x_q, n);
        for (int64_t a = 0; a < n; ++a) s->x_q[a] = s->x_q[a] - alpha[i] * Vi[a];
    }
    for (int64_t a = 0; a < n; ++a) s->x_r[a] = gamma * s->x_q[a];
    for (int i = 0; i < m; ++i)
        for (int64_t a = 0; a < n; ++a) s->x_r[a] = s->x_r[a] + alpha[i] * U[a + n * i];
    for (int64_t a = 0; a < n; ++a) s->x_tmp[a] = s->x[a] - s->x_r[a];
}

/* One iteration of admixture_qn! (algorithms_outer.jl:92-159), mode = :ZAL or :LBQN (s->mode).  With fix_q / fix_p
 * (s->fix bits 0 / 1) the block is copied instead of updated: q_next .= q, q_next2 .= q
 * (algorithms_outer.jl:98-116), likewise p.  info[0..4] = (prev, basic, qn, new, reldiff).
 * Returns 1 when reldiff < rtol. */
int orc_qn_iteration(orc_state *s, int iter, double rtol, double *info,
                     int32_t *st_q, int32_t *st_p)
{
    const int K = s->K;
    const int64_t I = s->I, J = s->J;
    s->ll_prev = s->ll_new;
    double ll_prev = s->ll_prev;
    const size_t nq = sizeof(double) * (size_t)K * I, np = sizeof(double) * (size_t)K * J;
    if (s->fix & 1) memcpy(Qof(s, s->x_next), Qof(s, s->x), nq); else orc_update_q(s, 0, st_q);
    if (s->fix & 2) memcpy(Pof(s, s->x_next), Pof(s, s->x), np); else orc_update_p(s, 0, st_p);
    if (s->fix & 1) memcpy(Qof(s, s->x_next2), Qof(s, s->x), nq); else orc_update_q(s, 1, st_q);
    if (s->fix & 2) memcpy(Pof(s, s->x_next2), Pof(s, s->x), np); else orc_update_p(s, 1, st_p);
    s->ll_prev = ll_prev;
    double ll_basic = orc_loglik_x(s, s->x_next2);
    if (s->mode == 1) orc_qn_step_lbqn(s, iter); else orc_qn_step(s, iter);
    orc_project_p(Pof(s, s->x_tmp), (int64_t)K * J);
    orc_project_q(Qof(s, s->x_tmp), I, K);
    double ll_qn = orc_loglik_x(s, s->x_tmp);
    const int64_t n = (int64_t)K * (I + J);
    if (s->ll_prev < ll_qn) { memcpy(s->x, s->x_tmp, sizeof(double) * (size_t)n); s->ll_new = ll_qn; }
    else { memcpy(s->x, s->x_next2, sizeof(double) * (size_t)n); s->ll_new = ll_basic; }
    double reldiff = fabs((s->ll_new - s->ll_prev) / s->ll_prev);
    if (info) { info[0] = s->ll_prev; info[1] = ll_basic; info[2] = ll_qn; info[3] = s->ll_new; info[4] = reldiff; }
    return reldiff < rtol;
}

/* admixture_qn! (algorithms_outer.jl:63-193).  hist receives 5 doubles per iteration.
 * Returns the number of iterations run; *converged is set like the reference's flag. */
int orc_admixture_qn(orc_state *s, int n_iter, double rtol, int iter_offset,
                     double *hist, int *converged)
{
    if (isnan(s->ll_new)) s->ll_new = orc_loglik_x(s, s->x);
    *converged = 0;
    int done = 0;
    for (int it = iter_offset + 1; it <= n_iter; ++it) {
        double info[5];
        int stop = orc_qn_iteration(s, it, rtol, info, NULL, NULL);
        if (hist) memcpy(hist + 5 * (size_t)done, info, sizeof(info));
        ++done;
        if (stop) { *converged = 1; break; }
    }
    return done;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
