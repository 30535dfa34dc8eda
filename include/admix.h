/*
 * admix.h -- C ABI of libadmix, the B200 (sm_100a) engine for OpenADMIXTURE.jl's
 * per-iteration likelihood / gradient / Hessian sweeps, block SQP updates and ZAL
 * quasi-Newton extrapolation.
 *
 * Plain C types only (pointers, sizes, status codes); one opaque handle per cohort.
 * Every entry point is synchronous: work is stream-ordered on the handle's stream and
 * the call returns after cudaStreamSynchronize (the reference wraps each GPU call in
 * CUDA.@sync, cuda/runners.jl:8,30,54,77,99).  A handle is not re-entrant; use one per
 * host thread.  Every call returns ADMIX_OK (0) or an error code, and the message is
 * available from admix_last_error().
 *
 * Array layout is the reference's (Julia column-major, structs.jl:16-43):
 *   bed : uint8 [ceil(I/4)] x J, SNP-major, PLINK 2-bit codes, no 3-byte magic
 *         (the SnpArray data matrix g_la.s.data, cuda/structs.jl:37)
 *   q   : K x I doubles,  p : K x J doubles   (x = [q p], K x (I+J))
 *   XtX : K x K x n doubles, Xtz : K x n doubles (n = I for the Q block, J for the P block)
 */
#ifndef ADMIX_H
#define ADMIX_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define ADMIX_OK               0
#define ADMIX_ERR_ARG          1   /* bad argument (the reference raises AssertionError) */
#define ADMIX_ERR_CUDA         2   /* CUDA runtime error */
#define ADMIX_ERR_NOMEM        3   /* device allocation failed */
#define ADMIX_ERR_UNSUPPORTED  4   /* size or option outside what the library supports */
#define ADMIX_ERR_STATE        5   /* call made in the wrong state */

/* buffer selectors: the reference's x, x_next, x_next2, x_tmp (structs.jl:16-19) */
#define ADMIX_X        0
#define ADMIX_X_NEXT   1
#define ADMIX_X_NEXT2  2
#define ADMIX_X_TMP    3

/* admix_create flags */
#define ADMIX_FLAG_MU_GERSHGORIN  1u  /* simplex tableau adds the Gerschgorin mu of qp.jl:54-58
                                          (default: mu = 0, what the aliased mul! yields) */
/* ADMIX_FLAG_MIXED is also what the host API maps the reference's T = Float32 to
 * (run_admixture(...; T=Float32), AdmixData{Float32}): a deliberate change of meaning.  The
 * reference then keeps every array and every sum in Float32; this engine keeps Q, P and the sums
 * in FP64 and runs the mixed form, so a T = Float32 run here is more accurate than the
 * reference's (it reaches the FP64 optimum) and returns Float32 copies of Q and P.  Callers who
 * need the reference's Float32 rounding itself get no bit-for-bit reproduction of it. */
#define ADMIX_FLAG_MIXED          2u  /* mixed-precision form: the iteration's Q/P gradient / Hessian
                                          sweeps (tcgen05 BF16 Hessians, FP32 gradient cells, FP64
                                          sums), its log-likelihoods (FP32 cells, FP64 reduction) and
                                          admix_init_em's EM sums and its final ll_new; admix_loglik,
                                          admix_em_q/_p, the QPs and the QN step stay FP64.  A mixed call whose
                                          tensor-core pipeline wait runs out returns ADMIX_ERR_CUDA. */

#define ADMIX_FLAG_MEAN_IMPUTE    4u  /* AdmixData(...; skipmissing=false) (structs.jl:105): the loops
                                          that impute a missing genotype by its SNP's mean dosage g.mu
                                          (loglikelihood_loop, em_q_loop!, em_p_loop!, update_q_loop!,
                                          update_p_loop!; loops.jl:493-514,589-608,679-698,840-865,
                                          896-921) instead of skipping it.  g.mu is computed once at
                                          creation from the genotypes (mean over non-missing
                                          individuals).  FP64 form of a device-resident handle only:
                                          with ADMIX_FLAG_MIXED or admix_create_streamed the call
                                          returns ADMIX_ERR_UNSUPPORTED (the reference's own GPU path
                                          asserts skipmissing, algorithms_inner.jl:191,267). */

#define ADMIX_MAX_K 16
#define ADMIX_MAX_Q 8

typedef struct admix_ctx admix_ctx;

/* One quasi-Newton iteration's record (what algorithms_outer.jl:161-164 prints). */
typedef struct {
    double ll_prev;     /* log-likelihood before the iteration */
    double ll_basic;    /* after two SQP sweeps (x_next2) */
    double ll_qn;       /* at the projected quasi-Newton point (x_tmp) */
    double ll_new;      /* accepted value */
    double reldiff;     /* |ll_new - ll_prev| / |ll_prev| */
    int32_t iter;       /* iteration number i */
    int32_t accepted_qn;/* 1 when x_tmp was accepted */
    int32_t qp_fail_q;  /* simplex QPs that returned 0 (qp.jl:192,202,291) over both Q updates */
    int32_t qp_fail_p;  /* box QPs that returned 0 over both P updates */
} admix_iterinfo;

/* --- lifetime ------------------------------------------------------------------ */

/* Allocate the device state and upload the genotype bytes once.
 * Replaces _cu_admixture_base / CuAdmixData (cuda/structs.jl:16-39, driver.jl:150-155).
 * K in [1, ADMIX_MAX_K], Q in [1, ADMIX_MAX_Q]. */
int admix_create(int64_t I, int64_t J, int32_t K, int32_t Q, const uint8_t *bed,
                 uint32_t flags, admix_ctx **out);
/* Same, with the genotype bytes already on the current device (the reference's g_cu, a
 * CuMatrix{UInt8} of ceil(I/4) x J, cuda/structs.jl:36-37), columns src_pitch bytes apart
 * (src_pitch >= ceil(I/4)).  The bytes are copied; the caller keeps ownership of d_bed. */
int admix_create_device(int64_t I, int64_t J, int32_t K, int32_t Q, const uint8_t *d_bed, int64_t src_pitch,
                        uint32_t flags, admix_ctx **out);
/* Out-of-core variant of admix_create for cohorts whose packed genotypes do not fit in device
 * memory (the reference needs the whole BED on the device, cuda/structs.jl:36-37): the genotypes
 * stay in the caller's host memory -- page-locked in place for the handle's lifetime, so they
 * must stay valid and unchanged until admix_destroy -- and every pass streams them in blocks of
 * block_snps SNPs (a positive multiple of 32) through two device buffers, the copy of the next
 * block overlapping the compute of the current one.  Results equal admix_create's up to the
 * order of the FP64 sums. */
int admix_create_streamed(int64_t I, int64_t J, int32_t K, int32_t Q, const uint8_t *bed, int64_t block_snps,
                          uint32_t flags, admix_ctx **out);
int admix_destroy(admix_ctx *h);
/* Last error message of h (or of the calling thread's last failed admix_create when h is NULL). */
const char *admix_last_error(const admix_ctx *h);
/* Device bytes held by the handle. */
int admix_device_bytes(const admix_ctx *h, int64_t *bytes);

/* --- state transfer (copyto_sync!, cuda/transfer.jl:1-7) ------------------------ */

/* Upload / download q (K x I) and p (K x J) of buffer `which`; either pointer may be NULL. */
int admix_set_x(admix_ctx *h, int32_t which, const double *q, const double *p);
int admix_get_x(admix_ctx *h, int32_t which, double *q, double *p);
/* d.ll_new of AdmixData (structs.jl:89-90), used by admixture_qn!'s first iteration. */
int admix_set_ll(admix_ctx *h, double ll_new);
int admix_get_ll(admix_ctx *h, double *ll_new);

/* --- sweeps ------------------------------------------------------------------------ */

/* Log-likelihood of buffer `which` (loglikelihood(d_cu, g_cu), cuda/runners.jl:13-20;
 * loglikelihood(g::SnpLinAlg, ...), algorithms_inner.jl:27-35).  FP64 accumulation. */
int admix_loglik(admix_ctx *h, int32_t which, double *out);

/* EM priming half-steps on buffer ADMIX_X (em_q!/em_p!, cuda/runners.jl:22-67;
 * algorithms_inner.jl:68-141): q_next = EM_Q(q, p); p_next = EM_P(q, p). */
int admix_em_q(admix_ctx *h);
int admix_em_p(admix_ctx *h);
/* init_em! (algorithms_outer.jl:12-45): `iters` EM iterations, ll_hist[iters] (may be NULL),
 * then sets ll_new (with ADMIX_FLAG_MIXED from the mixed log-likelihood pass that the iterations
 * use, not from admix_loglik's FP64 pass). */
int admix_init_em(admix_ctx *h, int32_t iters, double *ll_hist);

/* Gradient / Hessian sweep of the Q block at (q of which_q, p of which_p), written to the
 * host in the reference layout (update_q_cuda!, cuda/runners.jl:69-89;
 * update_q_loop_skipmissing!, loops.jl:867-894).  XtX: K x K x I, Xtz: K x I; either may be NULL. */
int admix_grad_hess_q(admix_ctx *h, int32_t which_q, int32_t which_p, double *XtX, double *Xtz);
/* Same for the P block (update_p_cuda!, cuda/runners.jl:91-111; loops.jl:923-950).
 * XtX: K x K x J, Xtz: K x J. */
int admix_grad_hess_p(admix_ctx *h, int32_t which_q, int32_t which_p, double *XtX, double *Xtz);

/* --- block SQP updates (update_q! / update_p!, algorithms_inner.jl:167-310) ------ */

/* update2 = 0: q_next = SQP_Q(q, p);        update2 = 1: q_next2 = SQP_Q(q_next, p_next).
 * qp_status (length I, may be NULL) receives quadratic_program!'s return value per problem. */
int admix_update_q(admix_ctx *h, int32_t update2, int32_t *qp_status);
/* update2 = 0: p_next = SQP_P(q_next, p);   update2 = 1: p_next2 = SQP_P(q_next2, p_next). */
int admix_update_p(admix_ctx *h, int32_t update2, int32_t *qp_status);

/* --- outer loop (admixture_qn!, algorithms_outer.jl:63-193, mode = :ZAL) ----------- */

/* One full iteration i on the device: 2 Q + 2 P SQP updates, loglik, ZAL secant update
 * (quasi_newton.jl:5-9,29-31), projection (projections.jl), loglik, accept/reject. */
/* fix_q / fix_p of admixture_qn! (algorithms_outer.jl:63-116, passed through by run_admixture,
 * driver.jl:169-197): later iterations (admix_qn_iteration, admix_run_qn, batches) copy the fixed
 * block (q_next .= q, q_next2 .= q, likewise p) instead of updating it.  Default: neither. */
int admix_set_fixed(admix_ctx *h, int32_t fix_q, int32_t fix_p);
/* (No counterpart in the reference.)  Self-test of the mixed form's failure reporting: runs a
 * kernel whose bounded mbarrier wait nothing completes, so it gives up after 1024 polls and sets
 * the error flag exactly as a tensor-core sweep's pipeline wait would; returns ADMIX_ERR_CUDA
 * with the same message, and the flag is cleared, so the handle stays usable.  Mixed-form
 * handles only (ADMIX_ERR_STATE otherwise). */
int admix_selftest_wait_timeout(admix_ctx *h);
/* --- SKFR AIM pre-selection (run_admixture's sparsity keyword, driver.jl:56-69; _filter_SKFR,
 * driver.jl:80-101; the reference calls the third-party SparseKmeansFeatureRanking.jl) ---------
 * Sparse k-means via feature ranking on the handle's genotypes, imputed and standardised per SNP:
 * k-means++ seeding from a splitmix64 stream (seed), then centres, per-SNP scores, the `sparsity`
 * SNPs of largest score kept and individuals reassigned on them, until no assignment changes or
 * max_iter iterations; mode ADMIX_SKFR_GLOBAL keeps one SNP set for all clusters
 * (sparsekmeans1), ADMIX_SKFR_LOCAL one per cluster (sparsekmeans2; the AIMs are their union).
 * tries > 1 repeats from new seeds (the stream continues) and keeps the run of least
 * within-cluster sum of squares (sparsekmeans_repeat).  k clusters (1..16).  Outputs: clusters
 * (I cluster indices 0..k-1), aims (the selected SNPs, 0-based, increasing; at most
 * aims_capacity written, *n_aims = how many there are), objective, iterations of the kept run.
 * Device-resident handles only (ADMIX_ERR_UNSUPPORTED for streamed ones). */
#define ADMIX_SKFR_GLOBAL 0
#define ADMIX_SKFR_LOCAL  1
int admix_skfr(admix_ctx *h, int32_t k, int64_t sparsity, int32_t mode, int32_t max_iter, int32_t tries,
               uint64_t seed, int32_t *clusters, int32_t *aims, int64_t aims_capacity, int64_t *n_aims,
               double *objective, int32_t *iterations);
/* (No counterpart in the reference.)  Diagnostic of the tensor-core arithmetic the mixed form is
 * designed around: d[128 x 16] (row-major FP32) = sum over K-steps s < nsteps (1..4) of
 * A[:, 16s:16s+16] * B[:, 16s:16s+16]^T, one tcgen05 BF16 MMA per step with the FP32 accumulator
 * in tensor memory.  a: 128 x 64 and b: 16 x 64 row-major BF16 bit patterns (host memory);
 * a_in_tmem = 1 reads A from tensor memory instead of shared memory.  Returns ADMIX_OK,
 * ADMIX_ERR_ARG or ADMIX_ERR_CUDA (no message; no handle needed). */
int admix_tc_probe(const uint16_t *a, const uint16_t *b, float *d, int32_t nsteps, int32_t a_in_tmem);
int admix_qn_iteration(admix_ctx *h, int32_t iter, admix_iterinfo *out);
/* admixture_qn!'s `mode` keyword (algorithms_outer.jl:63-65,126-137): ADMIX_QN_ZAL (default,
 * update_UV! / update_QN!, quasi_newton.jl:5-9,29-31) or ADMIX_QN_LBQN (limited-memory Broyden,
 * update_UV_LBQN! / update_QN_LBQN!, quasi_newton.jl:15-58).  Later iterations (admix_qn_iteration,
 * admix_run_qn, batches) use it; the secant history U, V is shared, as in the reference, so
 * switching modes in the middle of a run mixes the two modes' columns. */
#define ADMIX_QN_ZAL   0
#define ADMIX_QN_LBQN  1
int admix_set_qn_mode(admix_ctx *h, int32_t mode);
/* Iterations iter_offset+1 .. n_iter until reldiff < rtol.  hist (n_iter entries, may be
 * NULL) receives one record per iteration run. */
int admix_run_qn(admix_ctx *h, int32_t n_iter, double rtol, int32_t iter_offset,
                 admix_iterinfo *hist, int32_t *n_done, int32_t *converged);

/* --- instrumentation ------------------------------------------------------------------- */

/* The cudaStream_t (as void*) all of the handle's work is ordered on, so a caller can record
 * events on it or order its own work after the engine's. */
int admix_stream(admix_ctx *h, void **stream);

/* Pass identifiers for admix_time_pass */
#define ADMIX_PASS_LOGLIK   0   /* decode + qp + log reduction over x (loops.jl:517-539) */
#define ADMIX_PASS_QSWEEP   1   /* Q-block gradient / Hessian sweep (loops.jl:867-894) */
#define ADMIX_PASS_PSWEEP   2   /* P-block gradient / Hessian sweep (loops.jl:923-950) */
#define ADMIX_PASS_QQP      3   /* batched simplex QPs + projection of the Q block */
#define ADMIX_PASS_PQP      4   /* batched box QPs + projection of the P block */
#define ADMIX_PASS_EM       5   /* one EM priming iteration (em_q + em_p) */

/* Device time of `reps` back-to-back launches of one pass on the current buffers, measured
 * with CUDA events on the handle's stream; *ms_per_launch receives the mean.  The QP passes
 * solve the problems of the last sweep again (their outputs go to x_tmp). */
int admix_time_pass(admix_ctx *h, int32_t pass, int32_t reps, double *ms_per_launch);

/* Number of kernel launches in one captured quasi-Newton iteration (graph kernel nodes). */
int admix_iteration_kernels(admix_ctx *h, int32_t *count);

/* --- genotype decode ----------------------------------------------------------------- */

/* Missing-code (01) counts per SNP (length J) and per individual (length I); either may
 * be NULL.  Bit-exact integer counts of the decode rule of loops.jl:529-534. */
int admix_decode_counts(admix_ctx *h, int64_t *miss_per_snp, int64_t *miss_per_ind);

/* --- stateless device-pointer entry point --------------------------------------------- */

/* loglikelihood(g::CuArray{UInt8,2}, q::CuArray, p::CuArray, I, J) (cuda/runners.jl:2-11)
 * on caller-owned device memory.  d_work must hold admix_loglik_dev_workspace(I, J, K)
 * bytes; the result (one double) is written to d_out.  `stream` is a cudaStream_t
 * (NULL = legacy default stream); the call is asynchronous on that stream. */
size_t admix_loglik_dev_workspace(int64_t I, int64_t J, int32_t K);
int admix_loglik_dev(const uint8_t *d_bed, int64_t I, int64_t J, int32_t K,
                     const double *d_q, const double *d_p, double *d_out,
                     void *d_work, size_t work_bytes, void *stream);

/* No counterpart in the reference.  admix_loglik_dev for callers that cannot allocate device
 * memory (their device memory comes only from a pool they do not control, or they must not
 * pay cudaMalloc's implicit synchronisation): the partial sums live in a fixed array inside
 * the library, ADMIX_NOALLOC_MAX_PARTIALS doubles (256 KiB) held by every GPU that loads it.
 * Cohorts needing more partial sums (I beyond about 33 million) are rejected with
 * ADMIX_ERR_UNSUPPORTED.  The first call on a device looks up the array's device address
 * (make it before any stream capture); so does the first call after the device's context was
 * reset and recreated, since the array may have moved.  All calls share the array: calls that
 * overlap on the GPU race, so serialise them.  Asynchronous on `stream`; errors are reported by
 * admix_noalloc_last_error(), which a successful call clears. */
#define ADMIX_NOALLOC_MAX_PARTIALS 32768
int admix_loglik_dev_noalloc(const uint8_t *d_bed, int64_t I, int64_t J, int32_t K,
                             const double *d_q, const double *d_p, double *d_out, void *stream);
const char *admix_noalloc_last_error(void);

/* --- learned warm start (no counterpart in the reference; hooks into run_admixture's
 *     init_q / init_p, driver.jl:52-53,161-166,183-188) ---------------------------------- */

/* Sketch of each individual: dosages of the S SNPs listed in d_snps (int8, 3 = missing, I x S),
 * their allele frequencies d_freq (S), and R <= 32 projections of the frequency-standardised
 * dosages onto fixed +-1 directions drawn from `seed` (I x R).  Asynchronous on `stream`. */
int admix_sketch(const uint8_t *d_bed, int64_t pitch, int64_t I, const int32_t *d_snps, int32_t S,
                 int32_t R, uint64_t seed, float *d_freq, int8_t *d_dos, float *d_proj, void *stream);

/* MLP encoder (S + R) -> H -> H -> K: ReLU, ReLU, softmax.  Row-major FP32 device arrays:
 * w1 (S+R) x H, w2 H x H, w3 H x K, biases of length H, H, K. */
typedef struct {
    int32_t S, R, H, K;
    const float *w1, *b1, *w2, *b2, *w3, *b3;
} admix_mlp;
typedef struct {
    float *w1, *b1, *w2, *b2, *w3, *b3;
} admix_mlp_grads;

/* Forward pass of n individuals: hidden activations h1, h2 (n x H), logits and probs (n x K). */
int admix_mlp_forward(const admix_mlp *net, int64_t n, const int8_t *dos, const float *center, const float *proj,
                      float *h1, float *h2, float *logits, float *probs, void *stream);
/* Backward pass of the mean cross-entropy against soft targets (n x K): gradients into grad,
 * scratch dlogits (n x K), dh2, dh1 (n x H); the summed loss is added into *loss. */
int admix_mlp_backward(const admix_mlp *net, const admix_mlp_grads *grad, int64_t n, const int8_t *dos,
                       const float *center, const float *proj, const float *h1, const float *h2, const float *logits,
                       const float *target, float *probs, float *dlogits, float *dh2, float *dh1, float *loss,
                       void *stream);
/* One Adam step (step number t >= 1) on n parameters. */
int admix_mlp_adam(float *w, const float *g, float *m, float *v, int64_t n, float lr, float beta1, float beta2,
                   float eps, int32_t t, void *stream);
/* Starting P from a predicted Q (K x I): p_kj = sum_i nm q_ki g_ij / (2 sum_i nm q_ki), clamped to
 * [1e-5, 1 - 1e-5]; output K x J. */
int admix_warm_p(const uint8_t *d_bed, int64_t pitch, int64_t I, int64_t J, int32_t K, const double *d_q,
                 double *d_p, void *stream);

/* --- batching: random restarts and K sweeps over one cohort ----------------------------
 * The reference runs one problem per run_admixture call (driver.jl:35-75); a user who wants
 * several restarts or several K calls it once per seed / K.  A batch holds n member problems
 * (member m has K = Ks[m]; repeat a K for restarts) over ONE device copy of the genotypes.
 * Each member is an ordinary handle (admix_batch_member) for set_x / get_x / loglik / ...;
 * the batch calls below advance all members together: one batch iteration is one CUDA graph
 * launch whose independent branches are the members' captured admixture_qn! iterations, so the
 * members' kernels run concurrently.  Members that converge drop out of later launches. */
typedef struct admix_batch admix_batch;

int admix_batch_create(int64_t I, int64_t J, const uint8_t *bed, int32_t n, const int32_t *Ks, int32_t Q,
                       uint32_t flags, admix_batch **out);
/* as admix_batch_create, genotypes already on the current device at src_pitch bytes per column */
int admix_batch_create_device(int64_t I, int64_t J, const uint8_t *d_bed, int64_t src_pitch, int32_t n,
                              const int32_t *Ks, int32_t Q, uint32_t flags, admix_batch **out);
int admix_batch_destroy(admix_batch *b);
const char *admix_batch_last_error(const admix_batch *b);
int admix_batch_size(const admix_batch *b, int32_t *n);
/* borrowed handle of member m (owned by the batch; do not destroy it) */
int admix_batch_member(admix_batch *b, int32_t m, admix_ctx **h);
/* init_em! (algorithms_outer.jl:12-45) on every member, concurrently; ll_hist: n x iters or NULL */
int admix_batch_init_em(admix_batch *b, int32_t iters, double *ll_hist);
/* Work split of the members' passes: every member's sweep and log-likelihood plans are sized
 * as if it had the GPU's SM count divided by `divisor` to itself (1 = the single-problem plans). */
int admix_batch_set_split(admix_batch *b, int32_t divisor);
/* Autotuner: times one concurrent launch of every member's Q sweep, P sweep and log-likelihood
 * pass (read-only on the iterates) for divisor = 1, 2, 4, ... up to 4n, keeps the fastest and
 * applies it.  Outputs the chosen divisor and its milliseconds (either may be NULL). */
int admix_batch_autotune(admix_batch *b, int32_t *divisor, double *ms);
/* admixture_qn! on every member until it converges (reldiff < rtol) or n_iter iterations:
 * per member (arrays of length n, any may be NULL) the iterations run, whether it converged and
 * its last iteration record; ms_device = summed device time of the batch launches. */
int admix_batch_run_qn(admix_batch *b, int32_t n_iter, double rtol, int32_t *n_done, int32_t *converged,
                       admix_iterinfo *last, double *ms_device);

#ifdef __cplusplus
}
#endif
#endif
