/*
 * kernels.h -- host-side launchers of libadmix's device kernels (internal).
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include "common.cuh"

struct LoglikPlan { int gx = 1, gy = 1; int64_t jslice = 1; };
struct SweepPlan  { int gx = 1, S = 1; int64_t slice = 1; };

LoglikPlan plan_loglik(int64_t I, int64_t J, int sms);
SweepPlan plan_sweep_q(int K, int64_t I, int64_t J, int sms);
SweepPlan plan_sweep_p(int K, int64_t I, int64_t J, int sms);

/* FP64 sweeps (sweeps_f64.cu) */
cudaError_t prepare_sweeps(int K);
/* mu (J doubles, the SNP means) != nullptr selects the reference's non-skipmissing loops */
cudaError_t launch_loglik_f64(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                              const double *p, const LoglikPlan &pl, double *partial, double *out,
                              cudaStream_t st, const double *mu = nullptr);
cudaError_t launch_sweep_q_f64(int K, int mode, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                               const double *q, const double *p, const SweepPlan &pl, double *out,
                               cudaStream_t st, const double *mu = nullptr);
cudaError_t launch_sweep_p_f64(int K, int mode, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                               const double *q, const double *p, const SweepPlan &pl, double *out,
                               cudaStream_t st, const double *mu = nullptr);
/* g.mu of the SnpLinAlg: mean non-missing dosage per SNP of the padded device genotypes */
cudaError_t launch_snp_means(const uint8_t *bed, int64_t J, int64_t pitch, double *mu, cudaStream_t st);
/* SKFR AIM pre-selection (csrc/skfr.cu) on padded device genotypes; clusters_out: I, aims_out:
 * up to aims_capacity sorted SNP indices (n_aims: how many there are) */
cudaError_t skfr_run(const uint8_t *bed, int64_t pitch, int64_t I, int64_t J, int K, int64_t sparsity, int local,
                     int max_iter, int tries, uint64_t seed, cudaStream_t st, int32_t *clusters_out, int32_t *aims_out,
                     int64_t aims_capacity, int64_t *n_aims, double *objective_out, int32_t *iters_out);
/* fixed-order FP64 sum of n doubles into *dst (one block) */
cudaError_t launch_sum_doubles(const double *src, int64_t n, double *dst, cudaStream_t st);
cudaError_t launch_emq_finalize(int64_t I, int K, int64_t J, int S, const double *parts,
                                const double *q, double *q_next, int sms, cudaStream_t st, int E = 0, int off = 0);
cudaError_t launch_emp_finalize(int64_t J, int K, int S, const double *parts, const double *p,
                                double *p_next, int sms, cudaStream_t st);
cudaError_t launch_expand_hess(int64_t nprob, int K, int S, const double *parts, double *XtX,
                               double *Xtz, int sms, cudaStream_t st);
cudaError_t launch_decode_counts(const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                                 unsigned long long *miss_snp, unsigned long long *miss_ind,
                                 int sms, cudaStream_t st);

/* mixed-precision sweeps on tensor cores (sweeps_mixed.cu) */
cudaError_t prepare_mixed(int K);
/* The mixed-form plans pick their slice count for whole waves of resident CTAs, at most smax
 * slices (the partial-sum buffers of a handle are sized for its first plans). */
SweepPlan plan_sweep_q_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax = INT64_MAX);
/* The mixed Q sweep first builds its per-chunk P packages in pkg (sweep_q_mixed_pkg_bytes). */
cudaError_t launch_sweep_q_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                 const double *p, const SweepPlan &pl, double *out, int *err, uint8_t *pkg,
                                 cudaStream_t st);
size_t sweep_q_mixed_pkg_bytes(int K, int64_t J);

SweepPlan plan_sweep_p_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax = INT64_MAX);
/* The mixed P sweep first builds its per-chunk Q packages in pkg (sweep_p_mixed_pkg_bytes).
 * mode 0: gradient / Hessian rows (T + K); mode 1: the EM P-step's two sums (2K, k_emp_finalize). */
cudaError_t launch_sweep_p_mixed(int K, int mode, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch,
                                 const double *q, const double *p, const SweepPlan &pl, double *out, int *err,
                                 uint8_t *pkg, cudaStream_t st);
size_t sweep_p_mixed_pkg_bytes(int K, int64_t I);
/* The mixed log-likelihood first builds its per-chunk Q limb packages in pkg (this many bytes). */
size_t loglik_mixed_pkg_bytes(int K, int64_t I);
/* one CTA whose bounded wait on an mbarrier nothing completes runs out and sets *err */
cudaError_t launch_wait_probe(int *err, uint32_t polls, cudaStream_t st);
SweepPlan plan_loglik_mixed(int K, int64_t I, int64_t J, int sms, int64_t smax = INT64_MAX);
/* err and pkg are accepted for symmetry with the sweeps; the log-likelihood stays on the CUDA cores. */
cudaError_t launch_loglik_mixed(int K, const uint8_t *bed, int64_t I, int64_t J, int64_t pitch, const double *q,
                                const double *p, const SweepPlan &pl, double *partial, double *out, int *err,
                                uint8_t *pkg, cudaStream_t st);

cudaError_t launch_mask_tail(uint8_t *bed, int64_t I, int64_t J, int64_t pitch, int sms, cudaStream_t st);

/* batched QP + projection (qp_batch.cu) */
cudaError_t prepare_qp(int K);
cudaError_t launch_qp(int K, bool simplex, int64_t nprob, const double *parts, int S,
                      const double *x, double *x_next, int32_t *status, int32_t *fail_count,
                      const double *vt, int mu_mode, int damp_retry, cudaStream_t st);

/* quasi-Newton (qn.cu) */
struct QNPlan { int blocks = 1; };
QNPlan plan_qn(int64_t n, int sms);
cudaError_t launch_qn(int Q, int64_t I, int64_t J, int K, const double *x0, const double *x1,
                      const double *x2, double *U, double *V, double *x_tmp, double *partial,
                      const QNPlan &pl, DevScalars *sc, int sms, cudaStream_t st);
cudaError_t launch_lbqn(int Q, int64_t I, int64_t J, int K, const double *x0, const double *x1,
                        const double *x2, double *U, double *V, double *x_tmp, double *partial,
                        const QNPlan &pl, DevScalars *sc, int sms, cudaStream_t st);
cudaError_t launch_iter_begin(DevScalars *sc, cudaStream_t st);
cudaError_t launch_accept(int64_t n, const double *x_tmp, const double *x_next2, double *x,
                          DevScalars *sc, int sms, cudaStream_t st);
cudaError_t launch_copy(int64_t n, const double *src, double *dst, int sms, cudaStream_t st);
