/*
 * admix_capi.cu -- the C ABI of libadmix: device-resident state of one cohort and the
 * orchestration of the reference's GPU-facing calls.
 *
 * The reference keeps Q/P on the host and copies them to the device around every sweep
 * (algorithms_inner.jl:192-194, 268-270; algorithms_outer.jl:28-33, 119-123, 144-148).
 * Here the four iterates x, x_next, x_next2, x_tmp (structs.jl:16-19), the secant matrices
 * U, V (structs.jl:175-178), the sweep accumulators and the log-likelihood bookkeeping all
 * stay in HBM; a quasi-Newton iteration is one captured CUDA graph and returns a 64-byte
 * record to the host.
 */
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <vector>
#include "../../include/admix.h"
#include "common.cuh"
#include "kernels.h"

struct admix_ctx {
    int64_t I = 0, J = 0, Ib = 0;
    int64_t pitch = 0;               /* column stride of the device genotypes: Ib rounded up to 16 */
    int K = 0, Q = 0;
    uint32_t flags = 0;
    int fix = 0;                     /* bit 0: fix_q, bit 1: fix_p (admixture_qn!'s keywords) */
    int qn_mode = ADMIX_QN_ZAL;      /* admixture_qn!'s mode keyword: :ZAL or :LBQN */
    int dev = 0, sms = 148;
    cudaStream_t st = nullptr;
    uint8_t *bed = nullptr;
    bool owns_bed = true;            /* false for batch members: the batch owns the genotypes */
    /* out-of-core: the packed genotypes stay in the caller's (page-locked) host memory and every
     * pass streams SNP blocks of blk columns through two device buffers */
    bool streamed = false;
    const uint8_t *host_bed = nullptr;
    bool host_registered = false;
    int64_t blk = 0;
    int nblk = 1;
    uint8_t *sbuf[2] = {nullptr, nullptr};
    cudaStream_t cst = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_copied[2] = {nullptr, nullptr}, ev_freed[2] = {nullptr, nullptr};
    double *ll_blk = nullptr;
    double *xbuf = nullptr;          /* 4 * K(I+J): x, x_next, x_next2, x_tmp */
    double *x[4] = {nullptr, nullptr, nullptr, nullptr};
    double *parts_q = nullptr, *parts_p = nullptr;
    double *U = nullptr, *V = nullptr, *vt = nullptr;
    int32_t *status_q = nullptr, *status_p = nullptr;
    uint8_t *pkg = nullptr;          /* mixed sweeps: per-chunk packages of the fixed block */
    double *mu = nullptr;            /* ADMIX_FLAG_MEAN_IMPUTE: the SNP means g.mu (J) */
    double *ll_partial = nullptr, *qn_partial = nullptr;
    DevScalars *sc = nullptr;
    DevScalars *sc_host = nullptr;   /* pinned mirror */
    int32_t *iter_host = nullptr;    /* pinned */
    unsigned long long *counts = nullptr;
    LoglikPlan llp;
    SweepPlan sq, sp, sqm, spm, llm; /* *m: mixed-precision Q sweep, P sweep, loglik */
    int64_t cap_sqm = 1, cap_spm = 1, cap_llm = 1;   /* slice counts the partial buffers hold */
    QNPlan qnp;
    size_t bytes = 0;
    cudaGraphExec_t iter_graph = nullptr;
    cudaGraph_t iter_graph_def = nullptr;   /* the captured iteration (a batch embeds it) */
    char err[512] = {0};
};

static thread_local char g_err[512];

static int fail(admix_ctx *h, int code, const char *fmt, ...)
{
    char *dst = h ? h->err : g_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define CK(h, call)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail((h), ADMIX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

static bool valid_which(int w) { return w >= 0 && w < 4; }
static double *Qof(admix_ctx *h, int w) { return h->x[w]; }
static double *Pof(admix_ctx *h, int w) { return h->x[w] + (size_t)h->K * h->I; }

/* V' of svd(ones(1,K), full=true) (structs.jl:180) as LAPACK builds it: one Householder
 * reflector H = I - tau v v' from dlarfg on ones(K), generated by dorgl2. */
static void vt_ones(int K, double *vt)
{
    for (int a = 0; a < K * K; ++a) vt[a] = 0.0;
    if (K == 1) { vt[0] = 1.0; return; }
    const double alpha = 1.0, xnorm = sqrt((double)(K - 1));
    const double w = fmax(fabs(alpha), fabs(xnorm)), z = fmin(fabs(alpha), fabs(xnorm));
    const double nrm = w * sqrt(1.0 + (z / w) * (z / w));
    const double beta = -copysign(nrm, alpha);
    const double tau = (beta - alpha) / beta;
    const double vs = 1.0 / (alpha - beta);
    vt[0] = 1.0 - tau;
    for (int c = 1; c < K; ++c) vt[K * c] = -tau * vs;
    for (int r = 1; r < K; ++r)
        for (int c = 0; c < K; ++c) {
            const double vc = (c == 0) ? 1.0 : vs;
            vt[r + K * c] = ((r == c) ? 1.0 : 0.0) + vs * (-tau * vc);
        }
}

template <typename T>
static int dalloc(admix_ctx *h, T **p, size_t count)
{
    const size_t b = sizeof(T) * (count ? count : 1);
    cudaError_t e = cudaMalloc((void **)p, b);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(h, ADMIX_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", b, cudaGetErrorString(e));
    }
    h->bytes += b;
    return ADMIX_OK;
}

static void release(admix_ctx *h)
{
    if (!h) return;
    if (h->iter_graph) cudaGraphExecDestroy(h->iter_graph);
    if (h->iter_graph_def) cudaGraphDestroy(h->iter_graph_def);
    if (h->bed && h->owns_bed) cudaFree(h->bed);
    for (int b = 0; b < 2; ++b) {
        if (h->sbuf[b]) cudaFree(h->sbuf[b]);
        if (h->ev_copied[b]) cudaEventDestroy(h->ev_copied[b]);
        if (h->ev_freed[b]) cudaEventDestroy(h->ev_freed[b]);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ll_blk) cudaFree(h->ll_blk);
    if (h->cst) { cudaStreamSynchronize(h->cst); cudaStreamDestroy(h->cst); }
    if (h->host_registered) cudaHostUnregister((void *)h->host_bed);
    void *dps[] = {h->pkg, h->xbuf, h->parts_q, h->parts_p, h->U, h->V, h->vt, h->status_q,
                   h->status_p, h->ll_partial, h->qn_partial, h->sc, h->counts, h->mu};
    for (void *p : dps)
        if (p) cudaFree(p);
    if (h->sc_host) cudaFreeHost(h->sc_host);
    if (h->iter_host) cudaFreeHost(h->iter_host);
    if (h->st) cudaStreamDestroy(h->st);
}

extern "C" {

const char *admix_last_error(const admix_ctx *h) { return h ? h->err : g_err; }

/* Shared by admix_create (host genotypes) and admix_create_device (device genotypes at
 * src_pitch bytes per column). */
/* Copy packed genotypes (Ib bytes per column at src_pitch) into dst at a 16-byte column pitch,
 * padding bytes and the padding bits of each column's last byte set to the missing code 01
 * (never read by the reference's loops). */
static cudaError_t upload_genotypes(uint8_t *dst, int64_t pitch, const uint8_t *src, int64_t src_pitch, int64_t I,
                                    int64_t J, bool on_device, int sms, cudaStream_t st)
{
    const int64_t Ib = (I + 3) / 4;
    cudaError_t e = cudaMemsetAsync(dst, 0x55, (size_t)pitch * J + 64, st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dst, (size_t)pitch, src, (size_t)src_pitch, (size_t)Ib, (size_t)J,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = launch_mask_tail(dst, I, J, pitch, sms, st);
    return e;
}

static int create_common(int64_t I, int64_t J, int32_t K, int32_t Q, const uint8_t *bed, bool on_device,
                         int64_t src_pitch, uint32_t flags, admix_ctx **out, uint8_t *shared_bed = nullptr,
                         int64_t stream_blk = 0)
{
    if (!out) return fail(nullptr, ADMIX_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (I < 1 || J < 1) return fail(nullptr, ADMIX_ERR_ARG, "I and J must be >= 1 (I=%lld, J=%lld)", (long long)I, (long long)J);
    if (K < 1 || K > ADMIX_MAX_K) return fail(nullptr, ADMIX_ERR_UNSUPPORTED, "K=%d outside [1, %d]", K, ADMIX_MAX_K);
    if (Q < 1 || Q > ADMIX_MAX_Q) return fail(nullptr, ADMIX_ERR_UNSUPPORTED, "Q=%d outside [1, %d]", Q, ADMIX_MAX_Q);
    if (!bed) return fail(nullptr, ADMIX_ERR_ARG, "bed is NULL");
    if (flags & ~(ADMIX_FLAG_MU_GERSHGORIN | ADMIX_FLAG_MIXED | ADMIX_FLAG_MEAN_IMPUTE))
        return fail(nullptr, ADMIX_ERR_ARG, "unknown flags 0x%x", flags);
    if ((flags & ADMIX_FLAG_MEAN_IMPUTE) && ((flags & ADMIX_FLAG_MIXED) || stream_blk > 0))
        return fail(nullptr, ADMIX_ERR_UNSUPPORTED, "the mean-imputed loops run in the FP64 form of a device-resident "
                    "handle only (not with ADMIX_FLAG_MIXED or a streamed handle)");
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0)
        return fail(nullptr, ADMIX_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(ce));

    admix_ctx *h = new admix_ctx();
    h->I = I; h->J = J; h->K = K; h->Q = Q; h->flags = flags;
    h->Ib = (I + 3) / 4;
    h->pitch = (h->Ib + 15) / 16 * 16;
    int rc;
#define TRY(x) do { rc = (x); if (rc != ADMIX_OK) { strncpy(g_err, h->err, sizeof(g_err) - 1); release(h); delete h; return rc; } } while (0)
#define TRYC(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { fail(nullptr, ADMIX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); release(h); delete h; return ADMIX_ERR_CUDA; } } while (0)
    TRYC(cudaGetDevice(&h->dev));
    TRYC(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->dev));
    TRYC(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    TRYC(prepare_sweeps(K));
    TRYC(prepare_qp(K));
    if (flags & ADMIX_FLAG_MIXED) TRYC(prepare_mixed(K));

    const int64_t nx = (int64_t)K * (I + J);
    const int T = K * (K + 1) / 2, E = T + K;
    h->llp = plan_loglik(I, J, h->sms);
    h->sq = plan_sweep_q(K, I, J, h->sms);
    h->sp = plan_sweep_p(K, I, J, h->sms);
    h->sqm = plan_sweep_q_mixed(K, I, J, h->sms);
    h->spm = plan_sweep_p_mixed(K, I, J, h->sms);
    h->llm = plan_loglik_mixed(K, I, J, h->sms);
    h->qnp = plan_qn(nx, h->sms);
    h->cap_sqm = h->sqm.S;
    h->cap_spm = h->spm.S;
    h->cap_llm = h->llm.S;

    if (stream_blk > 0) {
        h->streamed = true;
        h->host_bed = bed;
        h->blk = stream_blk;
        h->nblk = (int)((J + stream_blk - 1) / stream_blk);
        for (int b = 0; b < 2; ++b) {
            TRY(dalloc(h, &h->sbuf[b], (size_t)h->pitch * stream_blk + 64));
            TRYC(cudaMemsetAsync(h->sbuf[b], 0x55, (size_t)h->pitch * stream_blk + 64, h->st));
            TRYC(cudaEventCreateWithFlags(&h->ev_copied[b], cudaEventDisableTiming));
            TRYC(cudaEventCreateWithFlags(&h->ev_freed[b], cudaEventDisableTiming));
        }
        TRYC(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
        TRYC(cudaStreamCreateWithFlags(&h->cst, cudaStreamNonBlocking));
        TRY(dalloc(h, &h->ll_blk, (size_t)h->nblk));
        cudaError_t re = cudaHostRegister((void *)bed, (size_t)h->Ib * J, cudaHostRegisterDefault);
        if (re == cudaSuccess) h->host_registered = true;
        else if (re == cudaErrorHostMemoryAlreadyRegistered) cudaGetLastError();   /* already page-locked */
        else TRYC(re);
    } else if (shared_bed) {
        h->bed = shared_bed;
        h->owns_bed = false;
    } else {
        TRY(dalloc(h, &h->bed, (size_t)h->pitch * J + 64));
    }
    TRY(dalloc(h, &h->xbuf, (size_t)4 * nx));
    for (int w = 0; w < 4; ++w) h->x[w] = h->xbuf + (size_t)w * nx;
    TRY(dalloc(h, &h->parts_q, (size_t)std::max(std::max(h->sq.S, (flags & ADMIX_FLAG_MIXED) ? h->sqm.S : 1),
                                                  h->nblk) * I * E));
    TRY(dalloc(h, &h->parts_p, (size_t)std::max(h->sp.S, (flags & ADMIX_FLAG_MIXED) ? h->spm.S : 1) * J * E));
    TRY(dalloc(h, &h->U, (size_t)nx * Q));
    TRY(dalloc(h, &h->V, (size_t)nx * Q));
    TRY(dalloc(h, &h->vt, (size_t)K * K));
    TRY(dalloc(h, &h->status_q, (size_t)I));
    if (flags & ADMIX_FLAG_MIXED)
        TRY(dalloc(h, &h->pkg, std::max({sweep_q_mixed_pkg_bytes(K, J), sweep_p_mixed_pkg_bytes(K, I),
                                          loglik_mixed_pkg_bytes(K, I)})));
    TRY(dalloc(h, &h->status_p, (size_t)J));
    /* per-CTA log-likelihood partials: the resident plans, and for a streamed handle the plans of
     * a full block and of the last block (the mixed plan's count can grow as its SNP range shrinks) */
    auto ll_parts = [&](int64_t nj) {
        const LoglikPlan a = plan_loglik(I, nj, h->sms);
        const SweepPlan b = plan_loglik_mixed(K, I, nj, h->sms);
        return std::max((size_t)a.gx * a.gy, (size_t)b.gx * b.S);
    };
    size_t n_ll = std::max((size_t)h->llp.gx * h->llp.gy, (size_t)h->llm.gx * h->llm.S);
    if (h->streamed)
        n_ll = std::max(n_ll, std::max(ll_parts(std::min<int64_t>(h->blk, J)), ll_parts(J - (int64_t)(h->nblk - 1) * h->blk)));
    TRY(dalloc(h, &h->ll_partial, n_ll));
    TRY(dalloc(h, &h->qn_partial, (size_t)h->qnp.blocks * (Q * Q + Q)));
    TRY(dalloc(h, &h->sc, 1));
    TRY(dalloc(h, &h->counts, (size_t)(I + J)));
    TRYC(cudaMallocHost((void **)&h->sc_host, sizeof(DevScalars)));
    TRYC(cudaMallocHost((void **)&h->iter_host, sizeof(int32_t)));

    if (!shared_bed && !h->streamed) TRYC(upload_genotypes(h->bed, h->pitch, bed, src_pitch, I, J, on_device, h->sms, h->st));
    if (flags & ADMIX_FLAG_MEAN_IMPUTE) {
        TRY(dalloc(h, &h->mu, (size_t)J));
        TRYC(launch_snp_means(h->bed, J, h->pitch, h->mu, h->st));
    }
    TRYC(cudaMemsetAsync(h->xbuf, 0, sizeof(double) * 4 * nx, h->st));
    TRYC(cudaMemsetAsync(h->U, 0, sizeof(double) * nx * Q, h->st));
    TRYC(cudaMemsetAsync(h->V, 0, sizeof(double) * nx * Q, h->st));
    std::vector<double> vt((size_t)K * K);
    vt_ones(K, vt.data());
    TRYC(cudaMemcpyAsync(h->vt, vt.data(), sizeof(double) * K * K, cudaMemcpyHostToDevice, h->st));
    DevScalars z;
    memset(&z, 0, sizeof(z));
    z.ll_new = NAN; z.ll_prev = NAN;
    TRYC(cudaMemcpyAsync(h->sc, &z, sizeof(z), cudaMemcpyHostToDevice, h->st));
    TRYC(cudaStreamSynchronize(h->st));
#undef TRY
#undef TRYC
    *out = h;
    return ADMIX_OK;
}

int admix_create(int64_t I, int64_t J, int32_t K, int32_t Q, const uint8_t *bed, uint32_t flags,
                 admix_ctx **out)
{
    return create_common(I, J, K, Q, bed, false, (I + 3) / 4, flags, out);
}

int admix_create_device(int64_t I, int64_t J, int32_t K, int32_t Q, const uint8_t *d_bed, int64_t src_pitch,
                        uint32_t flags, admix_ctx **out)
{
    if (src_pitch < (I + 3) / 4) return fail(nullptr, ADMIX_ERR_ARG, "src_pitch %lld is below ceil(I/4) = %lld",
                                             (long long)src_pitch, (long long)((I + 3) / 4));
    cudaPointerAttributes at;
    if (d_bed && (cudaPointerGetAttributes(&at, d_bed) != cudaSuccess || at.type != cudaMemoryTypeDevice)) {
        cudaGetLastError();
        return fail(nullptr, ADMIX_ERR_ARG, "d_bed is not device memory");
    }
    return create_common(I, J, K, Q, d_bed, true, src_pitch, flags, out);
}

int admix_create_streamed(int64_t I, int64_t J, int32_t K, int32_t Q, const uint8_t *bed, int64_t block_snps,
                          uint32_t flags, admix_ctx **out)
{
    if (block_snps < 32 || block_snps % 32 != 0)
        return fail(nullptr, ADMIX_ERR_ARG, "block_snps must be a positive multiple of 32 (got %lld)", (long long)block_snps);
    return create_common(I, J, K, Q, bed, false, (I + 3) / 4, flags, out, nullptr, std::min<int64_t>(block_snps, (J + 31) / 32 * 32));
}

int admix_destroy(admix_ctx *h)
{
    if (!h) return ADMIX_OK;
    if (h->st) cudaStreamSynchronize(h->st);
    release(h);
    delete h;
    return ADMIX_OK;
}

int admix_device_bytes(const admix_ctx *h, int64_t *bytes)
{
    if (!h || !bytes) return ADMIX_ERR_ARG;
    *bytes = (int64_t)h->bytes;
    return ADMIX_OK;
}

int admix_set_x(admix_ctx *h, int32_t which, const double *q, const double *p)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (!valid_which(which)) return fail(h, ADMIX_ERR_ARG, "invalid buffer selector %d", which);
    if (q) CK(h, cudaMemcpyAsync(Qof(h, which), q, sizeof(double) * h->K * h->I, cudaMemcpyHostToDevice, h->st));
    if (p) CK(h, cudaMemcpyAsync(Pof(h, which), p, sizeof(double) * h->K * h->J, cudaMemcpyHostToDevice, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

int admix_get_x(admix_ctx *h, int32_t which, double *q, double *p)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (!valid_which(which)) return fail(h, ADMIX_ERR_ARG, "invalid buffer selector %d", which);
    if (q) CK(h, cudaMemcpyAsync(q, Qof(h, which), sizeof(double) * h->K * h->I, cudaMemcpyDeviceToHost, h->st));
    if (p) CK(h, cudaMemcpyAsync(p, Pof(h, which), sizeof(double) * h->K * h->J, cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

int admix_set_ll(admix_ctx *h, double ll_new)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    CK(h, cudaMemcpyAsync(&h->sc->ll_new, &ll_new, sizeof(double), cudaMemcpyHostToDevice, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

int admix_get_ll(admix_ctx *h, double *ll_new)
{
    if (!h || !ll_new) return fail(h, ADMIX_ERR_ARG, "NULL argument");
    CK(h, cudaMemcpyAsync(ll_new, &h->sc->ll_new, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

} /* extern "C" */

/* ---- stream-ordered building blocks (no synchronisation) ---- */

/* Run fn(bed, j0, nj, b) for every SNP block.  In-HBM handles: one call over all SNPs.  Streamed
 * handles: block b is copied (2D, into the 16-byte pitch, padding coded missing) from page-locked
 * host memory into device buffer b & 1 on the copy stream while block b-1 computes; events order
 * the reuse of each buffer, so the whole pass can be captured into a graph. */
template <class F>
static cudaError_t for_blocks(admix_ctx *h, F fn)
{
    if (!h->streamed) return fn((const uint8_t *)h->bed, (int64_t)0, h->J, 0);
    cudaError_t e = cudaEventRecord(h->ev_fork, h->st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->cst, h->ev_fork, 0);
    for (int b = 0; b < h->nblk && e == cudaSuccess; ++b) {
        const int s = b & 1;
        const int64_t j0 = (int64_t)b * h->blk, nj = std::min(h->blk, h->J - j0);
        if (b >= 2) e = cudaStreamWaitEvent(h->cst, h->ev_freed[s], 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(h->sbuf[s], (size_t)h->pitch, h->host_bed + (size_t)j0 * h->Ib, (size_t)h->Ib,
                                  (size_t)h->Ib, (size_t)nj, cudaMemcpyHostToDevice, h->cst);
        if (e == cudaSuccess) e = launch_mask_tail(h->sbuf[s], h->I, nj, h->pitch, h->sms, h->cst);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_copied[s], h->cst);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(h->st, h->ev_copied[s], 0);
        if (e == cudaSuccess) e = fn((const uint8_t *)h->sbuf[s], j0, nj, b);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_freed[s], h->st);
    }
    return e;
}

/* plans of one streamed block: one slice, so block b's Q-side partials are slice b and its
 * P-side rows land at their global SNP index */
static SweepPlan block_plan(SweepPlan pl, int64_t len)
{
    pl.S = 1;
    pl.slice = len;
    return pl;
}

/* number of Q-side partial slices the QP / EM finaliser must add */
static int q_slices(const admix_ctx *h)
{
    if (h->streamed) return h->nblk;
    return (h->flags & ADMIX_FLAG_MIXED) ? h->sqm.S : h->sq.S;
}

/* FP64 log-likelihood (the verifier); fast = 1 selects the FP32-cell form in mixed mode */
static cudaError_t enq_loglik(admix_ctx *h, int which, double *dst, bool fast = false)
{
    const bool mx = fast && (h->flags & ADMIX_FLAG_MIXED);
    auto one = [&](const uint8_t *bed, int64_t j0, int64_t nj, int b) -> cudaError_t {
        double *o = h->streamed ? h->ll_blk + b : dst;
        const double *P = Pof(h, which) + (size_t)h->K * j0;
        if (mx) {
            const SweepPlan pl = h->streamed ? plan_loglik_mixed(h->K, h->I, nj, h->sms) : h->llm;
            return launch_loglik_mixed(h->K, bed, h->I, nj, h->pitch, Qof(h, which), P, pl, h->ll_partial, o,
                                       &h->sc->tc_err, h->pkg, h->st);
        }
        const LoglikPlan pl = h->streamed ? plan_loglik(h->I, nj, h->sms) : h->llp;
        return launch_loglik_f64(h->K, bed, h->I, nj, h->pitch, Qof(h, which), P, pl, h->ll_partial, o, h->st, h->mu);
    };
    cudaError_t e = for_blocks(h, one);
    if (e == cudaSuccess && h->streamed) e = launch_sum_doubles(h->ll_blk, h->nblk, dst, h->st);
    return e;
}

/* Q-side gradient / Hessian sweep (mode 0) or EM sums (mode 1, FP64) into parts_q; returns the
 * number of slices written. */
static cudaError_t enq_sweep_q_mode(admix_ctx *h, int mode, int wq, int wp, int *S)
{
    const bool mx = mode == 0 && (h->flags & ADMIX_FLAG_MIXED);
    /* entries per individual: T + K (gradient / Hessian) or K (EM sums) */
    const size_t slice = (size_t)h->I * (mode == 0 ? h->K * (h->K + 1) / 2 + h->K : h->K);
    *S = q_slices(h);
    return for_blocks(h, [&](const uint8_t *bed, int64_t j0, int64_t nj, int b) -> cudaError_t {
        const double *P = Pof(h, wp) + (size_t)h->K * j0;
        double *out = h->parts_q + (size_t)b * slice;
        if (mx) {
            const SweepPlan pl = h->streamed ? block_plan(h->sqm, nj) : h->sqm;
            return launch_sweep_q_mixed(h->K, bed, h->I, nj, h->pitch, Qof(h, wq), P, pl, out, &h->sc->tc_err,
                                        h->pkg, h->st);
        }
        const SweepPlan pl = h->streamed ? block_plan(h->sq, nj) : h->sq;
        return launch_sweep_q_f64(h->K, mode, bed, h->I, nj, h->pitch, Qof(h, wq), P, pl, out, h->st, h->mu);
    });
}

/* P-side gradient / Hessian sweep (mode 0) or EM sums (mode 1, FP64) into parts_p */
/* mode 0: gradient / Hessian (tensor-core pipeline in the mixed form); 1: the EM sums in FP64;
 * 2: the EM sums on the mixed pipeline (mixed handles only) */
static cudaError_t enq_sweep_p_mode(admix_ctx *h, int mode, int wq, int wp, int *S)
{
    const bool mx = (mode == 0 && (h->flags & ADMIX_FLAG_MIXED)) || mode == 2;
    /* entries per SNP: T + K (gradient / Hessian) or 2K (EM sums) */
    const size_t row = (size_t)(mode == 0 ? h->K * (h->K + 1) / 2 + h->K : 2 * h->K);
    *S = h->streamed ? 1 : (mx ? h->spm.S : h->sp.S);
    return for_blocks(h, [&](const uint8_t *bed, int64_t j0, int64_t nj, int b) -> cudaError_t {
        (void)b;
        const double *P = Pof(h, wp) + (size_t)h->K * j0;
        double *out = h->parts_p + (size_t)j0 * row;
        if (mx) {
            const SweepPlan pl = h->streamed ? block_plan(plan_sweep_p_mixed(h->K, h->I, nj, h->sms), (h->I + 31) / 32 * 32)
                                             : h->spm;
            return launch_sweep_p_mixed(h->K, mode == 2 ? 1 : 0, bed, h->I, nj, h->pitch, Qof(h, wq), P, pl, out,
                                        &h->sc->tc_err, h->pkg, h->st);
        }
        const SweepPlan pl = h->streamed ? block_plan(plan_sweep_p(h->K, h->I, nj, h->sms), (h->I + 3) / 4 * 4) : h->sp;
        return launch_sweep_p_f64(h->K, mode, bed, h->I, nj, h->pitch, Qof(h, wq), P, pl, out, h->st, h->mu);
    });
}

static cudaError_t enq_sweep_q(admix_ctx *h, int wq, int wp, int *S) { return enq_sweep_q_mode(h, 0, wq, wp, S); }
static cudaError_t enq_sweep_p(admix_ctx *h, int wq, int wp, int *S) { return enq_sweep_p_mode(h, 0, wq, wp, S); }

/* update_q!: q_out = project_q(q + QP(H_q, -Xtz_q)) */
static cudaError_t enq_update_q(admix_ctx *h, int update2)
{
    const int wq = update2 ? ADMIX_X_NEXT : ADMIX_X;
    const int wp = update2 ? ADMIX_X_NEXT : ADMIX_X;
    const int wo = update2 ? ADMIX_X_NEXT2 : ADMIX_X_NEXT;
    int S = 1;
    cudaError_t e = enq_sweep_q(h, wq, wp, &S);
    if (e != cudaSuccess) return e;
    return launch_qp(h->K, true, h->I, h->parts_q, S, Qof(h, wq), Qof(h, wo), h->status_q,
                     &h->sc->fail_q, h->vt, (h->flags & ADMIX_FLAG_MU_GERSHGORIN) ? 1 : 0,
                     (h->flags & ADMIX_FLAG_MIXED) ? 1 : 0, h->st);
}

/* update_p!: p_out = project_p(p + QP(H_p, -Xtz_p)), with q = q_next (update2 = 0) or q_next2 */
static cudaError_t enq_update_p(admix_ctx *h, int update2)
{
    const int wq = update2 ? ADMIX_X_NEXT2 : ADMIX_X_NEXT;
    const int wp = update2 ? ADMIX_X_NEXT : ADMIX_X;
    const int wo = update2 ? ADMIX_X_NEXT2 : ADMIX_X_NEXT;
    int S = 1;
    cudaError_t e = enq_sweep_p(h, wq, wp, &S);
    if (e != cudaSuccess) return e;
    return launch_qp(h->K, false, h->J, h->parts_p, S, Pof(h, wp), Pof(h, wo), h->status_p,
                     &h->sc->fail_p, h->vt, 0, (h->flags & ADMIX_FLAG_MIXED) ? 1 : 0, h->st);
}

static cudaError_t enq_em(admix_ctx *h)
{
    /* em_q! then em_p! (mode :base, both from (q, p)), then p, q <- next (algorithms_outer.jl:23-30).
     * The EM Q-step's sums are the Q-side gradient, so the mixed form takes them from its
     * tensor-core gradient / Hessian sweep; its P-step sums come from the EM mode of the mixed
     * P pipeline (FP32 cells, FP64 across chunks). */
    int Sq = 1, Sp = 1;
    cudaError_t e;
    const bool mixed = (h->flags & ADMIX_FLAG_MIXED) != 0;
    if (mixed) {
        const int T = h->K * (h->K + 1) / 2;
        e = enq_sweep_q_mode(h, 0, ADMIX_X, ADMIX_X, &Sq);
        if (e == cudaSuccess) e = launch_emq_finalize(h->I, h->K, h->J, Sq, h->parts_q, Qof(h, ADMIX_X), Qof(h, ADMIX_X_NEXT), h->sms, h->st, T + h->K, T);
    } else {
        e = enq_sweep_q_mode(h, 1, ADMIX_X, ADMIX_X, &Sq);
        if (e == cudaSuccess) e = launch_emq_finalize(h->I, h->K, h->J, h->streamed ? h->nblk : h->sq.S, h->parts_q, Qof(h, ADMIX_X), Qof(h, ADMIX_X_NEXT), h->sms, h->st);
    }
    if (e == cudaSuccess) e = enq_sweep_p_mode(h, mixed ? 2 : 1, ADMIX_X, ADMIX_X, &Sp);
    if (e == cudaSuccess) e = launch_emp_finalize(h->J, h->K, Sp, h->parts_p, Pof(h, ADMIX_X), Pof(h, ADMIX_X_NEXT), h->sms, h->st);
    return e;
}

/* one admixture_qn! iteration, stream-ordered; sc->iter must already hold i */
static cudaError_t enq_iteration(admix_ctx *h)
{
    const int64_t nx = (int64_t)h->K * (h->I + h->J);
    /* fix_q / fix_p (algorithms_outer.jl:98-116): the fixed block is copied, not updated */
    const size_t nq = sizeof(double) * (size_t)h->K * h->I, np = sizeof(double) * (size_t)h->K * h->J;
    auto copy_q = [&](int dst) { return cudaMemcpyAsync(Qof(h, dst), Qof(h, ADMIX_X), nq, cudaMemcpyDeviceToDevice, h->st); };
    auto copy_p = [&](int dst) { return cudaMemcpyAsync(Pof(h, dst), Pof(h, ADMIX_X), np, cudaMemcpyDeviceToDevice, h->st); };
    cudaError_t e = launch_iter_begin(h->sc, h->st);
    if (e == cudaSuccess) e = (h->fix & 1) ? copy_q(ADMIX_X_NEXT) : enq_update_q(h, 0);
    if (e == cudaSuccess) e = (h->fix & 2) ? copy_p(ADMIX_X_NEXT) : enq_update_p(h, 0);
    if (e == cudaSuccess) e = (h->fix & 1) ? copy_q(ADMIX_X_NEXT2) : enq_update_q(h, 1);
    if (e == cudaSuccess) e = (h->fix & 2) ? copy_p(ADMIX_X_NEXT2) : enq_update_p(h, 1);
    if (e == cudaSuccess) e = enq_loglik(h, ADMIX_X_NEXT2, &h->sc->ll_basic, true);
    if (e == cudaSuccess)
        e = (h->qn_mode == ADMIX_QN_LBQN ? launch_lbqn : launch_qn)(
            h->Q, h->I, h->J, h->K, h->x[ADMIX_X], h->x[ADMIX_X_NEXT], h->x[ADMIX_X_NEXT2], h->U, h->V,
            h->x[ADMIX_X_TMP], h->qn_partial, h->qnp, h->sc, h->sms, h->st);
    if (e == cudaSuccess) e = enq_loglik(h, ADMIX_X_TMP, &h->sc->ll_qn, true);
    if (e == cudaSuccess) e = launch_accept(nx, h->x[ADMIX_X_TMP], h->x[ADMIX_X_NEXT2], h->x[ADMIX_X], h->sc, h->sms, h->st);
    return e;
}

/* The tensor-core sweeps of the mixed form bound every pipeline wait; one that runs out sets
 * tc_err and leaves NaN in its outputs.  After the stream has drained and sc_host holds the
 * device's flag, report it as a failed call and clear it. */
static int tc_err_check(admix_ctx *h)
{
    if (!h->sc_host->tc_err) return ADMIX_OK;
    h->sc_host->tc_err = 0;
    CK(h, cudaMemsetAsync(&h->sc->tc_err, 0, sizeof(int32_t), h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return fail(h, ADMIX_ERR_CUDA, "a tensor-core pipeline wait gave up (bounded wait ran out); this call's results are invalid");
}

/* drain the stream and check the flag (mixed handles only: the FP64 kernels never wait) */
static int tc_err_sync(admix_ctx *h)
{
    if (h->flags & ADMIX_FLAG_MIXED)
        CK(h, cudaMemcpyAsync(&h->sc_host->tc_err, &h->sc->tc_err, sizeof(int32_t), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return tc_err_check(h);
}

static int read_scalars(admix_ctx *h)
{
    CK(h, cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return tc_err_check(h);
}

extern "C" {

int admix_loglik(admix_ctx *h, int32_t which, double *out)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (!valid_which(which)) return fail(h, ADMIX_ERR_ARG, "invalid buffer selector %d", which);
    if (!out) return fail(h, ADMIX_ERR_ARG, "out is NULL");
    CK(h, enq_loglik(h, which, &h->sc->ll_tmp));
    CK(h, cudaMemcpyAsync(out, &h->sc->ll_tmp, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

int admix_em_q(admix_ctx *h)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    int S = 1;
    CK(h, enq_sweep_q_mode(h, 1, ADMIX_X, ADMIX_X, &S));
    CK(h, launch_emq_finalize(h->I, h->K, h->J, h->streamed ? h->nblk : h->sq.S, h->parts_q, Qof(h, ADMIX_X), Qof(h, ADMIX_X_NEXT), h->sms, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

int admix_em_p(admix_ctx *h)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    int S = 1;
    CK(h, enq_sweep_p_mode(h, 1, ADMIX_X, ADMIX_X, &S));
    CK(h, launch_emp_finalize(h->J, h->K, h->streamed ? 1 : h->sp.S, h->parts_p, Pof(h, ADMIX_X), Pof(h, ADMIX_X_NEXT), h->sms, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

/* init_em! stream-ordered on the handle's stream (no synchronisation) */
static int enq_init_em(admix_ctx *h, int32_t iters, double *ll_hist)
{
    for (int it = 0; it < iters; ++it) {
        CK(h, enq_em(h));
        CK(h, cudaMemcpyAsync(Pof(h, ADMIX_X), Pof(h, ADMIX_X_NEXT), sizeof(double) * h->K * h->J, cudaMemcpyDeviceToDevice, h->st));
        CK(h, cudaMemcpyAsync(Qof(h, ADMIX_X), Qof(h, ADMIX_X_NEXT), sizeof(double) * h->K * h->I, cudaMemcpyDeviceToDevice, h->st));
        /* the per-iteration values are reported only; the mixed form uses its FP32-cell pass */
        if (ll_hist) {
            CK(h, enq_loglik(h, ADMIX_X, &h->sc->ll_tmp, true));
            CK(h, cudaMemcpyAsync(ll_hist + it, &h->sc->ll_tmp, sizeof(double), cudaMemcpyDeviceToHost, h->st));
        }
    }
    /* the first QN iteration's ll_prev, from the same pass as the iteration's own log-likelihoods
     * (the mixed pass in the mixed form: -1.5e-9 relative from the FP64 pass, at C5 0.05 s
     * instead of 0.58 s); the last reported value is that pass at the same point */
    if (ll_hist && iters > 0)
        CK(h, cudaMemcpyAsync(&h->sc->ll_new, &h->sc->ll_tmp, sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    else
        CK(h, enq_loglik(h, ADMIX_X, &h->sc->ll_new, true));
    return ADMIX_OK;
}

int admix_init_em(admix_ctx *h, int32_t iters, double *ll_hist)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (iters < 0) return fail(h, ADMIX_ERR_ARG, "iters must be >= 0");
    int rc = enq_init_em(h, iters, ll_hist);
    if (rc != ADMIX_OK) return rc;
    return tc_err_sync(h);
}

static int grad_hess_common(admix_ctx *h, bool qside, int32_t wq, int32_t wp, double *XtX, double *Xtz)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (!valid_which(wq) || !valid_which(wp)) return fail(h, ADMIX_ERR_ARG, "invalid buffer selector");
    const int64_t nprob = qside ? h->I : h->J;
    const int K = h->K;
    double *d_XtX = nullptr, *d_Xtz = nullptr;
    if (cudaMalloc((void **)&d_XtX, sizeof(double) * K * K * nprob) != cudaSuccess ||
        cudaMalloc((void **)&d_Xtz, sizeof(double) * K * nprob) != cudaSuccess) {
        if (d_XtX) cudaFree(d_XtX);
        return fail(h, ADMIX_ERR_NOMEM, "dump buffers: cudaMalloc failed");
    }
    cudaError_t e;
    if (qside) {
        int S = 1;
        e = enq_sweep_q(h, wq, wp, &S);
        if (e == cudaSuccess) e = launch_expand_hess(nprob, K, S, h->parts_q, d_XtX, d_Xtz, h->sms, h->st);
    } else {
        int S = 1;
        e = enq_sweep_p(h, wq, wp, &S);
        if (e == cudaSuccess) e = launch_expand_hess(nprob, K, S, h->parts_p, d_XtX, d_Xtz, h->sms, h->st);
    }
    if (e == cudaSuccess && XtX) e = cudaMemcpyAsync(XtX, d_XtX, sizeof(double) * K * K * nprob, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess && Xtz) e = cudaMemcpyAsync(Xtz, d_Xtz, sizeof(double) * K * nprob, cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    cudaFree(d_XtX);
    cudaFree(d_Xtz);
    if (e != cudaSuccess) return fail(h, ADMIX_ERR_CUDA, "grad/hess sweep failed: %s", cudaGetErrorString(e));
    return tc_err_sync(h);
}

int admix_grad_hess_q(admix_ctx *h, int32_t which_q, int32_t which_p, double *XtX, double *Xtz)
{
    return grad_hess_common(h, true, which_q, which_p, XtX, Xtz);
}

int admix_grad_hess_p(admix_ctx *h, int32_t which_q, int32_t which_p, double *XtX, double *Xtz)
{
    return grad_hess_common(h, false, which_q, which_p, XtX, Xtz);
}

int admix_skfr(admix_ctx *h, int32_t k, int64_t sparsity, int32_t mode, int32_t max_iter, int32_t tries,
               uint64_t seed, int32_t *clusters, int32_t *aims, int64_t aims_capacity, int64_t *n_aims,
               double *objective, int32_t *iterations)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (!clusters || !aims || !n_aims || !objective || !iterations) return fail(h, ADMIX_ERR_ARG, "an output pointer is NULL");
    if (k < 1 || k > 16) return fail(h, ADMIX_ERR_UNSUPPORTED, "k=%d outside [1, 16]", k);
    if (sparsity < 1) return fail(h, ADMIX_ERR_ARG, "sparsity must be >= 1 (got %lld)", (long long)sparsity);
    if (mode != ADMIX_SKFR_GLOBAL && mode != ADMIX_SKFR_LOCAL) return fail(h, ADMIX_ERR_ARG, "skfr mode can only be global (0) or local (1)");
    if (max_iter < 1 || tries < 1) return fail(h, ADMIX_ERR_ARG, "max_iter and tries must be >= 1");
    if (aims_capacity < 0) return fail(h, ADMIX_ERR_ARG, "aims_capacity < 0");
    if (h->streamed) return fail(h, ADMIX_ERR_UNSUPPORTED, "SKFR needs device-resident genotypes");
    CK(h, skfr_run(h->bed, h->pitch, h->I, h->J, k, sparsity, mode == ADMIX_SKFR_LOCAL ? 1 : 0, max_iter, tries, seed, h->st,
                   clusters, aims, aims_capacity, n_aims, objective, iterations));
    return ADMIX_OK;
}

int admix_selftest_wait_timeout(admix_ctx *h)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (!(h->flags & ADMIX_FLAG_MIXED)) return fail(h, ADMIX_ERR_STATE, "the self-test needs a mixed-form handle");
    CK(h, launch_wait_probe(&h->sc->tc_err, 1024u, h->st));
    return tc_err_sync(h);
}

int admix_update_q(admix_ctx *h, int32_t update2, int32_t *qp_status)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    CK(h, enq_update_q(h, update2 ? 1 : 0));
    if (qp_status) CK(h, cudaMemcpyAsync(qp_status, h->status_q, sizeof(int32_t) * h->I, cudaMemcpyDeviceToHost, h->st));
    return tc_err_sync(h);
}

int admix_update_p(admix_ctx *h, int32_t update2, int32_t *qp_status)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    CK(h, enq_update_p(h, update2 ? 1 : 0));
    if (qp_status) CK(h, cudaMemcpyAsync(qp_status, h->status_p, sizeof(int32_t) * h->J, cudaMemcpyDeviceToHost, h->st));
    return tc_err_sync(h);
}

static int ensure_graph(admix_ctx *h)
{
    if (h->iter_graph) return ADMIX_OK;
    cudaGraph_t g = nullptr;
    CK(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enq_iteration(h);
    cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(h, ADMIX_ERR_CUDA, "iteration capture failed: %s / %s", cudaGetErrorString(e), cudaGetErrorString(e2));
    }
    e = cudaGraphInstantiate(&h->iter_graph, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        h->iter_graph = nullptr;
        return fail(h, ADMIX_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    }
    h->iter_graph_def = g;
    return ADMIX_OK;
}

static int run_one(admix_ctx *h, int32_t iter, admix_iterinfo *out)
{
    int rc = ensure_graph(h);
    if (rc != ADMIX_OK) return rc;
    *h->iter_host = iter;
    CK(h, cudaMemcpyAsync(&h->sc->iter, h->iter_host, sizeof(int32_t), cudaMemcpyHostToDevice, h->st));
    CK(h, cudaGraphLaunch(h->iter_graph, h->st));
    rc = read_scalars(h);
    if (rc != ADMIX_OK) return rc;
    const DevScalars &s = *h->sc_host;
    if (out) {
        out->ll_prev = s.ll_prev; out->ll_basic = s.ll_basic; out->ll_qn = s.ll_qn;
        out->ll_new = s.ll_new; out->reldiff = s.reldiff; out->iter = iter;
        out->accepted_qn = s.accepted; out->qp_fail_q = s.fail_q; out->qp_fail_p = s.fail_p;
    }
    return ADMIX_OK;
}

int admix_set_fixed(admix_ctx *h, int32_t fix_q, int32_t fix_p)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    const int fix = (fix_q ? 1 : 0) | (fix_p ? 2 : 0);
    if (fix != h->fix) {
        CK(h, cudaStreamSynchronize(h->st));
        if (h->iter_graph) { cudaGraphExecDestroy(h->iter_graph); h->iter_graph = nullptr; }
        if (h->iter_graph_def) { cudaGraphDestroy(h->iter_graph_def); h->iter_graph_def = nullptr; }
        h->fix = fix;
    }
    return ADMIX_OK;
}

int admix_set_qn_mode(admix_ctx *h, int32_t mode)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (mode != ADMIX_QN_ZAL && mode != ADMIX_QN_LBQN)
        return fail(h, ADMIX_ERR_ARG, "mode %d is neither ADMIX_QN_ZAL (0) nor ADMIX_QN_LBQN (1)", (int)mode);
    if (mode != h->qn_mode) {
        CK(h, cudaStreamSynchronize(h->st));
        if (h->iter_graph) { cudaGraphExecDestroy(h->iter_graph); h->iter_graph = nullptr; }
        if (h->iter_graph_def) { cudaGraphDestroy(h->iter_graph_def); h->iter_graph_def = nullptr; }
        h->qn_mode = mode;
    }
    return ADMIX_OK;
}

int admix_qn_iteration(admix_ctx *h, int32_t iter, admix_iterinfo *out)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (iter < 1) return fail(h, ADMIX_ERR_ARG, "iteration number must be >= 1 (got %d)", iter);
    return run_one(h, iter, out);
}

int admix_run_qn(admix_ctx *h, int32_t n_iter, double rtol, int32_t iter_offset,
                 admix_iterinfo *hist, int32_t *n_done, int32_t *converged)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (iter_offset < 0) return fail(h, ADMIX_ERR_ARG, "iter_offset must be >= 0");
    int rc = read_scalars(h);
    if (rc != ADMIX_OK) return rc;
    if (isnan(h->sc_host->ll_new)) {   /* algorithms_outer.jl:76-83 (the iteration's own pass) */
        CK(h, enq_loglik(h, ADMIX_X, &h->sc->ll_new, true));
        CK(h, cudaStreamSynchronize(h->st));
    }
    int done = 0, conv = 0;
    for (int it = iter_offset + 1; it <= n_iter; ++it) {
        admix_iterinfo info;
        rc = run_one(h, it, &info);
        if (rc != ADMIX_OK) return rc;
        if (hist) hist[done] = info;
        ++done;
        if (info.reldiff < rtol) { conv = 1; break; }
    }
    if (n_done) *n_done = done;
    if (converged) *converged = conv;
    return ADMIX_OK;
}

int admix_stream(admix_ctx *h, void **stream)
{
    if (!h || !stream) return fail(h, ADMIX_ERR_ARG, "NULL argument");
    *stream = (void *)h->st;
    return ADMIX_OK;
}

int admix_time_pass(admix_ctx *h, int32_t pass, int32_t reps, double *ms_per_launch)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    if (reps < 1 || !ms_per_launch) return fail(h, ADMIX_ERR_ARG, "reps must be >= 1 and ms_per_launch non-NULL");
    if (pass < ADMIX_PASS_LOGLIK || pass > ADMIX_PASS_EM) return fail(h, ADMIX_ERR_ARG, "unknown pass %d", pass);
    const int mu = (h->flags & ADMIX_FLAG_MU_GERSHGORIN) ? 1 : 0;
    auto one = [&]() -> cudaError_t {
        switch (pass) {
        case ADMIX_PASS_LOGLIK: return enq_loglik(h, ADMIX_X, &h->sc->ll_tmp, true);
        case ADMIX_PASS_QSWEEP: { int S; return enq_sweep_q(h, ADMIX_X, ADMIX_X, &S); }
        case ADMIX_PASS_PSWEEP: { int S; return enq_sweep_p(h, ADMIX_X, ADMIX_X, &S); }
        case ADMIX_PASS_QQP: return launch_qp(h->K, true, h->I, h->parts_q, q_slices(h), Qof(h, ADMIX_X), Qof(h, ADMIX_X_TMP), h->status_q, nullptr, h->vt, mu, (h->flags & ADMIX_FLAG_MIXED) ? 1 : 0, h->st);
        case ADMIX_PASS_PQP: return launch_qp(h->K, false, h->J, h->parts_p, h->streamed ? 1 : ((h->flags & ADMIX_FLAG_MIXED) ? h->spm.S : h->sp.S), Pof(h, ADMIX_X), Pof(h, ADMIX_X_TMP), h->status_p, nullptr, h->vt, 0, (h->flags & ADMIX_FLAG_MIXED) ? 1 : 0, h->st);
        default: return enq_em(h);
        }
    };
    cudaEvent_t e0, e1;
    CK(h, cudaEventCreate(&e0));
    CK(h, cudaEventCreate(&e1));
    cudaError_t e = one();   /* warm-up launch */
    if (e == cudaSuccess) e = cudaEventRecord(e0, h->st);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = one();
    if (e == cudaSuccess) e = cudaEventRecord(e1, h->st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail(h, ADMIX_ERR_CUDA, "timing pass %d failed: %s", pass, cudaGetErrorString(e));
    *ms_per_launch = (double)ms / reps;
    return ADMIX_OK;
}

int admix_iteration_kernels(admix_ctx *h, int32_t *count)
{
    if (!h || !count) return fail(h, ADMIX_ERR_ARG, "NULL argument");
    cudaGraph_t g = nullptr;
    CK(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enq_iteration(h);
    cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(h, ADMIX_ERR_CUDA, "capture failed");
    }
    size_t n = 0;
    e = cudaGraphGetNodes(g, nullptr, &n);
    std::vector<cudaGraphNode_t> nodes(n);
    if (e == cudaSuccess && n) e = cudaGraphGetNodes(g, nodes.data(), &n);
    int32_t k = 0;
    for (size_t t = 0; t < n && e == cudaSuccess; ++t) {
        cudaGraphNodeType ty;
        if (cudaGraphNodeGetType(nodes[t], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++k;
    }
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(h, ADMIX_ERR_CUDA, "graph query failed: %s", cudaGetErrorString(e));
    *count = k;
    return ADMIX_OK;
}

int admix_decode_counts(admix_ctx *h, int64_t *miss_per_snp, int64_t *miss_per_ind)
{
    if (!h) return fail(nullptr, ADMIX_ERR_ARG, "handle is NULL");
    CK(h, cudaMemsetAsync(h->counts, 0, sizeof(unsigned long long) * (h->I + h->J), h->st));
    CK(h, for_blocks(h, [&](const uint8_t *bed, int64_t j0, int64_t nj, int b) -> cudaError_t {
        (void)b;
        return launch_decode_counts(bed, h->I, nj, h->pitch, h->counts + h->I + j0, h->counts, h->sms, h->st);
    }));
    if (miss_per_snp) CK(h, cudaMemcpyAsync(miss_per_snp, h->counts + h->I, sizeof(int64_t) * h->J, cudaMemcpyDeviceToHost, h->st));
    if (miss_per_ind) CK(h, cudaMemcpyAsync(miss_per_ind, h->counts, sizeof(int64_t) * h->I, cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

size_t admix_loglik_dev_workspace(int64_t I, int64_t J, int32_t K)
{
    (void)K;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const LoglikPlan pl = plan_loglik(I, J, sms);
    return sizeof(double) * (size_t)pl.gx * pl.gy;
}

int admix_loglik_dev(const uint8_t *d_bed, int64_t I, int64_t J, int32_t K, const double *d_q,
                     const double *d_p, double *d_out, void *d_work, size_t work_bytes, void *stream)
{
    if (!d_bed || !d_q || !d_p || !d_out || !d_work) return fail(nullptr, ADMIX_ERR_ARG, "NULL device pointer");
    if (I < 1 || J < 1) return fail(nullptr, ADMIX_ERR_ARG, "I and J must be >= 1");
    if (K < 1 || K > ADMIX_MAX_K) return fail(nullptr, ADMIX_ERR_UNSUPPORTED, "K=%d outside [1, %d]", K, ADMIX_MAX_K);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return fail(nullptr, ADMIX_ERR_CUDA, "no current CUDA device");
    const LoglikPlan pl = plan_loglik(I, J, sms);
    if (work_bytes < sizeof(double) * (size_t)pl.gx * pl.gy)
        return fail(nullptr, ADMIX_ERR_ARG, "workspace of %zu bytes is below the %zu required", work_bytes,
                    sizeof(double) * (size_t)pl.gx * pl.gy);
    cudaError_t e = launch_loglik_f64(K, d_bed, I, J, (I + 3) / 4, d_q, d_p, pl, (double *)d_work, d_out, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(nullptr, ADMIX_ERR_CUDA, "loglik launch failed: %s", cudaGetErrorString(e));
    return ADMIX_OK;
}

} /* extern "C" */

/* ===================================================================== batches
 * Restarts and K sweeps over one cohort: n member handles over one device copy of the
 * genotypes.  A batch iteration is one graph launch: per active member a branch
 * [iteration number H2D] -> [the member's captured iteration graph] -> [scalars D2H]; branches
 * are independent, so the members' kernels run concurrently and fill the GPU even when one
 * member alone would not. */

struct admix_batch {
    int64_t I = 0, J = 0, pitch = 0;
    uint32_t flags = 0;
    int sms = 148, divisor = 1;
    cudaStream_t st = nullptr;
    uint8_t *bed = nullptr;
    std::vector<admix_ctx *> m;
    cudaGraphExec_t exec = nullptr;
    std::vector<int> exec_members;
    char err[512] = {0};
};

static int bfail(admix_batch *b, int code, const char *fmt, ...)
{
    char *dst = b ? b->err : g_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
    return code;
}

#define BCK(b, call)                                                                           \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return bfail((b), ADMIX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

static void batch_release(admix_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (admix_ctx *h : b->m) {
        if (!h) continue;
        if (h->st) cudaStreamSynchronize(h->st);
        release(h);
        delete h;
    }
    if (b->bed) cudaFree(b->bed);
    if (b->st) cudaStreamDestroy(b->st);
}

/* Plans of one member as if it had sms_eff SMs to itself.  The partial-sum buffers were sized
 * for the full SM count: the FP64 plans' slice counts only shrink with fewer SMs, and the mixed
 * plans are held to the slice counts of the handle's first plans. */
static void set_plans(admix_ctx *h, int sms_eff)
{
    h->llp = plan_loglik(h->I, h->J, sms_eff);
    h->sq = plan_sweep_q(h->K, h->I, h->J, sms_eff);
    h->sp = plan_sweep_p(h->K, h->I, h->J, sms_eff);
    h->sqm = plan_sweep_q_mixed(h->K, h->I, h->J, sms_eff, h->cap_sqm);
    h->spm = plan_sweep_p_mixed(h->K, h->I, h->J, sms_eff, h->cap_spm);
    h->llm = plan_loglik_mixed(h->K, h->I, h->J, sms_eff, h->cap_llm);
    if (h->iter_graph) { cudaGraphExecDestroy(h->iter_graph); h->iter_graph = nullptr; }
    if (h->iter_graph_def) { cudaGraphDestroy(h->iter_graph_def); h->iter_graph_def = nullptr; }
}

static void batch_invalidate(admix_batch *b)
{
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    b->exec_members.clear();
}

static int batch_sync_members(admix_batch *b)
{
    for (admix_ctx *h : b->m) BCK(b, cudaStreamSynchronize(h->st));
    return ADMIX_OK;
}

/* one graph: per listed member an independent branch built by `branch` */
template <class F>
static int batch_compose(admix_batch *b, const std::vector<int> &members, F branch, cudaGraphExec_t *exec)
{
    cudaGraph_t g = nullptr;
    BCK(b, cudaGraphCreate(&g, 0));
    for (int mi : members) {
        int rc = branch(g, b->m[mi]);
        if (rc != ADMIX_OK) { cudaGraphDestroy(g); return rc; }
    }
    cudaError_t e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { *exec = nullptr; return bfail(b, ADMIX_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e)); }
    return ADMIX_OK;
}

static int batch_iteration_graph(admix_batch *b, const std::vector<int> &active)
{
    if (b->exec && active == b->exec_members) return ADMIX_OK;
    batch_invalidate(b);
    auto branch = [b](cudaGraph_t g, admix_ctx *h) -> int {
        if (ensure_graph(h) != ADMIX_OK) return bfail(b, ADMIX_ERR_CUDA, "member capture: %s", h->err);
        cudaGraphNode_t n0, n1, n2;
        BCK(b, cudaGraphAddMemcpyNode1D(&n0, g, nullptr, 0, &h->sc->iter, h->iter_host, sizeof(int32_t),
                                        cudaMemcpyHostToDevice));
        BCK(b, cudaGraphAddChildGraphNode(&n1, g, &n0, 1, h->iter_graph_def));
        BCK(b, cudaGraphAddMemcpyNode1D(&n2, g, &n1, 1, h->sc_host, h->sc, sizeof(DevScalars),
                                        cudaMemcpyDeviceToHost));
        return ADMIX_OK;
    };
    int rc = batch_compose(b, active, branch, &b->exec);
    if (rc == ADMIX_OK) b->exec_members = active;
    return rc;
}

/* Member passes captured as one graph per member: Q sweep, P sweep and the iteration's
 * log-likelihood form, all on X (they write only partial sums and a scratch scalar). */
static int capture_probe(admix_batch *b, admix_ctx *h, cudaGraph_t *out)
{
    *out = nullptr;
    BCK(b, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    int S;
    cudaError_t e = enq_sweep_q(h, ADMIX_X, ADMIX_X, &S);
    if (e == cudaSuccess) e = enq_sweep_p(h, ADMIX_X, ADMIX_X, &S);
    if (e == cudaSuccess) e = enq_loglik(h, ADMIX_X, &h->sc->ll_tmp, true);
    cudaError_t e2 = cudaStreamEndCapture(h->st, out);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (*out) cudaGraphDestroy(*out);
        *out = nullptr;
        return bfail(b, ADMIX_ERR_CUDA, "probe capture: %s / %s", cudaGetErrorString(e), cudaGetErrorString(e2));
    }
    return ADMIX_OK;
}

static int time_probe(admix_batch *b, double *ms)
{
    std::vector<int> all(b->m.size());
    for (size_t t = 0; t < all.size(); ++t) all[t] = (int)t;
    cudaGraphExec_t ex = nullptr;
    auto branch = [b](cudaGraph_t g, admix_ctx *h) -> int {
        cudaGraph_t pg = nullptr;
        int rc = capture_probe(b, h, &pg);
        if (rc != ADMIX_OK) return rc;
        cudaGraphNode_t n;
        cudaError_t e = cudaGraphAddChildGraphNode(&n, g, nullptr, 0, pg);
        cudaGraphDestroy(pg);
        if (e != cudaSuccess) return bfail(b, ADMIX_ERR_CUDA, "probe node: %s", cudaGetErrorString(e));
        return ADMIX_OK;
    };
    int rc = batch_compose(b, all, branch, &ex);
    if (rc != ADMIX_OK) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaGraphLaunch(ex, b->st);                 /* warm-up */
    if (e == cudaSuccess) e = cudaEventRecord(e0, b->st);
    for (int r = 0; r < 2 && e == cudaSuccess; ++r) e = cudaGraphLaunch(ex, b->st);
    if (e == cudaSuccess) e = cudaEventRecord(e1, b->st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float f = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGraphExecDestroy(ex);
    if (e != cudaSuccess) return bfail(b, ADMIX_ERR_CUDA, "probe timing: %s", cudaGetErrorString(e));
    *ms = f / 2.0;
    return ADMIX_OK;
}

extern "C" {

static int batch_create_common(int64_t I, int64_t J, const uint8_t *bed, bool on_device, int64_t src_pitch,
                               int32_t n, const int32_t *Ks, int32_t Q, uint32_t flags, admix_batch **out)
{
    if (!out) return bfail(nullptr, ADMIX_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (n < 1 || !Ks) return bfail(nullptr, ADMIX_ERR_ARG, "a batch needs n >= 1 members and their K (n=%d)", n);
    if (I < 1 || J < 1) return bfail(nullptr, ADMIX_ERR_ARG, "I and J must be >= 1");
    if (!bed) return bfail(nullptr, ADMIX_ERR_ARG, "bed is NULL");
    if (src_pitch < (I + 3) / 4) return bfail(nullptr, ADMIX_ERR_ARG, "src_pitch %lld is below ceil(I/4) = %lld",
                                              (long long)src_pitch, (long long)((I + 3) / 4));
    for (int t = 0; t < n; ++t)
        if (Ks[t] < 1 || Ks[t] > ADMIX_MAX_K)
            return bfail(nullptr, ADMIX_ERR_UNSUPPORTED, "member %d: K=%d outside [1, %d]", t, Ks[t], ADMIX_MAX_K);
    if (Q < 1 || Q > ADMIX_MAX_Q) return bfail(nullptr, ADMIX_ERR_UNSUPPORTED, "Q=%d outside [1, %d]", Q, ADMIX_MAX_Q);
    if (flags & ~(ADMIX_FLAG_MU_GERSHGORIN | ADMIX_FLAG_MIXED | ADMIX_FLAG_MEAN_IMPUTE))
        return bfail(nullptr, ADMIX_ERR_ARG, "unknown flags 0x%x", flags);
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0) return bfail(nullptr, ADMIX_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(ce));

    admix_batch *b = new admix_batch();
    b->I = I; b->J = J; b->flags = flags;
    b->pitch = ((I + 3) / 4 + 15) / 16 * 16;
    b->m.assign((size_t)n, nullptr);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        e = cudaMalloc((void **)&b->bed, (size_t)b->pitch * J + 64);
        if (e != cudaSuccess) {
            b->bed = nullptr;
            bfail(nullptr, ADMIX_ERR_NOMEM, "cudaMalloc of %lld genotype bytes failed", (long long)(b->pitch * J + 64));
            batch_release(b); delete b;
            return ADMIX_ERR_NOMEM;
        }
    }
    if (e == cudaSuccess) e = upload_genotypes(b->bed, b->pitch, bed, src_pitch, I, J, on_device, b->sms, b->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) {
        bfail(nullptr, ADMIX_ERR_CUDA, "batch genotypes: %s", cudaGetErrorString(e));
        batch_release(b); delete b;
        return ADMIX_ERR_CUDA;
    }
    for (int t = 0; t < n; ++t) {
        int rc = create_common(I, J, Ks[t], Q, bed, on_device, src_pitch, flags, &b->m[t], b->bed);
        if (rc != ADMIX_OK) {
            char msg[512];
            snprintf(msg, sizeof(msg), "member %d: %s", t, g_err);
            batch_release(b); delete b;
            bfail(nullptr, rc, "%s", msg);
            return rc;
        }
    }
    *out = b;
    return ADMIX_OK;
}

int admix_batch_create(int64_t I, int64_t J, const uint8_t *bed, int32_t n, const int32_t *Ks, int32_t Q,
                       uint32_t flags, admix_batch **out)
{
    return batch_create_common(I, J, bed, false, (I + 3) / 4, n, Ks, Q, flags, out);
}

int admix_batch_create_device(int64_t I, int64_t J, const uint8_t *d_bed, int64_t src_pitch, int32_t n,
                              const int32_t *Ks, int32_t Q, uint32_t flags, admix_batch **out)
{
    cudaPointerAttributes at;
    if (d_bed && (cudaPointerGetAttributes(&at, d_bed) != cudaSuccess || at.type != cudaMemoryTypeDevice)) {
        cudaGetLastError();
        return bfail(nullptr, ADMIX_ERR_ARG, "d_bed is not device memory");
    }
    return batch_create_common(I, J, d_bed, true, src_pitch, n, Ks, Q, flags, out);
}

int admix_batch_destroy(admix_batch *b)
{
    if (!b) return ADMIX_OK;
    if (b->st) cudaStreamSynchronize(b->st);
    batch_release(b);
    delete b;
    return ADMIX_OK;
}

const char *admix_batch_last_error(const admix_batch *b) { return b ? b->err : g_err; }

int admix_batch_size(const admix_batch *b, int32_t *n)
{
    if (!b || !n) return bfail(nullptr, ADMIX_ERR_ARG, "NULL argument");
    *n = (int32_t)b->m.size();
    return ADMIX_OK;
}

int admix_batch_member(admix_batch *b, int32_t m, admix_ctx **h)
{
    if (!b || !h) return bfail(b, ADMIX_ERR_ARG, "NULL argument");
    if (m < 0 || m >= (int32_t)b->m.size()) return bfail(b, ADMIX_ERR_ARG, "member %d outside [0, %d)", m, (int)b->m.size());
    *h = b->m[m];
    return ADMIX_OK;
}

int admix_batch_init_em(admix_batch *b, int32_t iters, double *ll_hist)
{
    if (!b) return bfail(nullptr, ADMIX_ERR_ARG, "batch is NULL");
    if (iters < 0) return bfail(b, ADMIX_ERR_ARG, "iters must be >= 0");
    for (size_t t = 0; t < b->m.size(); ++t) {          /* member streams run concurrently */
        int rc = enq_init_em(b->m[t], iters, ll_hist ? ll_hist + t * (size_t)iters : nullptr);
        if (rc != ADMIX_OK) return bfail(b, rc, "member %d: %s", (int)t, b->m[t]->err);
    }
    for (size_t t = 0; t < b->m.size(); ++t) {
        const int rc = tc_err_sync(b->m[t]);
        if (rc != ADMIX_OK) return bfail(b, rc, "member %d: %s", (int)t, b->m[t]->err);
    }
    return ADMIX_OK;
}

int admix_batch_set_split(admix_batch *b, int32_t divisor)
{
    if (!b) return bfail(nullptr, ADMIX_ERR_ARG, "batch is NULL");
    if (divisor < 1) return bfail(b, ADMIX_ERR_ARG, "divisor must be >= 1 (got %d)", divisor);
    int rc = batch_sync_members(b);
    if (rc != ADMIX_OK) return rc;
    batch_invalidate(b);
    const int sms_eff = std::max(1, b->sms / divisor);
    for (admix_ctx *h : b->m) set_plans(h, sms_eff);
    b->divisor = divisor;
    return ADMIX_OK;
}

int admix_batch_autotune(admix_batch *b, int32_t *divisor, double *ms)
{
    if (!b) return bfail(nullptr, ADMIX_ERR_ARG, "batch is NULL");
    int rc = batch_sync_members(b);
    if (rc != ADMIX_OK) return rc;
    const int limit = std::max(1, 4 * (int)b->m.size());
    int best_d = 1;
    double best = 1e300;
    for (int d = 1; d <= limit && d <= b->sms; d *= 2) {
        rc = admix_batch_set_split(b, d);
        if (rc != ADMIX_OK) return rc;
        double t = 0.0;
        rc = time_probe(b, &t);
        if (rc != ADMIX_OK) return rc;
        if (t < best) { best = t; best_d = d; }
    }
    rc = admix_batch_set_split(b, best_d);
    if (rc != ADMIX_OK) return rc;
    if (divisor) *divisor = best_d;
    if (ms) *ms = best;
    return ADMIX_OK;
}

int admix_batch_run_qn(admix_batch *b, int32_t n_iter, double rtol, int32_t *n_done, int32_t *converged,
                       admix_iterinfo *last, double *ms_device)
{
    if (!b) return bfail(nullptr, ADMIX_ERR_ARG, "batch is NULL");
    if (n_iter < 0) return bfail(b, ADMIX_ERR_ARG, "n_iter must be >= 0");
    const int n = (int)b->m.size();
    int rc = batch_sync_members(b);
    if (rc != ADMIX_OK) return rc;
    /* a member without a log-likelihood gets its FP64 value first (algorithms_outer.jl:76-83) */
    for (admix_ctx *h : b->m) {
        BCK(b, cudaMemcpyAsync(h->sc_host, h->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->st));
        BCK(b, cudaStreamSynchronize(h->st));
        if (isnan(h->sc_host->ll_new)) BCK(b, enq_loglik(h, ADMIX_X, &h->sc->ll_new, true));
    }
    rc = batch_sync_members(b);
    if (rc != ADMIX_OK) return rc;
    batch_invalidate(b);                                /* members' fixed-block modes may have changed */
    std::vector<int> active(n), done(n, 0), conv(n, 0);
    for (int t = 0; t < n; ++t) active[t] = t;
    std::vector<admix_iterinfo> rec((size_t)n);
    memset(rec.data(), 0, sizeof(admix_iterinfo) * n);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    BCK(b, cudaEventCreate(&e0));
    cudaError_t e = cudaEventCreate(&e1);
    double total = 0.0;
    for (int it = 1; it <= n_iter && !active.empty() && e == cudaSuccess; ++it) {
        rc = batch_iteration_graph(b, active);
        if (rc != ADMIX_OK) break;
        for (int t : active) *b->m[t]->iter_host = it;
        e = cudaEventRecord(e0, b->st);
        if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, b->st);
        if (e == cudaSuccess) e = cudaEventRecord(e1, b->st);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float f = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
        total += f;
        std::vector<int> still;
        for (int t : active) {
            if (e != cudaSuccess) break;
            rc = tc_err_check(b->m[t]);   /* sc_host was copied inside the graph */
            if (rc != ADMIX_OK) {
                rc = bfail(b, rc, "member %d: %s", t, b->m[t]->err);
                break;
            }
            const DevScalars &s = *b->m[t]->sc_host;
            admix_iterinfo &r = rec[t];
            r.ll_prev = s.ll_prev; r.ll_basic = s.ll_basic; r.ll_qn = s.ll_qn; r.ll_new = s.ll_new;
            r.reldiff = s.reldiff; r.iter = it; r.accepted_qn = s.accepted; r.qp_fail_q = s.fail_q;
            r.qp_fail_p = s.fail_p;
            done[t] = it;
            if (s.reldiff < rtol) conv[t] = 1;
            else still.push_back(t);
        }
        if (rc != ADMIX_OK) break;
        active.swap(still);
    }
    cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc != ADMIX_OK) return rc;
    if (e != cudaSuccess) return bfail(b, ADMIX_ERR_CUDA, "batch iteration: %s", cudaGetErrorString(e));
    for (int t = 0; t < n; ++t) {
        if (n_done) n_done[t] = done[t];
        if (converged) converged[t] = conv[t];
        if (last) last[t] = rec[t];
    }
    if (ms_device) *ms_device = total;
    return ADMIX_OK;
}

} /* extern "C" */
