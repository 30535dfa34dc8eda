/*
 * loglik_noalloc.cu -- log-likelihood on caller-owned device arrays without allocating.
 *
 * admix_loglik_dev needs a workspace for its per-block partial sums, which the caller must
 * allocate.  Some callers cannot: a host whose device memory is handed out only by its own
 * pool allocator (and that has no scratch to lend), or a caller on a latency-critical path
 * that must not pay cudaMalloc's implicit device-wide synchronisation.  For them,
 * admix_loglik_dev_noalloc keeps the partial sums in a fixed array compiled into this library
 * (ADMIX_NOALLOC_MAX_PARTIALS doubles = 256 KiB); every GPU that loads the library holds that
 * array until the process exits.
 *
 * The array is shared by every call.  Each call writes all the partial-sum slots it later
 * reads, so no slot has to start at zero, but two calls that overlap on the GPU (different
 * streams or host threads) race on the slots and can return wrong results: serialise them.
 *
 * Host code cannot hand the array's name to a kernel (in host code it is only a stand-in
 * for the symbol, not a device address).  The first call on each device, with that device
 * current, looks the device address up with cudaGetSymbolAddress and caches it together with
 * the device's current context; make that first call before any stream capture.  A device
 * reset (cudaDeviceReset, or a host runtime that destroys and recreates the primary context)
 * reloads the module and may move the array, so the address is looked up again whenever the
 * current context is not the one it was cached under.
 */
#include <cuda.h>
#include <cuda_runtime.h>
#include <mutex>
#include <stdio.h>
#include "../../include/admix.h"
#include "kernels.h"

static __device__ __align__(256) double g_loglik_scratch[ADMIX_NOALLOC_MAX_PARTIALS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch[kMaxDevices];
CUcontext g_ctx[kMaxDevices];      /* the context each cached address belongs to */
bool g_ready[kMaxDevices];
thread_local char g_msg[256];

int noalloc_fail(int code, const char *msg)
{
    snprintf(g_msg, sizeof(g_msg), "%s", msg);
    return code;
}
} // namespace

extern "C" const char *admix_noalloc_last_error(void) { return g_msg; }

extern "C" int admix_loglik_dev_noalloc(const uint8_t *d_bed, int64_t I, int64_t J, int32_t K,
                                        const double *d_q, const double *d_p, double *d_out,
                                        void *stream)
{
    g_msg[0] = 0;   /* a successful call leaves no stale message behind */
    if (!d_bed || !d_q || !d_p || !d_out) return noalloc_fail(ADMIX_ERR_ARG, "NULL device pointer");
    if (I < 1 || J < 1) return noalloc_fail(ADMIX_ERR_ARG, "I and J must be >= 1");
    if (K < 1 || K > ADMIX_MAX_K) return noalloc_fail(ADMIX_ERR_UNSUPPORTED, "K outside [1, ADMIX_MAX_K]");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return noalloc_fail(ADMIX_ERR_CUDA, "no current CUDA device");
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(ADMIX_ERR_UNSUPPORTED, "device index beyond 63");
    const LoglikPlan pl = plan_loglik(I, J, sms);
    const int64_t nparts = (int64_t)pl.gx * pl.gy;
    if (nparts > ADMIX_NOALLOC_MAX_PARTIALS) {
        char buf[200];
        snprintf(buf, sizeof(buf), "this cohort needs %lld partial sums; the static scratch holds %d "
                 "(I up to about 33 million individuals)", (long long)nparts, ADMIX_NOALLOC_MAX_PARTIALS);
        return noalloc_fail(ADMIX_ERR_UNSUPPORTED, buf);
    }
    /* the runtime call above made the device's primary context current; the driver's
     * cuCtxGetCurrent is reached through the runtime, so the library needs no libcuda link */
    CUcontext ctx = nullptr;
    {
        static CUresult (*get_ctx)(CUcontext *) = nullptr;
        if (!get_ctx) {
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
                q != cudaDriverEntryPointSuccess || !fn)
                return noalloc_fail(ADMIX_ERR_CUDA, "cuCtxGetCurrent is not available");
            get_ctx = (CUresult(*)(CUcontext *))fn;
        }
        if (get_ctx(&ctx) != CUDA_SUCCESS || ctx == nullptr)
            return noalloc_fail(ADMIX_ERR_CUDA, "no current CUDA context");
    }
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_ready[dev] || g_ctx[dev] != ctx) {
            cudaError_t e = cudaGetSymbolAddress(&g_scratch[dev], g_loglik_scratch);
            if (e != cudaSuccess) {
                char buf[200];
                snprintf(buf, sizeof(buf), "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return noalloc_fail(ADMIX_ERR_CUDA, buf);
            }
            g_ctx[dev] = ctx;
            g_ready[dev] = true;
        }
        scratch = g_scratch[dev];
    }
    cudaError_t e = launch_loglik_f64(K, d_bed, I, J, (I + 3) / 4, d_q, d_p, pl, (double *)scratch, d_out,
                                      (cudaStream_t)stream);
    if (e != cudaSuccess) return noalloc_fail(ADMIX_ERR_CUDA, cudaGetErrorString(e));
    return ADMIX_OK;
}
