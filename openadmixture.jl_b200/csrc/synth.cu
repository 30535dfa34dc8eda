/*
 * synth.cu -- seeded synthetic admixed cohorts written as PLINK .bed columns.
 *
 * Host entry points (C, OpenMP) generate the ground-truth Q (Dirichlet) and P
 * (uniform or clipped Beta), the genotype bytes, and the random initial point the
 * reference draws in AdmixData (structs.jl:107,128: x = rand(K, I+J), Q columns
 * normalised, P left unprojected).  A device entry point fills the same bytes on the
 * GPU for cohorts too large to build on the host quickly; both share synth.h, so the
 * bytes are identical.
 *
 * This library is a data utility for tests and benchmarks; it is not part of the
 * likelihood engine (libadmix).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "synth.h"

/* ---- host-side sequential stream seeded from the counter hash ---- */
typedef struct { uint64_t s; } syn_stream;

static inline double st_u01(syn_stream *st)
{
    st->s += 0x9E3779B97F4A7C15ULL;
    return syn_u01(syn_mix(st->s));
}

static double st_normal(syn_stream *st)
{
    double u1 = 1.0 - st_u01(st);         /* (0, 1] */
    double u2 = st_u01(st);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* Marsaglia & Tsang (2000), "A simple method for generating gamma variables";
 * shape < 1 via the boost Gamma(a) = Gamma(a+1) * U^(1/a). */
static double st_gamma(syn_stream *st, double a)
{
    if (a < 1.0) {
        double g = st_gamma(st, a + 1.0);
        double u = 1.0 - st_u01(st);
        return g * pow(u, 1.0 / a);
    }
    double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
    for (;;) {
        double x = st_normal(st), v = 1.0 + c * x;
        if (v <= 0.0) continue;
        v = v * v * v;
        double u = 1.0 - st_u01(st);
        if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) return d * v;
    }
}

extern "C" {

/* Ground truth: q_true (K x I, columns ~ Dirichlet(alpha 1_K)) and p_true (K x J):
 * p_dist 0: Uniform(p_lo, p_hi); p_dist 1: Beta(beta_a, beta_a) clipped to [p_lo, p_hi]. */
int syn_truth(int64_t I, int64_t J, int32_t K, uint64_t seed, int32_t p_dist,
              double p_lo, double p_hi, double beta_a, double alpha,
              double *q_true, double *p_true)
{
    if (I < 0 || J < 0 || K < 1 || !q_true || !p_true) return 1;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < I; ++i) {
        syn_stream st = { syn_hash3(seed ^ 0x51ULL, 1, (uint64_t)i) };
        double s = 0.0;
        for (int k = 0; k < K; ++k) { double g = st_gamma(&st, alpha); q_true[(size_t)K * i + k] = g; s += g; }
        if (!(s > 0.0)) {               /* all shapes underflowed: put the mass on one cluster */
            for (int k = 0; k < K; ++k) q_true[(size_t)K * i + k] = (k == (int)(i % K)) ? 1.0 : 0.0;
        } else {
            for (int k = 0; k < K; ++k) q_true[(size_t)K * i + k] /= s;
        }
    }
    #pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < J; ++j) {
        syn_stream st = { syn_hash3(seed ^ 0x52ULL, 2, (uint64_t)j) };
        for (int k = 0; k < K; ++k) {
            double v;
            if (p_dist == 0) {
                v = p_lo + (p_hi - p_lo) * st_u01(&st);
            } else {
                double a = st_gamma(&st, beta_a), b = st_gamma(&st, beta_a);
                v = (a + b > 0.0) ? a / (a + b) : 0.5;
                v = fmin(fmax(v, p_lo), p_hi);
            }
            p_true[(size_t)K * j + k] = v;
        }
    }
    return 0;
}

/* Genotype bytes on the host: bed is ceil(I/4) x J, SNP-major; padding bits are 00. */
int syn_bed_host(int64_t I, int64_t J, int32_t K, uint64_t seed, double miss_rate,
                 const double *q, const double *p, uint8_t *bed)
{
    if (I < 0 || J < 0 || K < 1 || !bed) return 1;
    const int64_t Ib = (I + 3) / 4;
    #pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < J; ++j) {
        const double *pj = p + (size_t)K * j;
        uint8_t *col = bed + (size_t)Ib * j;
        for (int64_t b = 0; b < Ib; ++b) {
            unsigned byte = 0;
            for (int s = 0; s < 4; ++s) {
                int64_t i = 4 * b + s;
                if (i >= I) break;
                double f = syn_freq(q + (size_t)K * i, pj, K);
                byte |= syn_code(seed, i, j, f, miss_rate) << (2 * s);
            }
            col[b] = (uint8_t)byte;
        }
    }
    return 0;
}

/* Initial point of AdmixData{T}(I, J, K, Q) (structs.jl:107,128): x ~ U(0,1)^(K x (I+J)),
 * then the Q block's columns divided by their sums.  x is K*(I+J), Q block first. */
int syn_init_x(int64_t I, int64_t J, int32_t K, uint64_t seed, double *x)
{
    if (I < 0 || J < 0 || K < 1 || !x) return 1;
    const int64_t n = I + J;
    #pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c)
        for (int k = 0; k < K; ++k)
            x[(size_t)K * c + k] = syn_u01(syn_hash3(seed ^ 0x1717ULL, (uint64_t)c, (uint64_t)k));
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < I; ++i) {
        double s = 0.0;
        for (int k = 0; k < K; ++k) s += x[(size_t)K * i + k];
        for (int k = 0; k < K; ++k) x[(size_t)K * i + k] /= s;
    }
    return 0;
}

} /* extern "C" */

/* ---- device generator: one thread per output byte ---- */
static __global__ void syn_bed_kernel(int64_t I, int64_t J, int K, uint64_t seed, double miss_rate,
                                      const double *__restrict__ q, const double *__restrict__ p,
                                      uint8_t *__restrict__ bed)
{
    const int64_t Ib = (I + 3) / 4;
    const int64_t total = Ib * J;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t j = t / Ib, b = t - j * Ib;
        const double *pj = p + (size_t)K * j;
        unsigned byte = 0;
        for (int s = 0; s < 4; ++s) {
            int64_t i = 4 * b + s;
            if (i >= I) break;
            double f = syn_freq(q + (size_t)K * i, pj, K);
            byte |= syn_code(seed, i, j, f, miss_rate) << (2 * s);
        }
        bed[t] = (uint8_t)byte;
    }
}

extern "C" int syn_bed_device(int64_t I, int64_t J, int32_t K, uint64_t seed, double miss_rate,
                              const double *d_q, const double *d_p, uint8_t *d_bed, void *stream)
{
    if (I <= 0 || J <= 0 || K < 1 || !d_q || !d_p || !d_bed) return 1;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    syn_bed_kernel<<<sms * 8, 256, 0, (cudaStream_t)stream>>>(I, J, K, seed, miss_rate, d_q, d_p, d_bed);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
