/*
 * synth.h -- seeded synthetic admixed cohorts, one genotype cell at a time.
 *
 * The cell function is shared by the host generator (C, OpenMP) and the device
 * generator (CUDA): it uses only integer hashing, explicit fma() and comparisons, all
 * of which are correctly rounded on both sides, so both produce the same bytes.
 *
 * Model (the cohort generator the benchmark configurations describe):
 *   f_ij = sum_k q_ki p_kj, g_ij ~ Binomial(2, f_ij), missing with probability m.
 * PLINK 1 .bed 2-bit codes, LSB first, SNP-major:
 *   00 -> 0 copies, 10 -> 1 copy, 11 -> 2 copies, 01 -> missing
 * (the decode table of loops.jl:2-5, g_map = [0,0,1,2], nonmissing = [1,0,1,1]).
 */
#ifndef ADMIX_SYNTH_H
#define ADMIX_SYNTH_H
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define SYN_FN __host__ __device__ static inline
#else
#define SYN_FN static inline
#endif

/* splitmix64 finaliser used as a counter-based hash. */
SYN_FN uint64_t syn_mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

SYN_FN uint64_t syn_hash3(uint64_t seed, uint64_t a, uint64_t b)
{
    return syn_mix(syn_mix(seed + 0x9E3779B97F4A7C15ULL * (a + 1)) ^ (b * 0xD1B54A32D192ED03ULL + 0x8CB92BA72F3D8DD7ULL));
}

/* uniform double in [0,1) with 53 random bits (exact conversion) */
SYN_FN double syn_u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

/* 2-bit code of individual i at SNP j given the allele frequency f = sum_k q_ki p_kj. */
SYN_FN unsigned syn_code(uint64_t seed, int64_t i, int64_t j, double f, double miss_rate)
{
    uint64_t base = (uint64_t)i * 3u;
    double um = syn_u01(syn_hash3(seed, (uint64_t)j, base + 2));
    if (um < miss_rate) return 1u;
    double u1 = syn_u01(syn_hash3(seed, (uint64_t)j, base + 0));
    double u2 = syn_u01(syn_hash3(seed, (uint64_t)j, base + 1));
    int g = (u1 < f) + (u2 < f);
    return g == 0 ? 0u : (g == 1 ? 2u : 3u);
}

/* f = sum_k q[k] p[k] as an explicit fma chain in k order (bit-identical host/device). */
SYN_FN double syn_freq(const double *qi, const double *pj, int K)
{
    double s = 0.0;
    for (int k = 0; k < K; ++k) s = fma(qi[k], pj[k], s);
    return s;
}

#endif
