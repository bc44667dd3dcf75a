/*
 * Seeded synthetic single-cell counts, shared by the CPU and GPU generators.
 *
 * Count of gene g in cell c is negative-binomial with mean
 *   mu = lib[c] * prob[label[c]][g]
 * and dispersion phi (variance mu + phi mu^2), drawn by inversion of its CDF
 * with one counter-based uniform per (cell, gene): u = SplitMix64(seed,
 * c, g) / 2^64.  Zero when u < P(0) = (1 + phi mu)^(-1/phi); otherwise the
 * smallest k with CDF(k) > u, using P(k)/P(k-1) = (k - 1 + r)/k * q,
 * r = 1/phi, q = phi mu / (1 + phi mu).
 *
 * Because every (cell, gene) draw is independent of the others, the same
 * matrix comes out of any partition of the work, on the CPU or the GPU (up
 * to last-ulp differences of exp/log1p between libm and CUDA, which can only
 * flip a draw whose uniform lies within ~1e-16 of a CDF value).
 */
#ifndef CREST_SYNTH_CORE_H
#define CREST_SYNTH_CORE_H

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SYN_HD __host__ __device__ __forceinline__
#else
#define SYN_HD static inline
#endif

SYN_HD uint64_t syn_mix(uint64_t x) { /* SplitMix64 finaliser (Steele, Lea, Flood 2014) */
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

SYN_HD double syn_uniform(uint64_t seed, uint64_t cell, uint64_t gene) {
    const uint64_t key = syn_mix(seed ^ syn_mix(cell * 0xd1b54a32d192ed03ull + 0x8cb92ba72f3d8dd7ull)) +
                         gene * 0xaef17502108ef2d9ull;
    return (double)(syn_mix(key) >> 11) * 0x1.0p-53;
}

/* Returns the count; r = 1/phi. */
SYN_HD uint32_t syn_count(double mu, double phi, double r, double u) {
    if (!(mu > 0.0)) return 0u;
    /* P(0) = (1 + phi mu)^(-1/phi) >= 1 - mu (Bernoulli's inequality), so a
     * uniform clearly below 1 - mu draws zero without exp/log1p: the same
     * count as the full test, at a fraction of the cost for rare genes. */
    if (u < 1.0 - mu - 1e-12) return 0u;
    const double pm = phi * mu;
    const double p0 = exp(-r * log1p(pm));
    if (u < p0) return 0u;
    const double q = pm / (1.0 + pm);
    double pk = p0, cdf = p0;
    uint32_t k = 0;
    while (cdf <= u && k < 1000000u) {
        k += 1;
        pk *= ((double)(k - 1) + r) / (double)k * q;
        cdf += pk;
        if (pk == 0.0 && cdf <= u) break; /* numerically exhausted tail */
    }
    return k;
}

#endif
