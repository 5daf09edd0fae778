/*
 * sdtfe_rng.h - counter-based random numbers for the Monte Carlo line-of-sight
 * samples and for the degeneracy perturbation of the ray walk.
 *
 * The reference draws both from the C library rand() (src/dtfe.c:621-622 for
 * the per-pixel sample offsets, src/dtfe.c:223 for the perturbation vertex),
 * which is shared between OpenMP threads and therefore not reproducible across
 * thread counts.  This library replaces that stream by pure functions of
 * (seed, pixel, sample) and (seed, ray, call counter), so that a GPU thread, a
 * CPU thread and the parity harness that drives the reference code all draw
 * the same numbers for the same ray.
 *
 * Mixing function: the SplitMix64 finaliser (Steele, Lea, Flood, "Fast
 * splittable pseudorandom number generators", OOPSLA 2014; constants as
 * published by S. Vigna).  Header-only; usable from C, C++ and CUDA.
 */
#ifndef SDTFE_RNG_H
#define SDTFE_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define SDTFE_HD __host__ __device__ __forceinline__
#else
#define SDTFE_HD static inline
#endif

SDTFE_HD uint64_t sdtfe_mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/* Uniform double in [0, 1) with 53 random bits for sample `sample` of pixel
 * `pixel`; axis 0 drives x, axis 1 drives y.  Plays the role of
 * (double)rand()/RAND_MAX in src/dtfe.c:621-622. */
SDTFE_HD double sdtfe_sample_u01(uint64_t seed, uint64_t pixel, uint32_t sample, uint32_t axis) {
  uint64_t h = sdtfe_mix64(seed + 0x632be59bd9b4e019ULL * (pixel + 1ULL));
  h = sdtfe_mix64(h ^ (((uint64_t)sample << 1) | (uint64_t)(axis & 1u)));
  return (double)(h >> 11) * 0x1.0p-53;
}

/* Non-negative 31-bit integer for the `counter`-th perturbation of ray `ray`:
 * the value the reference's perturb_ray (src/dtfe.c:223) takes modulo 4. */
SDTFE_HD int sdtfe_rand31(uint64_t seed, uint64_t ray, uint64_t counter) {
  uint64_t h = sdtfe_mix64((seed ^ 0xd1b54a32d192ed03ULL) + 0x9e3779b97f4a7c15ULL * (ray + 1ULL));
  h = sdtfe_mix64(h + counter);
  return (int)(h >> 33);
}

#undef SDTFE_HD
#endif /* SDTFE_RNG_H */
