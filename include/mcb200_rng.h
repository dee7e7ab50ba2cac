/*
 * mcb200_rng.h -- the uniform random stream shared by the B200 carrier engine
 * and by anything that must reproduce its draws (the CPU oracle hook).
 *
 * The reference draws every uniform from one global sequential generator
 * (`Random()` / `ran1`, src/utils.cpp:426-470), consumed in particle order,
 * so its results depend on the order particles are visited.  This engine
 * replaces that generator with a counter-based Philox4x32-10 stream
 * (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11) keyed per particle, so every particle's draws are independent of
 * launch order and can be replayed exactly on the host.
 *
 * Stream of draw number n for (seed, uid, step, sub):
 *   key     = { seed & 0xffffffff, seed >> 32 }
 *   counter = { n >> 1, uid, step, sub }
 *   block   = Philox4x32-10(counter, key)            -> words w0..w3
 *   (hi,lo) = (w1,w0) for even n, (w3,w2) for odd n
 *   bits    = ((hi << 32) | lo) >> 12                 (52 bits)
 *   u       = (bits + 0.5) * 2^-52                    in (0, 1), never 0 or 1
 *
 * The FP32 flight path draws floats from the same blocks, four per block:
 *   block   = Philox4x32-10({ n >> 2, uid, step, sub }, key)
 *   w       = word (n & 3) of the block
 *   u       = ((w >> 9) + 0.5) * 2^-23                in (0, 1), never 0 or 1
 * (23 random bits; every value is exactly representable as a float).
 *
 * `sub` separates streams of the same particle within one step: 0 for the
 * particle's own flight, other values for particles created mid-step and for
 * the per-cell refresh draws.  Everything here is integer arithmetic plus one
 * exact int->double conversion and one exact scaling, so host and device
 * produce bit-identical doubles.
 */
#ifndef MCB200_RNG_H
#define MCB200_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define MCB200_HD __host__ __device__ __forceinline__
#else
#define MCB200_HD static inline
#endif

#define MCB200_PHILOX_M0 0xD2511F53u
#define MCB200_PHILOX_M1 0xCD9E8D57u
#define MCB200_PHILOX_W0 0x9E3779B9u
#define MCB200_PHILOX_W1 0xBB67AE85u

typedef struct { uint32_t w[4]; } mcb200_philox_block;

MCB200_HD void mcb200_mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
#if defined(__CUDA_ARCH__)
  *lo = a * b;
  *hi = __umulhi(a, b);
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *lo = (uint32_t)p;
  *hi = (uint32_t)(p >> 32);
#endif
}

MCB200_HD mcb200_philox_block mcb200_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                   uint32_t c3, uint32_t k0, uint32_t k1) {
  mcb200_philox_block r;
#if defined(__CUDA_ARCH__)
  /* kept rolled on the device: the block is computed at many call sites of
     the flight loop, and ten unrolled rounds at each would crowd the
     instruction cache */
#pragma unroll 1
#endif
  for (int round = 0; round < 10; ++round) {
    uint32_t hi0, lo0, hi1, lo1;
    mcb200_mulhilo32(MCB200_PHILOX_M0, c0, &hi0, &lo0);
    mcb200_mulhilo32(MCB200_PHILOX_M1, c2, &hi1, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += MCB200_PHILOX_W0;
    k1 += MCB200_PHILOX_W1;
  }
  r.w[0] = c0;
  r.w[1] = c1;
  r.w[2] = c2;
  r.w[3] = c3;
  return r;
}

/* Two 32-bit words -> a double in (0,1): 52 random bits centred in their bin. */
MCB200_HD double mcb200_bits_to_unit(uint32_t hi, uint32_t lo) {
  uint64_t bits = (((uint64_t)hi << 32) | (uint64_t)lo) >> 12;
  return ((double)bits + 0.5) * (1.0 / 4503599627370496.0); /* 2^-52 */
}

/* Draw number n of the stream (seed, uid, step, sub). */
MCB200_HD double mcb200_uniform(uint64_t seed, uint32_t uid, uint32_t step, uint32_t sub,
                                uint32_t n) {
  mcb200_philox_block b = mcb200_philox4x32_10(n >> 1, uid, step, sub, (uint32_t)seed,
                                               (uint32_t)(seed >> 32));
  return (n & 1u) ? mcb200_bits_to_unit(b.w[3], b.w[2]) : mcb200_bits_to_unit(b.w[1], b.w[0]);
}

/* One 32-bit word -> a float in (0,1): 23 random bits centred in their bin. */
MCB200_HD float mcb200_bits_to_unit_f32(uint32_t w) {
  return ((float)(w >> 9) + 0.5f) * (1.0f / 8388608.0f); /* 2^-23 */
}

/* Draw number n of the FP32 stream (seed, uid, step, sub). */
MCB200_HD float mcb200_uniform_f32(uint64_t seed, uint32_t uid, uint32_t step, uint32_t sub,
                                   uint32_t n) {
  mcb200_philox_block b = mcb200_philox4x32_10(n >> 2, uid, step, sub, (uint32_t)seed,
                                               (uint32_t)(seed >> 32));
  return mcb200_bits_to_unit_f32(b.w[n & 3u]);
}

#endif /* MCB200_RNG_H */
