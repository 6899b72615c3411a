/*
 * Philox4x32-10 counter-based random number generator, host and device.
 *
 * Written from the published description: J. K. Salmon, M. A. Moraes,
 * R. O. Dror and D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11.  One call maps a 128-bit counter and a 64-bit key to 128 random
 * bits; ten rounds of the multiply/xor bijection are applied, with the key
 * bumped by the Weyl constants between rounds.
 *
 * The sampler kernels never carry generator state: every random word is a
 * pure function of (key, counter), so any sub-range of a chain can be
 * recomputed bit for bit (halo rows of a tile, a CPU replay, a request that
 * is served alone or batched with others).
 *
 * Counter layout used by every kernel in this library:
 *   c0  unit index (MSC word, site or work item inside the colour class)
 *   c1  sweep index of the chain (low 32 bits)
 *   c2  stream tag: purpose | colour | plane group (see CRITMC_TAG_*)
 *   c3  chain-local extra index (lane quad, PT temperature pair, ...)
 */
#ifndef CRITMC_PHILOX_H
#define CRITMC_PHILOX_H

#include <stdint.h>

#if defined(__CUDACC__)
#define CRITMC_HD __host__ __device__ __forceinline__
#else
#define CRITMC_HD static inline
#endif

#define CRITMC_PHILOX_M0 0xD2511F53u
#define CRITMC_PHILOX_M1 0xCD9E8D57u
#define CRITMC_PHILOX_W0 0x9E3779B9u
#define CRITMC_PHILOX_W1 0xBB67AE85u

#ifndef CRITMC_PHILOX_ROUNDS
#define CRITMC_PHILOX_ROUNDS 10
#endif

/* stream tags (counter word c2); bits 0..7 purpose, 8..15 sub-index */
#define CRITMC_TAG_PLANES 0x01u   /* MSC acceptance planes, sub-index = plane group */
#define CRITMC_TAG_SITE 0x02u     /* per-site draws (byte/float layouts) */
#define CRITMC_TAG_SITE2 0x03u    /* per-site extra draws (rejection loops) */
#define CRITMC_TAG_SWAP 0x04u     /* replica-exchange acceptance */
#define CRITMC_TAG_INIT 0x05u     /* initial configurations */
#define CRITMC_TAG_COUPLING 0x06u /* quenched couplings */

typedef struct {
  uint32_t v[4];
} critmc_u32x4;

/* Philox4x32 with `rounds` rounds: 10 is the library's stream everywhere;
 * 7 (Salmon et al.'s smallest round count that passes BigCrush) is offered
 * only as an explicit option of the multi-spin-coded acceptance planes. */
CRITMC_HD critmc_u32x4 critmc_philox4x32_rounds(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                uint32_t k0, uint32_t k1, int rounds) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int r = 0; r < rounds; ++r) {
    /* one 32x32->64 product per lane word: a single wide multiply-add on the GPU */
    const uint64_t p0 = (uint64_t)CRITMC_PHILOX_M0 * c0;
    const uint64_t p1 = (uint64_t)CRITMC_PHILOX_M1 * c2;
    c0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    c1 = (uint32_t)p1;
    c2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c3 = (uint32_t)p0;
    k0 += CRITMC_PHILOX_W0;
    k1 += CRITMC_PHILOX_W1;
  }
  critmc_u32x4 out;
  out.v[0] = c0;
  out.v[1] = c1;
  out.v[2] = c2;
  out.v[3] = c3;
  return out;
}

CRITMC_HD critmc_u32x4 critmc_philox4x32(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                         uint32_t k0, uint32_t k1) {
  return critmc_philox4x32_rounds(c0, c1, c2, c3, k0, k1, CRITMC_PHILOX_ROUNDS);
}

/* ---------------------------------------------------------------------------
 * Acceptance planes of many words at once.  Plane group g of word w of one
 * colour at sweep t is Philox4x32-10(c0 = w, c1 = t, c2 = G_g, c3 = 0) under
 * the chain's key, G_g = TAG_PLANES | g << 8 | colour << 16.  Across the
 * words of one launch only c0 varies, so the rounds split into:
 *   round 0: outputs c0, c1 depend on (t, G_g, key) only; c2, c3 on w and the
 *            key but not on g;
 *   round 1: the product M0 * c0 is uniform, the product M1 * c2 is the same
 *            for every g;
 *   rounds 2..9: everything varies.
 * critmc_plane_stream holds the uniform values (round keys and the
 * g-dependent constants, for up to CRITMC_PLANE_GROUPS groups),
 * critmc_plane_word() the varying work shared by the groups of a word, and
 * critmc_plane_group() the rest of one group.  The result equals
 * critmc_philox4x32(w, t, G_g, 0, k0, k1) bit for bit; a word with KG
 * groups costs 2 + 16 KG wide multiplies instead of 20 KG.
 * ------------------------------------------------------------------------- */
#define CRITMC_PLANE_GROUPS 2

typedef struct {
  uint32_t k1;                                   /* key word 1 of round 0 */
  uint32_t x1[CRITMC_PLANE_GROUPS];              /* round-0 c1 ^ round-1 key word 0 */
  uint32_t x2[CRITMC_PLANE_GROUPS];              /* hi(M0 * round-0 c0) ^ round-1 key word 1 */
  uint32_t x3[CRITMC_PLANE_GROUPS];              /* lo(M0 * round-0 c0) ^ round-2 key word 1 */
  uint32_t k0_2;                                 /* key word 0 of round 2 */
  uint32_t rk0[CRITMC_PHILOX_ROUNDS - 3];        /* keys of rounds 3 .. */
  uint32_t rk1[CRITMC_PHILOX_ROUNDS - 3];
} critmc_plane_stream;

typedef struct {
  uint32_t v3, h1, l1; /* round-0 c3; hi and lo of the round-1 product M1 * c2 */
} critmc_plane_word_t;

CRITMC_HD void critmc_plane_stream_init(critmc_plane_stream* ps, uint32_t k0, uint32_t k1, uint32_t sweep,
                                        uint32_t col, int n_groups) {
  ps->k1 = k1;
  for (int g = 0; g < n_groups; ++g) {
    const uint32_t G = CRITMC_TAG_PLANES | ((uint32_t)g << 8) | (col << 16);
    const uint64_t p1 = (uint64_t)CRITMC_PHILOX_M1 * G;
    const uint32_t a = (uint32_t)(p1 >> 32) ^ sweep ^ k0;      /* round-0 c0 */
    const uint64_t pa = (uint64_t)CRITMC_PHILOX_M0 * a;         /* round-1 M0 * c0 */
    ps->x1[g] = (uint32_t)p1 ^ (k0 + CRITMC_PHILOX_W0);
    ps->x2[g] = (uint32_t)(pa >> 32) ^ (k1 + CRITMC_PHILOX_W1);
    ps->x3[g] = (uint32_t)pa ^ (k1 + 2u * CRITMC_PHILOX_W1);
  }
  ps->k0_2 = k0 + 2u * CRITMC_PHILOX_W0;
  for (int r = 3; r < CRITMC_PHILOX_ROUNDS; ++r) {
    ps->rk0[r - 3] = k0 + (uint32_t)r * CRITMC_PHILOX_W0;
    ps->rk1[r - 3] = k1 + (uint32_t)r * CRITMC_PHILOX_W1;
  }
}

CRITMC_HD critmc_plane_word_t critmc_plane_word(const critmc_plane_stream* ps, uint32_t w) {
  const uint64_t p0 = (uint64_t)CRITMC_PHILOX_M0 * w;
  const uint32_t v2 = (uint32_t)(p0 >> 32) ^ ps->k1;
  const uint64_t p1 = (uint64_t)CRITMC_PHILOX_M1 * v2;
  critmc_plane_word_t pw;
  pw.v3 = (uint32_t)p0;
  pw.h1 = (uint32_t)(p1 >> 32);
  pw.l1 = (uint32_t)p1;
  return pw;
}

/* planes 4 g .. 4 g + 3 of a word (word q of the result is plane 4 g + q), for a
 * Philox of `rounds` rounds (3 .. CRITMC_PHILOX_ROUNDS; the stream object holds
 * the keys of the longest) */
CRITMC_HD critmc_u32x4 critmc_plane_group_rounds(const critmc_plane_stream* ps, critmc_plane_word_t pw, int g,
                                                 int rounds) {
  uint32_t c0 = pw.h1 ^ ps->x1[g]; /* state after round 1 */
  uint32_t c1 = pw.l1;
  uint32_t c2 = pw.v3 ^ ps->x2[g];
  uint64_t p0 = (uint64_t)CRITMC_PHILOX_M0 * c0; /* round 2: its c3 input is uniform */
  uint64_t p1 = (uint64_t)CRITMC_PHILOX_M1 * c2;
  c0 = (uint32_t)(p1 >> 32) ^ c1 ^ ps->k0_2;
  c1 = (uint32_t)p1;
  c2 = (uint32_t)(p0 >> 32) ^ ps->x3[g];
  uint32_t c3 = (uint32_t)p0;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int r = 0; r < rounds - 3; ++r) {
    p0 = (uint64_t)CRITMC_PHILOX_M0 * c0;
    p1 = (uint64_t)CRITMC_PHILOX_M1 * c2;
    c0 = (uint32_t)(p1 >> 32) ^ c1 ^ ps->rk0[r];
    c1 = (uint32_t)p1;
    c2 = (uint32_t)(p0 >> 32) ^ c3 ^ ps->rk1[r];
    c3 = (uint32_t)p0;
  }
  critmc_u32x4 out;
  out.v[0] = c0;
  out.v[1] = c1;
  out.v[2] = c2;
  out.v[3] = c3;
  return out;
}

CRITMC_HD critmc_u32x4 critmc_plane_group(const critmc_plane_stream* ps, critmc_plane_word_t pw, int g) {
  return critmc_plane_group_rounds(ps, pw, g, CRITMC_PHILOX_ROUNDS);
}

/* uniform double in [0, 1) with 53 random bits from two words */
CRITMC_HD double critmc_u01_53(uint32_t a, uint32_t b) {
  const uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return (double)m * (1.0 / 9007199254740992.0);
}

/* uniform float in (0, 1] with 24 random bits (never 0, safe for logf) */
CRITMC_HD float critmc_u01f_open0(uint32_t a) {
  return (float)((a >> 8) + 1u) * (1.0f / 16777216.0f);
}

/* uniform float in [0, 1) with 24 random bits */
CRITMC_HD float critmc_u01f(uint32_t a) { return (float)(a >> 8) * (1.0f / 16777216.0f); }

#endif /* CRITMC_PHILOX_H */
