/* Host harness: the split evaluation of the acceptance-plane stream
 * (critmc_plane_stream_init / _word / _group in philox.h) next to the plain
 * Philox4x32-10 call it must equal. */
#include <stdint.h>

#include "philox.h"

/* rows of `in`: k0, k1, sweep, colour, word; out_*: [n][groups][4]; rounds 0 = the default */
void plane_eval(int n, int groups, int rounds, const uint32_t* in, uint32_t* out_plain, uint32_t* out_split) {
  for (int i = 0; i < n; ++i) {
    const uint32_t* a = in + 5 * i;
    critmc_plane_stream ps;
    critmc_plane_stream_init(&ps, a[0], a[1], a[2], a[3], groups);
    const critmc_plane_word_t pw = critmc_plane_word(&ps, a[4]);
    for (int g = 0; g < groups; ++g) {
      const uint32_t G = CRITMC_TAG_PLANES | ((uint32_t)g << 8) | (a[3] << 16);
      const critmc_u32x4 ref = rounds ? critmc_philox4x32_rounds(a[4], a[2], G, 0u, a[0], a[1], rounds)
                                      : critmc_philox4x32(a[4], a[2], G, 0u, a[0], a[1]);
      const critmc_u32x4 got = rounds ? critmc_plane_group_rounds(&ps, pw, g, rounds) : critmc_plane_group(&ps, pw, g);
      for (int q = 0; q < 4; ++q) {
        out_plain[(i * groups + g) * 4 + q] = ref.v[q];
        out_split[(i * groups + g) * 4 + q] = got.v[q];
      }
    }
  }
}

/* plain Philox4x32 with `rounds` rounds of the library header, for comparison with the oracle's */
void philox_eval(int n, int rounds, const uint32_t* in, uint32_t* out) {
  for (int i = 0; i < n; ++i) {
    const uint32_t* a = in + 6 * i;
    const critmc_u32x4 r = critmc_philox4x32_rounds(a[0], a[1], a[2], a[3], a[4], a[5], rounds);
    for (int q = 0; q < 4; ++q) out[4 * i + q] = r.v[q];
  }
}
