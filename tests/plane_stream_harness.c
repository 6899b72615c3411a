/* Host harness: the split evaluation of the acceptance-plane stream
 * (critmc_plane_stream_init / _word / _group in philox.h) next to the plain
 * Philox4x32-10 call it must equal. */
#include <stdint.h>

#include "philox.h"

/* rows of `in`: k0, k1, sweep, colour, word; out_*: [n][groups][4] */
void plane_eval(int n, int groups, const uint32_t* in, uint32_t* out_plain, uint32_t* out_split) {
  for (int i = 0; i < n; ++i) {
    const uint32_t* a = in + 5 * i;
    critmc_plane_stream ps;
    critmc_plane_stream_init(&ps, a[0], a[1], a[2], a[3], groups);
    const critmc_plane_word_t pw = critmc_plane_word(&ps, a[4]);
    for (int g = 0; g < groups; ++g) {
      const critmc_u32x4 ref =
          critmc_philox4x32(a[4], a[2], CRITMC_TAG_PLANES | ((uint32_t)g << 8) | (a[3] << 16), 0u, a[0], a[1]);
      const critmc_u32x4 got = critmc_plane_group(&ps, pw, g);
      for (int q = 0; q < 4; ++q) {
        out_plain[(i * groups + g) * 4 + q] = ref.v[q];
        out_split[(i * groups + g) * 4 + q] = got.v[q];
      }
    }
  }
}
