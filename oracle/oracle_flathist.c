/*
 * CPU oracle for the flat-histogram walks -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates critmc's Wang-Landau and multicanonical kernels
 *   wl_ising, wl_potts, muca_ising, muca_potts   src/critmc/kernels/flathist.py:28-132
 * for one walker with the GPU's random stream: move t draws
 * Philox(t mod 2^32, t / 2^32, 0x0A, 0); word 0 picks the site, word 1 the
 * Potts proposal, words 2, 3 the 53-bit uniform u.  critmc accepts when
 * ln w(new) >= ln w(old) or u < exp(ln w(new) - ln w(old)) (flathist.py:22-25);
 * this restatement tests ln u < ln w(new) - ln w(old) instead, the same event
 * in exact arithmetic, with cm_log of critmc_b200/csrc/fpmath.h (this file is
 * built without floating-point contraction).
 */
#include <math.h>
#include <stdint.h>

#include "fpmath.h"
#include "oracle.h"

static double u53(uint32_t a, uint32_t b) {
  const uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return (double)m * (1.0 / 9007199254740992.0);
}

static int64_t delta(const int8_t* s, int dim, int lx, int ly, int lz, int q, int i, uint32_t w1, int* nv) {
  const int x = i % lx, y = (i / lx) % ly, z = i / (lx * ly);
  int nb[6], zc = 2;
  nb[0] = (x + 1 == lx ? 0 : x + 1) + lx * (y + ly * z);
  nb[1] = (x == 0 ? lx - 1 : x - 1) + lx * (y + ly * z);
  if (dim >= 2) {
    nb[2] = x + lx * ((y + 1 == ly ? 0 : y + 1) + ly * z);
    nb[3] = x + lx * ((y == 0 ? ly - 1 : y - 1) + ly * z);
    zc = 4;
  }
  if (dim == 3) {
    nb[4] = x + lx * (y + ly * (z + 1 == lz ? 0 : z + 1));
    nb[5] = x + lx * (y + ly * (z == 0 ? lz - 1 : z - 1));
    zc = 6;
  }
  const int old = s[i];
  if (q == 0) {
    int field = 0;
    for (int k = 0; k < zc; ++k) field += s[nb[k]];
    *nv = -old;
    return (old * field) / 2; /* even: exact */
  }
  int ns = (int)(((uint64_t)w1 * (uint64_t)(q - 1)) >> 32);
  if (ns >= old) ++ns;
  *nv = ns;
  int n_old = 0, n_new = 0;
  for (int k = 0; k < zc; ++k) {
    if (s[nb[k]] == old) ++n_old;
    else if (s[nb[k]] == ns) ++n_new;
  }
  return n_old - n_new;
}

int oracle_fh_run(int mode, int8_t* s, int dim, int lx, int ly, int lz, int q, const uint32_t key[2],
                  int64_t* idx_io, int64_t* order, double* lng, int64_t* hist, int lo, int hi,
                  uint64_t* trials, double ln_f, double n_levels, int one_over_t, uint64_t t_base,
                  int64_t moves, int n_meas, int64_t* idx_out, int64_t* order_out) {
  if (dim < 2) ly = 1;
  if (dim < 3) lz = 1;
  const int n = lx * ly * lz;
  int64_t idx = *idx_io;
  uint64_t t = *trials;
  int64_t m = q == 0 ? order[0] : 0;
  const int rounds = mode == 0 ? 1 : n_meas;
  for (int meas = 0; meas < rounds; ++meas) {
    for (int64_t j = 0; j < moves; ++j, ++t) {
      uint32_t w[4];
      const uint32_t ctr[4] = {(uint32_t)t, (uint32_t)(t >> 32), 0x0Au, 0u};
      oracle_philox(ctr, key, w);
      const int i = (int)(((uint64_t)w[0] * (uint64_t)n) >> 32);
      int nv;
      const int64_t nidx = idx + delta(s, dim, lx, ly, lz, q, i, w[1], &nv);
      if (lo <= nidx && nidx <= hi) {
        const double w_old = mode == 0 ? -lng[idx] : lng[idx];
        const double w_new = mode == 0 ? -lng[nidx] : lng[nidx];
        int ok = w_new >= w_old;
        if (!ok) ok = cm_log(u53(w[2], w[3])) < w_new - w_old;
        if (ok) {
          const int old = s[i];
          s[i] = (int8_t)nv;
          if (q == 0) {
            m += nv - old;
          } else {
            --order[old];
            ++order[nv];
          }
          idx = nidx;
        }
      }
      if (mode == 0) lng[idx] += one_over_t ? n_levels / ((double)(t - t_base) + 1.0) : ln_f;
      ++hist[idx];
    }
    if (mode == 1) {
      idx_out[meas] = idx;
      int64_t o = m;
      if (q != 0) {
        o = 0;
        for (int k = 0; k < q; ++k) o += order[k] * order[k];
      }
      order_out[meas] = o;
    }
  }
  *idx_io = idx;
  *trials = t;
  if (q == 0) order[0] = m;
  return 0;
}

/* Greedy descent into [lo, hi] (critmc flathist.py:96-130 _walk_into_window)
 * with the GPU's stream: step j draws Philox(j mod 2^32, j / 2^32, 0x0C, 0);
 * a move is kept when the level does not move away from the window.  Returns
 * the steps taken, or -1 if max_steps did not reach the window. */
int64_t oracle_fh_descend(int8_t* s, int dim, int lx, int ly, int lz, int q, const uint32_t key[2], int64_t* idx_io,
                          int64_t* order, int lo, int hi, int64_t max_steps) {
  if (dim < 2) ly = 1;
  if (dim < 3) lz = 1;
  const int n = lx * ly * lz;
  int64_t idx = *idx_io;
  for (int64_t j = 0; j <= max_steps; ++j) {
    if (lo <= idx && idx <= hi) {
      *idx_io = idx;
      return j;
    }
    if (j == max_steps) break;
    uint32_t w[4];
    const uint32_t ctr[4] = {(uint32_t)j, (uint32_t)(j >> 32), 0x0Cu, 0u};
    oracle_philox(ctr, key, w);
    const int i = (int)(((uint64_t)w[0] * (uint64_t)n) >> 32);
    int nv;
    const int64_t nidx = idx + delta(s, dim, lx, ly, lz, q, i, w[1], &nv);
    if ((idx < lo && nidx >= idx) || (idx > hi && nidx <= idx)) {
      const int old = s[i];
      s[i] = (int8_t)nv;
      if (q == 0) {
        order[0] += nv - old;
      } else {
        --order[old];
        ++order[nv];
      }
      idx = nidx;
    }
  }
  *idx_io = idx;
  return -1;
}
