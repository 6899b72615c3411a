/*
 * CPU oracle for the byte-lattice kernels (int8 Ising, q-state Potts) --
 * TEST INFRASTRUCTURE ONLY.
 *
 * Restates critmc's numba kernels site by site:
 *   Ising  metropolis/heatbath sweeps  src/critmc/kernels/ising.py:69-107, run :174-237
 *   Potts  metropolis_sweep            src/critmc/kernels/potts.py:45-71
 *          heatbath_sweep              src/critmc/kernels/potts.py:75-103
 *          run (E, counts, aux)        src/critmc/kernels/potts.py:171-235
 * visiting sites colour by colour (colour = (x+y+z)&1).  Each site draws one
 * Philox4x32-10 block per sweep with counter (slot, sweep, 0x02 | colour<<16, 0),
 * slot = (y + ly z) * (lx/2) + x/2:
 *   Ising:  word 0 is the 32-bit uniform compared with thr[class];
 *   Potts Metropolis: word 0 picks the proposal ((w0 (q-1)) >> 32, skipping the
 *     old state), word 1 is the uniform compared with round(2^32 e^{-beta d});
 *   Potts heat bath: u = w0:w1 (64 bits); the state is the first k with
 *     hi64(u * total) < cum_k, weights round(2^52 e^{beta n - max}).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct {
  int dim, lx, ly, lz, z, n;
} BGeo;

static void bgeo(BGeo* g, int dim, int lx, int ly, int lz) {
  g->dim = dim;
  g->lx = lx;
  g->ly = dim >= 2 ? ly : 1;
  g->lz = dim >= 3 ? lz : 1;
  g->z = 2 * dim;
  g->n = g->lx * g->ly * g->lz;
}

/* neighbours of site (x, y, z) in critmc order: +e_a, -e_a per axis */
static void site_nbrs(const BGeo* g, int x, int y, int z, int* nb) {
  int k = 0;
  nb[k++] = ((x + 1) % g->lx) + g->lx * (y + g->ly * z);
  nb[k++] = ((x + g->lx - 1) % g->lx) + g->lx * (y + g->ly * z);
  if (g->dim >= 2) {
    nb[k++] = x + g->lx * (((y + 1) % g->ly) + g->ly * z);
    nb[k++] = x + g->lx * (((y + g->ly - 1) % g->ly) + g->ly * z);
  }
  if (g->dim >= 3) {
    nb[k++] = x + g->lx * (y + g->ly * ((z + 1) % g->lz));
    nb[k++] = x + g->lx * (y + g->ly * ((z + g->lz - 1) % g->lz));
  }
}

static void site_random(const BGeo* g, int x, int y, int z, int col, uint32_t sweep,
                        const uint32_t key[2], uint32_t out[4]) {
  const uint32_t slot = (uint32_t)((y + g->ly * z) * (g->lx / 2) + x / 2);
  const uint32_t ctr[4] = {slot, sweep, 0x02u | ((uint32_t)col << 16), 0u};
  oracle_philox(ctr, key, out);
}

int oracle_ising_byte_run(int8_t* s, int dim, int lx, int ly, int lz, const uint32_t key[2],
                          const uint32_t* tables, uint32_t sweep0, const int64_t* schedule,
                          int n_rows, int n_meas, int64_t* running, int64_t* e_out,
                          int64_t* m_out, int64_t* aux_out) {
  BGeo g;
  bgeo(&g, dim, lx, ly, lz);
  int64_t e_b = running[0], m = running[1];
  uint32_t sweep = sweep0;
  int nb[6];
  for (int meas = 0; meas < n_meas; ++meas) {
    int64_t acc = 0;
    for (int row = 0; row < n_rows; ++row) {
      const int code = (int)schedule[2 * row];
      const uint32_t* kind = tables + (code == 2 ? 32 : 0);
      const uint32_t* thr = kind + 16;
      for (int64_t rep = 0; rep < schedule[2 * row + 1]; ++rep) {
        for (int col = 0; col < 2; ++col)
          for (int z = 0; z < g.lz; ++z)
            for (int y = 0; y < g.ly; ++y)
              for (int x = 0; x < g.lx; ++x) {
                if (((x + y + z) & 1) != col) continue;
                const int i = x + g.lx * (y + g.ly * z);
                site_nbrs(&g, x, y, z, nb);
                int field = 0;
                for (int k = 0; k < g.z; ++k) field += s[nb[k]];
                uint32_t r[4];
                site_random(&g, x, y, z, col, sweep, key, r);
                const int si = s[i];
                if (code == 0) { /* ising.py:75-87 */
                  const int a = si * field, c = 2 * ((g.z - a) / 2) + (si > 0);
                  const int flip = kind[c] == 1 || (kind[c] == 2 && r[0] < thr[c]);
                  if (flip) {
                    s[i] = (int8_t)(-si);
                    e_b += 2 * a;
                    m -= 2 * si;
                    ++acc;
                  }
                } else { /* ising.py:95-106 */
                  const int c = 2 * ((field + g.z) / 2) + (si > 0);
                  const int nw = (kind[c] == 1 || (kind[c] == 2 && r[0] < thr[c])) ? 1 : -1;
                  if (nw != si) {
                    e_b += 2 * si * field;
                    m += 2 * nw;
                    s[i] = (int8_t)nw;
                    ++acc;
                  }
                }
              }
        ++sweep;
      }
    }
    e_out[meas] = e_b;
    m_out[meas] = m;
    aux_out[4 * meas] = acc;
    aux_out[4 * meas + 1] = aux_out[4 * meas + 2] = aux_out[4 * meas + 3] = 0;
  }
  running[0] = e_b;
  running[1] = m;
  return 0;
}

int oracle_potts_tables(int z, double beta, uint64_t* boltz, uint64_t* weight) {
  for (int d = 0; d < 8; ++d) {
    double p = exp(-beta * d); /* potts.py:192-194 */
    if (d == 0 || p >= 1.0) {
      boltz[d] = 1ULL << 32;
    } else {
      double t = nearbyint(ldexp(p, 32));
      boltz[d] = t >= 4294967296.0 ? (1ULL << 32) : (uint64_t)t;
    }
  }
  double mx = -INFINITY;
  for (int n = 0; n <= z; ++n)
    if (beta * n > mx) mx = beta * n;
  for (int n = 0; n < 8; ++n) weight[n] = n <= z ? (uint64_t)nearbyint(ldexp(exp(beta * n - mx), 52)) : 0;
  return 0;
}

int oracle_potts_run(int8_t* s, int dim, int lx, int ly, int lz, int q, const uint32_t key[2],
                     double beta, uint32_t sweep0, const int64_t* schedule, int n_rows, int n_meas,
                     int64_t* energy, int64_t* counts, int64_t* e_out, int64_t* counts_out,
                     int64_t* aux_out) {
  BGeo g;
  bgeo(&g, dim, lx, ly, lz);
  uint64_t boltz[8], weight[8];
  oracle_potts_tables(g.z, beta, boltz, weight);
  int64_t e = *energy;
  uint32_t sweep = sweep0;
  int nb[6], nk[128];
  for (int meas = 0; meas < n_meas; ++meas) {
    int64_t acc = 0;
    for (int row = 0; row < n_rows; ++row) {
      const int code = (int)schedule[2 * row];
      for (int64_t rep = 0; rep < schedule[2 * row + 1]; ++rep) {
        for (int col = 0; col < 2; ++col)
          for (int z = 0; z < g.lz; ++z)
            for (int y = 0; y < g.ly; ++y)
              for (int x = 0; x < g.lx; ++x) {
                if (((x + y + z) & 1) != col) continue;
                const int i = x + g.lx * (y + g.ly * z);
                site_nbrs(&g, x, y, z, nb);
                uint32_t r[4];
                site_random(&g, x, y, z, col, sweep, key, r);
                const int old = s[i];
                if (code == 0) { /* potts.py:52-70 */
                  int nw = (int)(((uint64_t)r[0] * (uint64_t)(q - 1)) >> 32);
                  if (nw >= old) ++nw;
                  int n_old = 0, n_new = 0;
                  for (int k = 0; k < g.z; ++k) {
                    const int v = s[nb[k]];
                    if (v == old) ++n_old;
                    else if (v == nw) ++n_new;
                  }
                  const int delta = n_old - n_new;
                  if (delta <= 0 || (uint64_t)r[1] < boltz[delta]) {
                    s[i] = (int8_t)nw;
                    counts[old] -= 1;
                    counts[nw] += 1;
                    e += delta;
                    ++acc;
                  }
                } else { /* potts.py:80-102 */
                  for (int k = 0; k < q; ++k) nk[k] = 0;
                  for (int c = 0; c < g.z; ++c) nk[s[nb[c]]] += 1;
                  uint64_t total = 0;
                  for (int k = 0; k < q; ++k) total += weight[nk[k]];
                  const uint64_t u = ((uint64_t)r[0] << 32) | r[1];
                  const uint64_t xx = (uint64_t)(((unsigned __int128)u * total) >> 64);
                  int nw = q - 1;
                  uint64_t cum = 0;
                  for (int k = 0; k < q; ++k) {
                    cum += weight[nk[k]];
                    if (xx < cum) {
                      nw = k;
                      break;
                    }
                  }
                  if (nw != old) {
                    e += nk[old] - nk[nw];
                    counts[old] -= 1;
                    counts[nw] += 1;
                    s[i] = (int8_t)nw;
                    ++acc;
                  }
                }
              }
        ++sweep;
      }
    }
    e_out[meas] = e;
    for (int k = 0; k < q; ++k) counts_out[(int64_t)meas * q + k] = counts[k];
    aux_out[4 * meas] = acc;
    aux_out[4 * meas + 1] = aux_out[4 * meas + 2] = aux_out[4 * meas + 3] = 0;
  }
  *energy = e;
  return 0;
}
