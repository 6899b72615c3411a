/*
 * CPU oracle for the checkerboard Ising sweeps -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, site by site in plain C, the update rules of critmc's
 * numba Ising kernels:
 *   metropolis_table / metropolis_sweep  src/critmc/kernels/ising.py:48-57, :69-87
 *   heatbath_table / heatbath_sweep      src/critmc/kernels/ising.py:60-65, :91-107
 *   run (schedule executor, E_b/M/aux)   src/critmc/kernels/ising.py:174-237
 *   bond_energy / magnetization          src/critmc/kernels/ising.py:32-45
 * with two deliberate differences that the GPU kernels share:
 *   - sites are visited colour by colour (checkerboard), colour = (x+y+z)&1;
 *   - the uniform of a site is a 32-bit integer u taken from the Philox
 *     plane stream described below, compared with thr = round(p 2^32).
 * It is the bit-exact reference of the device kernels.  Its statistical
 * correctness is pinned separately against critmc's exact results (tests).
 *
 * Random stream of the multi-spin-coded layout: a colour-c site at
 * (x, y, z) has row r = y + ly z, row parity p = (c + y + z) & 1, in-row
 * index i = (x - p) / 2, word w = r * (lx / 64) + i / 32 and lane j = i % 32.
 * Bit (31 - q) of its u is bit j of Philox4x32-10 word (q % 4) of the call
 * with counter (w, sweep, 0x01 | (q / 4) << 8 | c << 16, 0); the optional
 * reduced-round planes use Philox4x32-7 with the same counters.
 *
 * Philox4x32-10 is implemented here independently of the library header,
 * from Salmon et al. (SC'11), and pinned against the Random123 known-answer
 * vectors in the tests.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---------------- Philox4x32-R (R = 10 everywhere; 7 for the optional planes) ---------------- */
void oracle_philox_rounds(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4], int rounds) {
  uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3];
  uint32_t ka = key[0], kb = key[1];
  for (int round = 0; round < rounds; ++round) {
    uint64_t p0 = (uint64_t)0xD2511F53u * x0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ x1 ^ ka;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ x3 ^ kb;
    x1 = (uint32_t)p1;
    x3 = (uint32_t)p0;
    x0 = n0;
    x2 = n2;
    ka += 0x9E3779B9u;
    kb += 0xBB67AE85u;
  }
  out[0] = x0;
  out[1] = x1;
  out[2] = x2;
  out[3] = x3;
}

void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  oracle_philox_rounds(ctr, key, out, 10);
}

/* ---------------- acceptance tables ----------------
 * kind/thr per class c = 2 v + sb (see include/critmc_b200.h).            */
static void table_entry(double p, uint32_t* kind, uint32_t* thr) {
  if (!(p > 0.0)) {
    *kind = 0;
    *thr = 0;
    return;
  }
  if (p >= 1.0) {
    *kind = 1;
    *thr = 0;
    return;
  }
  double t = nearbyint(ldexp(p, 32));
  if (t >= 4294967296.0) {
    *kind = 1;
    *thr = 0;
  } else if (t <= 0.0) {
    *kind = 0;
    *thr = 0;
  } else {
    *kind = 2;
    *thr = (uint32_t)t;
  }
}

int oracle_ising_table(int algo, int z, double beta, double h, uint32_t* kind, uint32_t* thr) {
  for (int c = 0; c < 16; ++c) {
    kind[c] = 0;
    thr[c] = 0;
  }
  for (int v = 0; v <= z; ++v) {
    for (int sb = 0; sb < 2; ++sb) {
      double spin = sb ? 1.0 : -1.0, p;
      if (algo == 0) {
        /* metropolis_table: index a = s_i sum_j s_j; dE = 2a + 2hs */
        double a = (double)(z - 2 * v);
        double d_e = 2.0 * a + 2.0 * h * spin;
        p = d_e <= 0.0 ? 1.0 : exp(-beta * d_e);
      } else if (algo == 2) {
        /* heatbath_table: index sum_j s_j = 2 v - z */
        double field = (double)(2 * v - z);
        p = 1.0 / (1.0 + exp(-2.0 * beta * (field + h)));
      } else {
        return -1;
      }
      table_entry(p, &kind[2 * v + sb], &thr[2 * v + sb]);
    }
  }
  return 0;
}

/* ---------------- geometry ---------------- */
typedef struct {
  int dim, lx, ly, lz, z, n;
  int64_t* nbr; /* (n, z): columns 2a = +e_a, 2a+1 = -e_a (lattice.py:129-134) */
} Geo;

static int geo_init(Geo* g, int dim, int lx, int ly, int lz) {
  g->dim = dim;
  g->lx = lx;
  g->ly = dim >= 2 ? ly : 1;
  g->lz = dim >= 3 ? lz : 1;
  g->z = 2 * dim;
  g->n = g->lx * g->ly * g->lz;
  g->nbr = (int64_t*)malloc(sizeof(int64_t) * (size_t)g->n * g->z);
  if (!g->nbr) return -1;
  int ext[3] = {g->lx, g->ly, g->lz};
  for (int i = 0; i < g->n; ++i) {
    int c[3] = {i % g->lx, (i / g->lx) % g->ly, i / (g->lx * g->ly)};
    for (int a = 0; a < dim; ++a) {
      for (int sgn = 0; sgn < 2; ++sgn) {
        int d[3] = {c[0], c[1], c[2]};
        d[a] = (d[a] + (sgn ? ext[a] - 1 : 1)) % ext[a];
        g->nbr[(size_t)i * g->z + 2 * a + sgn] = d[0] + g->lx * (d[1] + g->ly * d[2]);
      }
    }
  }
  return 0;
}

static void geo_free(Geo* g) { free(g->nbr); }

int64_t oracle_ising_bond_energy(const int8_t* s, int dim, int lx, int ly, int lz) {
  Geo g;
  if (geo_init(&g, dim, lx, ly, lz)) return 0;
  int64_t e = 0;
  for (int i = 0; i < g.n; ++i)
    for (int a = 0; a < dim; ++a) e -= (int64_t)s[i] * s[g.nbr[(size_t)i * g.z + 2 * a]];
  geo_free(&g);
  return e;
}

/* ---------------- MSC-stream checkerboard sweeps ---------------- */
/* Planes of one word, computed four at a time on first use. */
typedef struct {
  uint32_t w, sweep, col;
  int rounds; /* Philox rounds of the planes: 10, or 7 when asked for */
  const uint32_t* key;
  uint32_t planes[32];
  unsigned have; /* bit g set: planes 4g..4g+3 computed */
} PlaneCache;

static uint32_t plane(PlaneCache* pc, int q) {
  const unsigned grp = (unsigned)q >> 2;
  if (!(pc->have & (1u << grp))) {
    uint32_t ctr[4] = {pc->w, pc->sweep, 0x01u | (grp << 8) | (pc->col << 16), 0u}, out[4];
    oracle_philox_rounds(ctr, pc->key, out, pc->rounds);
    for (int k = 0; k < 4; ++k) pc->planes[4 * grp + k] = out[k];
    pc->have |= 1u << grp;
  }
  return pc->planes[q];
}

/* u_j < thr, comparing the bits of u_j (bit 31-q = bit j of plane q) from the top */
static int lane_less(PlaneCache* pc, int j, uint32_t thr) {
  for (int q = 0; q < 32; ++q) {
    const uint32_t ub = (plane(pc, q) >> j) & 1u, tb = (thr >> (31 - q)) & 1u;
    if (ub != tb) return ub < tb;
  }
  return 0; /* u == thr */
}

static int decide(uint32_t kind, uint32_t thr, PlaneCache* pc, int j) {
  if (kind == 1) return 1;
  if (kind == 2) return lane_less(pc, j, thr);
  return 0;
}

/* One checkerboard sweep; accumulates (dE_b, dM, changed) through the pointers. */
static void msc_sweep(int8_t* s, const Geo* g, int algo, const uint32_t* kind, const uint32_t* thr,
                      const uint32_t key[2], uint32_t sweep, int rounds, int64_t* d_eb, int64_t* d_m,
                      int64_t* changed) {
  const int wc = g->lx / 64;
  PlaneCache pc;
  pc.rounds = rounds;
  pc.key = key;
  pc.sweep = sweep;
  for (int col = 0; col < 2; ++col) {
    for (int z = 0; z < g->lz; ++z) {
      for (int y = 0; y < g->ly; ++y) {
        const int p = (col + y + z) & 1;
        const int r = y + g->ly * z;
        for (int k = 0; k < wc; ++k) {
          pc.w = (uint32_t)(r * wc + k);
          pc.col = (uint32_t)col;
          pc.have = 0;
          for (int j = 0; j < 32; ++j) {
            const int x = 2 * (32 * k + j) + p;
            const int i = x + g->lx * (y + g->ly * z);
            /* the 2 dim neighbours +-e_a (lattice.py:129-134), periodic */
            const int xp = x + 1 == g->lx ? 0 : x + 1, xm = x == 0 ? g->lx - 1 : x - 1;
            const int yp = y + 1 == g->ly ? 0 : y + 1, ym = y == 0 ? g->ly - 1 : y - 1;
            int field = s[xp + g->lx * (y + g->ly * z)] + s[xm + g->lx * (y + g->ly * z)] +
                        s[x + g->lx * (yp + g->ly * z)] + s[x + g->lx * (ym + g->ly * z)];
            if (g->dim == 3) {
              const int zp = z + 1 == g->lz ? 0 : z + 1, zm = z == 0 ? g->lz - 1 : z - 1;
              field += s[x + g->lx * (y + g->ly * zp)] + s[x + g->lx * (y + g->ly * zm)];
            }
            const int si = s[i];
            if (algo == 0) {
              const int a = si * field;
              const int v = (g->z - a) / 2, c = 2 * v + (si > 0);
              if (decide(kind[c], thr[c], &pc, j)) {
                s[i] = (int8_t)(-si);
                *d_eb += 2 * a;
                *d_m -= 2 * si;
                *changed += 1;
              }
            } else {
              const int v = (field + g->z) / 2, c = 2 * v + (si > 0);
              const int nw = decide(kind[c], thr[c], &pc, j) ? 1 : -1;
              if (nw != si) {
                *d_eb += 2 * si * field;
                *d_m += 2 * nw;
                s[i] = (int8_t)nw;
                *changed += 1;
              }
            }
          }
        }
      }
    }
  }
}

int oracle_ising_msc_run(int8_t* s, int dim, int lx, int ly, int lz, const uint32_t key[2],
                         const uint32_t* tables, uint32_t sweep0, const int64_t* schedule,
                         int n_rows, int n_meas, int64_t* running, int64_t* e_out, int64_t* m_out,
                         int64_t* aux_out) {
  return oracle_ising_msc_run_rounds(s, dim, lx, ly, lz, key, tables, sweep0, schedule, n_rows, n_meas, running,
                                     e_out, m_out, aux_out, 10);
}

int oracle_ising_msc_run_rounds(int8_t* s, int dim, int lx, int ly, int lz, const uint32_t key[2],
                                const uint32_t* tables, uint32_t sweep0, const int64_t* schedule,
                                int n_rows, int n_meas, int64_t* running, int64_t* e_out, int64_t* m_out,
                                int64_t* aux_out, int rounds) {
  Geo g;
  if (rounds < 1 || rounds > 16) return -1;
  if (dim < 2 || dim > 3 || lx % 64) return -1;
  g.dim = dim;
  g.lx = lx;
  g.ly = ly;
  g.lz = dim == 3 ? lz : 1;
  g.z = 2 * dim;
  g.n = lx * ly * g.lz;
  g.nbr = NULL;
  int64_t e_b = running[0], m = running[1];
  uint32_t sweep = sweep0;
  for (int meas = 0; meas < n_meas; ++meas) {
    int64_t acc = 0;
    for (int row = 0; row < n_rows; ++row) {
      const int code = (int)schedule[2 * row];
      const int algo_slot = code == 2 ? 1 : 0;
      const uint32_t* kind = tables + algo_slot * 32;
      const uint32_t* thr = kind + 16;
      for (int64_t rep = 0; rep < schedule[2 * row + 1]; ++rep) {
        msc_sweep(s, &g, code, kind, thr, key, sweep, rounds, &e_b, &m, &acc);
        ++sweep;
      }
    }
    e_out[meas] = e_b;
    m_out[meas] = m;
    aux_out[4 * meas + 0] = acc;
    aux_out[4 * meas + 1] = 0;
    aux_out[4 * meas + 2] = 0;
    aux_out[4 * meas + 3] = 0;
  }
  running[0] = e_b;
  running[1] = m;
  return 0;
}
