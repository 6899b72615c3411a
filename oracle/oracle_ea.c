/*
 * CPU oracle of the Edwards-Anderson parallel-tempering kernel -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * Restates critmc's pt_run (src/critmc/kernels/glass.py:81-163) with the
 * data layout of the reference: spins[r][c][i] per configuration c in critmc's
 * site order, perm[r][k] = configuration at temperature k, labels[r][c].
 *   sweeps          glass.py:42-53 (checkerboard order here, +-J couplings)
 *   energies        glass.py:34-38 (exact integers for +-J)
 *   swaps           glass.py:128-137 (u < round(2^32 exp(x)) from a table)
 *   labels, trips   glass.py:138-152
 *   measurement     glass.py:57-77, :153-163
 * Random words: configuration at temperature k of set r draws bit k of the
 * plane words of Philox(slot, sweep, 0x01 | grp << 8 | colour << 16, 0) with
 * the key of set r (the MSC plane stream, lane = temperature index); swap k
 * draws word 0 of Philox(k, step, 0x04 | r << 16, 0).
 * q(k_min) is evaluated from per-plane overlap counts S_d[x]:
 * re_d = sum_x cos(2 pi x / L) (2 S_d[x] - N/L), x ascending (same arithmetic
 * as the GPU).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define ORACLE_PI 3.14159265358979323846 /* the value of M_PI */

typedef struct {
  uint32_t w, sweep, col;
  const uint32_t* key;
  uint32_t planes[32];
  unsigned have;
} EPlanes;

static uint32_t eplane(EPlanes* pc, int q) {
  const unsigned grp = (unsigned)q >> 2;
  if (!(pc->have & (1u << grp))) {
    uint32_t ctr[4] = {pc->w, pc->sweep, 0x01u | (grp << 8) | (pc->col << 16), 0u}, out[4];
    oracle_philox(ctr, pc->key, out);
    for (int k = 0; k < 4; ++k) pc->planes[4 * grp + k] = out[k];
    pc->have |= 1u << grp;
  }
  return pc->planes[q];
}

static int elane_less(EPlanes* pc, int j, uint32_t thr) {
  for (int q = 0; q < 32; ++q) {
    const uint32_t ub = (eplane(pc, q) >> j) & 1u, tb = (thr >> (31 - q)) & 1u;
    if (ub != tb) return ub < tb;
  }
  return 0;
}

typedef struct {
  int dim, lx, ly, lz, z, n;
} EGeo;

static int esite(const EGeo* g, int x, int y, int z) {
  x = (x + g->lx) % g->lx;
  y = (y + g->ly) % g->ly;
  z = (z + g->lz) % g->lz;
  return x + g->lx * (y + g->ly * z);
}

/* neighbour j of site (x,y,z) in direction a with sign, and the bond coupling */
static void enbr(const EGeo* g, const double* J, int x, int y, int z, int a, int sgn, int* j, double* jj) {
  int d[3] = {0, 0, 0};
  d[a] = sgn;
  const int me = esite(g, x, y, z);
  *j = esite(g, x + d[0], y + d[1], z + d[2]);
  /* bond a*N + i is (i, i + e_a) (critmc lattice.py:147-149) */
  *jj = sgn > 0 ? J[(size_t)a * g->n + me] : J[(size_t)a * g->n + *j];
}

int oracle_ea_pt_run(int8_t* spins, const double* J, int dim, int lx, int ly, int lz, int m,
                     const uint32_t* keys, const double* betas, const uint32_t* swap_thr, int width,
                     int* perm, int* labels, uint32_t t0, int n_steps, int n_bins,
                     int sweeps_per_step, double* acc, int64_t* swap_acc, int64_t* swap_try,
                     int64_t* label_hist, int64_t* trips) {
  EGeo g;
  g.dim = dim;
  g.lx = lx;
  g.ly = ly;
  g.lz = dim == 3 ? lz : 1;
  g.z = 2 * dim;
  g.n = lx * g.ly * g.lz;
  const int n = g.n, hx = lx / 2;
  const long long n_bonds = (long long)n * dim;
  /* Metropolis thresholds per temperature and unsatisfied-bond count v < z/2 */
  uint32_t thr[32][4];
  for (int k = 0; k < m; ++k)
    for (int v = 0; v < g.z / 2; ++v) {
      const double p = exp(-betas[k] * (2.0 * g.z - 4.0 * v));
      const double t = nearbyint(ldexp(p, 32));
      thr[k][v] = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
    }
  double cosx[64], sinx[64];
  for (int x = 0; x < lx; ++x) {
    cosx[x] = cos(2.0 * ORACLE_PI * x / lx);
    sinx[x] = sin(2.0 * ORACLE_PI * x / lx);
  }
  long long *energy = (long long*)malloc(sizeof(long long) * 2 * m);
  int* q = (int*)malloc(sizeof(int) * n);
  int b = 0;
  long long next_edge = 1;
  for (int t = 0; t < n_steps; ++t) {
    if (t >= next_edge) {
      ++b;
      next_edge = (1LL << (b + 1)) - 1;
    }
    const uint32_t step = t0 + (uint32_t)t;
    for (int r = 0; r < 2; ++r) {
      const uint32_t* key = keys + 2 * r;
      for (int sw = 0; sw < sweeps_per_step; ++sw) {
        const uint32_t sweep = step * (uint32_t)sweeps_per_step + (uint32_t)sw;
        for (int col = 0; col < 2; ++col)
          for (int z = 0; z < g.lz; ++z)
            for (int y = 0; y < g.ly; ++y) {
              const int p = (col + y + z) & 1;
              for (int i = 0; i < hx; ++i) {
                const int x = 2 * i + p;
                EPlanes pc;
                pc.w = (uint32_t)((y + g.ly * z) * hx + i);
                pc.sweep = sweep;
                pc.col = (uint32_t)col;
                pc.key = key;
                pc.have = 0;
                const int me = esite(&g, x, y, z);
                for (int k = 0; k < m; ++k) {
                  int8_t* s = spins + ((size_t)r * m + perm[r * m + k]) * n;
                  int unsat = 0;
                  for (int a = 0; a < dim; ++a)
                    for (int sgn = -1; sgn <= 1; sgn += 2) {
                      int j;
                      double jj;
                      enbr(&g, J, x, y, z, a, sgn, &j, &jj);
                      if (jj * s[me] * s[j] < 0) ++unsat;
                    }
                  /* dE = 2 s_i h_i = 2z - 4 unsat; accept if dE <= 0 or u < e^{-beta dE} */
                  const int flip = 2 * unsat >= g.z || elane_less(&pc, k, thr[k][unsat]);
                  if (flip) s[me] = (int8_t)(-s[me]);
                }
              }
            }
      }
      /* energies of all configurations of set r */
      for (int c = 0; c < m; ++c) {
        const int8_t* s = spins + ((size_t)r * m + c) * n;
        long long e = 0;
        for (int z = 0; z < g.lz; ++z)
          for (int y = 0; y < g.ly; ++y)
            for (int x = 0; x < lx; ++x)
              for (int a = 0; a < dim; ++a) {
                int j;
                double jj;
                enbr(&g, J, x, y, z, a, +1, &j, &jj);
                e -= (long long)(jj * s[esite(&g, x, y, z)] * s[j]);
              }
        energy[r * m + c] = e;
      }
      for (int k = 0; k + 1 < m; ++k) {
        const int c1 = perm[r * m + k], c2 = perm[r * m + k + 1];
        const long long de = energy[r * m + c1] - energy[r * m + c2];
        int ok = de <= 0; /* x = (b_k - b_k+1)(E_c1 - E_c2) >= 0 */
        if (!ok) {
          long long jd = de / 4;
          if (jd > width - 1) jd = width - 1;
          uint32_t ctr[4] = {(uint32_t)k, step, 0x04u | ((uint32_t)r << 16), 0u}, out[4];
          oracle_philox(ctr, key, out);
          ok = out[0] < swap_thr[(size_t)k * width + jd];
        }
        swap_try[k] += 1;
        if (ok) {
          perm[r * m + k] = c2;
          perm[r * m + k + 1] = c1;
          swap_acc[k] += 1;
        }
      }
      const int hot = perm[r * m], cold = perm[r * m + m - 1];
      if (labels[r * m + hot] == 2) trips[r] += 1;
      labels[r * m + hot] = 1;
      if (labels[r * m + cold] == 1) trips[r] += 1;
      labels[r * m + cold] = 2;
      for (int k = 0; k < m; ++k) {
        const int l = labels[r * m + perm[r * m + k]];
        if (l == 1) label_hist[2 * k] += 1;
        else if (l == 2) label_hist[2 * k + 1] += 1;
      }
    }
    /* measurement at every temperature */
    for (int k = 0; k < m; ++k) {
      const int ca = perm[k], cb = perm[m + k];
      const int8_t* sa = spins + (size_t)ca * n;
      const int8_t* sb = spins + ((size_t)m + cb) * n;
      long long qs = 0, ql = 0;
      for (int i = 0; i < n; ++i) {
        q[i] = sa[i] * sb[i];
        qs += q[i];
      }
      for (int z = 0; z < g.lz; ++z)
        for (int y = 0; y < g.ly; ++y)
          for (int x = 0; x < lx; ++x)
            for (int a = 0; a < dim; ++a) {
              int j;
              double jj;
              enbr(&g, J, x, y, z, a, +1, &j, &jj);
              ql += q[esite(&g, x, y, z)] * q[j];
            }
      const double nn = (double)n, nb = (double)n_bonds;
      const double qv = (double)qs / nn;
      double qk2 = 0.0;
      const int ext[3] = {lx, g.ly, g.lz};
      for (int d = 0; d < dim; ++d) {
        const double per = nn / ext[d];
        double re = 0.0, im = 0.0;
        for (int x = 0; x < ext[d]; ++x) {
          long long cnt = 0; /* sites with coordinate d equal to x and q_i = +1 */
          for (int i = 0; i < n; ++i) {
            const int cx[3] = {i % lx, (i / lx) % g.ly, i / (lx * g.ly)};
            if (cx[d] == x && q[i] > 0) ++cnt;
          }
          const double sx = 2.0 * (double)cnt - per;
          re += cosx[x] * sx;
          im += sinx[x] * sx;
        }
        qk2 += (re * re + im * im) / (nn * nn);
      }
      qk2 /= dim;
      double* a = acc + ((size_t)b * m + k) * 7;
      a[0] += 0.5 * (double)(energy[ca] + energy[m + cb]) / nn;
      a[1] += (double)ql / nb;
      a[2] += fabs(qv);
      a[3] += qv * qv;
      a[4] += qv * qv * qv * qv;
      a[5] += qk2;
      a[6] += 1.0;
    }
  }
  free(energy);
  free(q);
  return 0;
}
