/*
 * CPU oracle for the O(n) kernels (XY n = 2, Heisenberg n = 3) -- TEST
 * INFRASTRUCTURE ONLY.
 *
 * Restates critmc's numba O(n) kernels site by site, in single precision like
 * the GPU (critmc works in double):
 *   metropolis_sweep       src/critmc/kernels/on.py:113-137
 *   overrelax_sweep        src/critmc/kernels/on.py:141-183
 *   _von_mises             src/critmc/kernels/on.py:187-204
 *   heatbath_sweep         src/critmc/kernels/on.py:208-261
 *   energy, magnetization,
 *   stiffness_sums,
 *   normalize, run         src/critmc/kernels/on.py:36-87, :349-418
 * Sites are visited colour by colour.  Random words per site and sweep:
 * Philox(slot, sweep, 0x02 | colour << 16, 0) and, for later von Mises rounds
 * (k >= 1) and the Heisenberg Metropolis uniform (k = 0),
 * Philox(slot, sweep, 0x03 | colour << 16, k).  slot = (y + ly z)(lx/2) + x/2.
 * Spins are stored per site as n consecutive floats in critmc's site order.
 * The elementary functions are those of critmc_b200/csrc/fpmath.h (plain IEEE
 * operations, accuracy checked against libm in tests/test_fpmath_cpu.py); with
 * floating-point contraction off on both sides the spins follow the GPU bit for
 * bit.  Observables are sums of per-site FP64 terms rounded to 2^-36 and
 * added as int64, as on the GPU, so they agree exactly.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fpmath.h"
#include "oracle.h"

#define PI_F 3.14159265358979323846f

/* observables: per-site FP64 terms rounded to multiples of 2^-36, summed as int64 */
#define UNFIX36 (1.0 / 68719476736.0)
static int64_t fix36(double x) { return (int64_t)llrint(x * 68719476736.0); }

static float u01(uint32_t w) { return (float)(w >> 8) * (1.0f / 16777216.0f); }
static float u01o(uint32_t w) { return (float)((w >> 8) + 1u) * (1.0f / 16777216.0f); }

static void gauss2(uint32_t a, uint32_t b, float* g0, float* g1) {
  const float rad = sqrtf(-2.0f * cm_logf(u01o(a)));
  const float ang = 2.0f * PI_F * u01(b);
  *g0 = rad * cm_cosf(ang);
  *g1 = rad * cm_sinf(ang);
}

typedef struct {
  int dim, lx, ly, lz, z, n;
} OGeo;

/* neighbours in critmc's column order +x, -x, +y, -y, +z, -z */
static void nbrs(const OGeo* g, int x, int y, int z, int* nb) {
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

/* cos(theta) of a von Mises angle to the field, kappa >= 1e-8 (Best & Fisher 1979) */
static float von_mises_cos(float kappa, const uint32_t r0[4], uint32_t slot, uint32_t sweep,
                           uint32_t col, const uint32_t key[2]) {
  const float root = sqrtf(1.0f + 4.0f * kappa * kappa);
  const float tau = 1.0f + root;
  const float rho = 2.0f * kappa * tau / ((root + 1.0f) * (tau + sqrtf(2.0f * tau)));
  const float r = (1.0f + rho * rho) / (2.0f * rho);
  float f = 1.0f;
  uint32_t a = r0[0], b = r0[1];
  for (int it = 0; it < 64; ++it) {
    if (it > 0) {
      uint32_t ctr[4] = {slot, sweep, 0x03u | (col << 16), (uint32_t)it}, out[4];
      oracle_philox(ctr, key, out);
      a = out[0];
      b = out[1];
    }
    const float zz = cm_cosf(PI_F * u01(a));
    f = (1.0f + r * zz) / (r + zz);
    const float c = kappa * (r - f);
    const float u2 = u01(b);
    if (c * (2.0f - c) - u2 > 0.0f || cm_logf(c / u2) + 1.0f - c >= 0.0f) break;
  }
  return fminf(1.0f, fmaxf(-1.0f, f));
}

static void sweep_colour(float* s, const OGeo* g, int n, int code, int col, uint32_t sweep,
                         float beta, float step, const uint32_t key[2], int64_t* acc) {
  int nb[6];
  for (int z = 0; z < g->lz; ++z)
    for (int y = 0; y < g->ly; ++y)
      for (int x = 0; x < g->lx; ++x) {
        if (((x + y + z) & 1) != col) continue;
        const int i = x + g->lx * (y + g->ly * z);
        const uint32_t slot = (uint32_t)((y + g->ly * z) * (g->lx / 2) + x / 2);
        nbrs(g, x, y, z, nb);
        float h[3] = {0, 0, 0}, sv[3] = {0, 0, 0};
        for (int k = 0; k < n; ++k) {
          float a = 0.0f;
          for (int q = 0; q < g->z; ++q) a += s[(size_t)nb[q] * n + k];
          h[k] = a;
          sv[k] = s[(size_t)i * n + k];
        }
        float* out = s + (size_t)i * n;
        if (code == 5) { /* on.py:160-183 */
          float hh = 0.0f, sh = 0.0f;
          for (int k = 0; k < n; ++k) {
            hh += h[k] * h[k];
            sh += sv[k] * h[k];
          }
          if (hh == 0.0f) continue;
          const float f = 2.0f * sh / hh;
          for (int k = 0; k < n; ++k) out[k] = f * h[k] - sv[k];
          continue;
        }
        uint32_t r0[4];
        {
          uint32_t ctr[4] = {slot, sweep, 0x02u | ((uint32_t)col << 16), 0u};
          oracle_philox(ctr, key, r0);
        }
        if (code == 2) { /* on.py:208-261 */
          float hn = 0.0f;
          for (int k = 0; k < n; ++k) hn += h[k] * h[k];
          hn = sqrtf(hn);
          const float kappa = beta * hn;
          if (n == 2) {
            /* the field direction rotated by the von Mises angle theta (on.py:219-223
               draws atan2(h) + theta; the same spin without forming the angle) */
            if (kappa < 1e-8f) {
              const float phi = PI_F * (2.0f * u01(r0[0]) - 1.0f);
              out[0] = cm_cosf(phi);
              out[1] = cm_sinf(phi);
            } else {
              const float ct = von_mises_cos(kappa, r0, slot, sweep, (uint32_t)col, key);
              float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
              if (!(u01(r0[2]) < 0.5f)) st = -st;
              const float inv = 1.0f / hn;
              const float hx = h[0] * inv, hy = h[1] * inv;
              out[0] = ct * hx - st * hy;
              out[1] = ct * hy + st * hx;
            }
          } else {
            if (hn == 0.0f) {
              float g0, g1, g2, g3;
              gauss2(r0[0], r0[1], &g0, &g1);
              gauss2(r0[2], r0[3], &g2, &g3);
              const float nrm = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
              out[0] = g0 / nrm;
              out[1] = g1 / nrm;
              out[2] = g2 / nrm;
              continue;
            }
            const float rr = u01(r0[0]);
            float u = kappa < 1e-8f ? 2.0f * rr - 1.0f
                                    : 1.0f + cm_logf(rr + (1.0f - rr) * cm_expf(-2.0f * kappa)) / kappa;
            u = fminf(1.0f, fmaxf(-1.0f, u));
            const float hx = h[0] / hn, hy = h[1] / hn, hz = h[2] / hn;
            float ax = 1.0f, ay = 0.0f, az = 0.0f;
            if (!(fabsf(hx) < 0.9f)) {
              ax = 0.0f;
              ay = 1.0f;
            }
            const float proj = ax * hx + ay * hy + az * hz;
            float e1x = ax - proj * hx, e1y = ay - proj * hy, e1z = az - proj * hz;
            const float nrm = sqrtf(e1x * e1x + e1y * e1y + e1z * e1z);
            e1x /= nrm;
            e1y /= nrm;
            e1z /= nrm;
            const float e2x = hy * e1z - hz * e1y, e2y = hz * e1x - hx * e1z, e2z = hx * e1y - hy * e1x;
            const float phi = 2.0f * PI_F * u01(r0[1]);
            const float w = sqrtf(fmaxf(0.0f, 1.0f - u * u));
            const float cp = cm_cosf(phi), sp = cm_sinf(phi);
            out[0] = u * hx + w * (cp * e1x + sp * e2x);
            out[1] = u * hy + w * (cp * e1y + sp * e2y);
            out[2] = u * hz + w * (cp * e1z + sp * e2z);
          }
        } else { /* on.py:113-137 */
          float gv[4];
          gauss2(r0[0], r0[1], &gv[0], &gv[1]);
          uint32_t uacc = r0[2];
          if (n == 3) {
            gauss2(r0[2], r0[3], &gv[2], &gv[3]);
            uint32_t ctr[4] = {slot, sweep, 0x03u | ((uint32_t)col << 16), 0u}, o2[4];
            oracle_philox(ctr, key, o2);
            uacc = o2[0];
          }
          float tr[3], nrm = 0.0f;
          for (int k = 0; k < n; ++k) {
            tr[k] = sv[k] + step * gv[k];
            nrm += tr[k] * tr[k];
          }
          nrm = sqrtf(nrm);
          float d_e = 0.0f;
          for (int k = 0; k < n; ++k) {
            tr[k] /= nrm;
            d_e -= (tr[k] - sv[k]) * h[k];
          }
          if (d_e <= 0.0f || u01(uacc) < cm_expf(-beta * d_e)) {
            for (int k = 0; k < n; ++k) out[k] = tr[k];
            *acc += 1;
          }
        }
      }
}

int oracle_on_run(float* s, int dim, int lx, int ly, int lz, int n, const uint32_t key[2],
                  double beta, double step, uint32_t sweep0, const int64_t* schedule, int n_rows,
                  int n_meas, double* e_out, double* m_out, double* sc_out, double* ss_out,
                  int64_t* aux_out) {
  OGeo g;
  g.dim = dim;
  g.lx = lx;
  g.ly = dim >= 2 ? ly : 1;
  g.lz = dim >= 3 ? lz : 1;
  g.z = 2 * dim;
  g.n = g.lx * g.ly * g.lz;
  uint32_t sweep = sweep0;
  int nb[6];
  for (int meas = 0; meas < n_meas; ++meas) {
    int64_t acc = 0;
    for (int row = 0; row < n_rows; ++row)
      for (int64_t rep = 0; rep < schedule[2 * row + 1]; ++rep) {
        for (int col = 0; col < 2; ++col)
          sweep_colour(s, &g, n, (int)schedule[2 * row], col, sweep, (float)beta, (float)step, key, &acc);
        ++sweep;
      }
    /* normalize (on.py:79-87), then FP64 measurements (on.py:36-76) */
    for (int i = 0; i < g.n; ++i) {
      float nrm = 0.0f;
      for (int k = 0; k < n; ++k) nrm += s[(size_t)i * n + k] * s[(size_t)i * n + k];
      nrm = sqrtf(nrm);
      for (int k = 0; k < n; ++k) s[(size_t)i * n + k] /= nrm;
    }
    /* each site's FP64 term rounded to 2^-36 and summed as int64 (exact) */
    int64_t e = 0, m[3] = {0, 0, 0}, sc[3] = {0, 0, 0}, ss[3] = {0, 0, 0};
    for (int z = 0; z < g.lz; ++z)
      for (int y = 0; y < g.ly; ++y)
        for (int x = 0; x < g.lx; ++x) {
          const int i = x + g.lx * (y + g.ly * z);
          nbrs(&g, x, y, z, nb);
          const float* si = s + (size_t)i * n;
          for (int k = 0; k < n; ++k) m[k] += fix36((double)si[k]);
          for (int a = 0; a < dim; ++a) {
            const float* sj = s + (size_t)nb[2 * a] * n;
            double dot = 0.0;
            for (int k = 0; k < n; ++k) dot += (double)si[k] * (double)sj[k];
            e -= fix36(dot);
            sc[a] += fix36((double)si[0] * sj[0] + (double)si[1] * sj[1]);
            ss[a] += fix36((double)si[0] * sj[1] - (double)si[1] * sj[0]);
          }
        }
    e_out[meas] = (double)e * UNFIX36;
    for (int k = 0; k < n; ++k) m_out[(size_t)meas * n + k] = (double)m[k] * UNFIX36;
    for (int a = 0; a < dim; ++a) {
      sc_out[(size_t)meas * dim + a] = (double)sc[a] * UNFIX36;
      ss_out[(size_t)meas * dim + a] = (double)ss[a] * UNFIX36;
    }
    aux_out[4 * meas] = acc;
    aux_out[4 * meas + 1] = aux_out[4 * meas + 2] = aux_out[4 * meas + 3] = 0;
  }
  return 0;
}
