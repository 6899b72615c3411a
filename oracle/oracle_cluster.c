/*
 * CPU oracle for the cluster updates -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates critmc's Wolff and Swendsen-Wang updates
 *   Ising  wolff_update, sw_update   src/critmc/kernels/ising.py:111-171
 *   Potts  wolff/sw                  src/critmc/kernels/potts.py:107-168
 * on the colour-major layout (site u = colour * slots + row * (lx/2) + i), with
 * the GPU's random streams: bond (colour-0 site s, direction q) is active when
 * the ends agree and word q%4 of Philox(s, sweep, 0x07 | (q/4)<<8, 0) is below
 * round(p 2^32); clusters are connected components (sequential union-find, the
 * root of a cluster is its smallest site); Swendsen-Wang draws
 * Philox(root, sweep, 0x08, 0), Wolff Philox(0, sweep, 0x09, 0).  Directions
 * follow the device's neighbour order: same slot, adjacent slot, y-1, y+1,
 * z-1, z+1.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fpmath.h"
#include "oracle.h"

static int find_root(int* parent, int x) {
  int r = x;
  while (parent[r] != r) r = parent[r];
  while (parent[x] != r) {
    const int nx = parent[x];
    parent[x] = r;
    x = nx;
  }
  return r;
}

static void join(int* parent, int a, int b) {
  a = find_root(parent, a);
  b = find_root(parent, b);
  if (a == b) return;
  if (a < b) parent[b] = a;
  else parent[a] = b;
}

/* neighbours (colour-1 slots) of colour-0 slot s */
static void nbrs0(int dim, int lx, int ly, int lz, int s, int* nb) {
  const int hx = lx / 2;
  const int r = s / hx, i = s % hx;
  const int y = dim == 3 ? r % ly : r, z = dim == 3 ? r / ly : 0;
  const int p = (y + z) & 1;
  const int ia = p ? (i == hx - 1 ? 0 : i + 1) : (i == 0 ? hx - 1 : i - 1);
  nb[0] = r * hx + i;
  nb[1] = r * hx + ia;
  if (dim >= 2) {
    const int ym = y == 0 ? ly - 1 : y - 1, yp = y == ly - 1 ? 0 : y + 1;
    nb[2] = (ym + ly * z) * hx + i;
    nb[3] = (yp + ly * z) * hx + i;
  }
  if (dim == 3) {
    const int zm = z == 0 ? lz - 1 : z - 1, zp = z == lz - 1 ? 0 : z + 1;
    nb[4] = (y + ly * zm) * hx + i;
    nb[5] = (y + ly * zp) * hx + i;
  }
}

int oracle_cluster_update(int8_t* lay, int dim, int lx, int ly, int lz, int q, const uint32_t key[2],
                          double beta, int algo, uint32_t sweep, int64_t* d_energy, int64_t* d_mag,
                          int64_t* counts_delta, int64_t stats[3]) {
  if (dim < 2) ly = 1;
  if (dim < 3) lz = 1;
  const int hx = lx / 2, rows = ly * lz, slots = rows * hx, n = 2 * slots, z = 2 * dim;
  const int potts = q > 0;
  const double pb = -expm1(-(potts ? 1.0 : 2.0) * beta);
  const double t = nearbyint(ldexp(pb, 32));
  const uint32_t thr = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
  int* parent = (int*)malloc(sizeof(int) * n);
  int* size = (int*)calloc((size_t)n, sizeof(int));
  int8_t* nv = (int8_t*)malloc((size_t)n);
  if (!parent || !size || !nv) return -1;
  for (int u = 0; u < n; ++u) parent[u] = u;
  int nb[6];
  for (int s = 0; s < slots; ++s) {
    nbrs0(dim, lx, ly, lz, s, nb);
    uint32_t w[8];
    uint32_t ctr[4] = {(uint32_t)s, sweep, 0x07u, 0u};
    oracle_philox(ctr, key, w);
    if (z == 6) {
      ctr[2] = 0x07u | (1u << 8);
      oracle_philox(ctr, key, w + 4);
    }
    for (int k = 0; k < z; ++k) {
      const int u1 = slots + nb[k];
      if (w[k] < thr && lay[u1] == lay[s]) join(parent, s, u1);
    }
  }
  for (int u = 0; u < n; ++u) parent[u] = find_root(parent, u);
  if (algo == 4) stats[1] = stats[2] = 0; /* SW statistics describe this decomposition */
  if (algo == 3) { /* Wolff */
    uint32_t w[4];
    const uint32_t ctr[4] = {0u, sweep, 0x09u, 0u};
    oracle_philox(ctr, key, w);
    const int seed = (int)(((uint64_t)w[0] * (uint64_t)n) >> 32);
    const int root = parent[seed], old = lay[seed];
    const int nvv = potts ? (old + 1 + (int)(((uint64_t)w[1] * (uint64_t)(q - 1)) >> 32)) % q : -old;
    for (int u = 0; u < n; ++u) {
      nv[u] = lay[u];
      if (parent[u] == root) {
        nv[u] = (int8_t)nvv;
        ++stats[0];
      }
    }
  } else { /* Swendsen-Wang */
    for (int u = 0; u < n; ++u) ++size[parent[u]];
    for (int u = 0; u < n; ++u) {
      if (parent[u] == u) {
        stats[1] += (int64_t)size[u] * size[u];
        ++stats[2];
      }
      uint32_t w[4];
      const uint32_t ctr[4] = {(uint32_t)parent[u], sweep, 0x08u, 0u};
      oracle_philox(ctr, key, w);
      nv[u] = potts ? (int8_t)(((uint64_t)w[0] * (uint64_t)q) >> 32) : (int8_t)((w[0] >> 31) ? -lay[u] : lay[u]);
    }
  }
  int64_t de = 0, dm = 0;
  for (int s = 0; s < slots; ++s) {
    nbrs0(dim, lx, ly, lz, s, nb);
    for (int k = 0; k < z; ++k) {
      const int u1 = slots + nb[k];
      if (potts) de += (int64_t)(lay[s] == lay[u1]) - (int64_t)(nv[s] == nv[u1]);
      else de += (int64_t)lay[s] * lay[u1] - (int64_t)nv[s] * nv[u1];
    }
  }
  for (int u = 0; u < n; ++u) {
    if (potts && counts_delta && nv[u] != lay[u]) {
      --counts_delta[lay[u]];
      ++counts_delta[nv[u]];
    }
    if (!potts) dm += nv[u] - lay[u];
    lay[u] = nv[u];
  }
  *d_energy += de;
  if (d_mag) *d_mag += dm;
  free(parent);
  free(size);
  free(nv);
  return 0;
}

/* 24-bit uniform in [0, 1) of a Philox word (the device's critmc_u01f) */
static float u01f(uint32_t a) { return (float)(a >> 8) * (1.0f / 16777216.0f); }

/*
 * O(n) chains: restates critmc's embedded-Ising cluster updates
 *   wolff_update, sw_update   src/critmc/kernels/on.py:265-345
 * with the GPU's streams: axis r from Philox(0, sweep, 0x0B, 0) (XY: angle
 * 2 pi u0; n = 3: z = 2 u0 - 1, angle 2 pi u1), p_i = S_i . r, bond active
 * when p_i p_j > 0 and u01f(word) < 1 - exp(-2 beta p_i p_j), flipped clusters
 * reflected, S <- S - 2 p r.  s: float [ncomp][N], colour-major.  Float
 * arithmetic in the device's order with fpmath.h (built without contraction).
 */
int oracle_on_cluster_update(float* s, int dim, int lx, int ly, int lz, int ncomp, const uint32_t key[2],
                             double beta, int algo, uint32_t sweep, int64_t stats[3]) {
  if (dim < 2) ly = 1;
  if (dim < 3) lz = 1;
  const int hx = lx / 2, rows = ly * lz, slots = rows * hx, n = 2 * slots, z = 2 * dim;
  const float nb2 = (float)(-2.0 * beta);
  float r[3];
  {
    uint32_t w[4];
    const uint32_t ctr[4] = {0u, sweep, 0x0Bu, 0u};
    oracle_philox(ctr, key, w);
    const float two_pi = 6.28318530717958647692f;
    float sn, cs;
    if (ncomp == 2) {
      cm_sincosf(two_pi * u01f(w[0]), &sn, &cs);
      r[0] = cs;
      r[1] = sn;
      r[2] = 0.0f;
    } else {
      const float zc = 2.0f * u01f(w[0]) - 1.0f;
      const float rho = sqrtf(fmaxf(0.0f, 1.0f - zc * zc));
      cm_sincosf(two_pi * u01f(w[1]), &sn, &cs);
      r[0] = rho * cs;
      r[1] = rho * sn;
      r[2] = zc;
    }
  }
  int* parent = (int*)malloc(sizeof(int) * n);
  int* size = (int*)calloc((size_t)n, sizeof(int));
  float* proj = (float*)malloc(sizeof(float) * n);
  int8_t* flip = (int8_t*)calloc((size_t)n, 1);
  if (!parent || !size || !proj || !flip) return -1;
  for (int u = 0; u < n; ++u) {
    parent[u] = u;
    float p = s[u] * r[0] + s[n + u] * r[1];
    if (ncomp == 3) p = p + s[2 * n + u] * r[2];
    proj[u] = p;
  }
  int nb[6];
  for (int q = 0; q < slots; ++q) {
    nbrs0(dim, lx, ly, lz, q, nb);
    uint32_t w[8];
    uint32_t ctr[4] = {(uint32_t)q, sweep, 0x07u, 0u};
    oracle_philox(ctr, key, w);
    if (z == 6) {
      ctr[2] = 0x07u | (1u << 8);
      oracle_philox(ctr, key, w + 4);
    }
    for (int k = 0; k < z; ++k) {
      const int u1 = slots + nb[k];
      const float x = proj[q] * proj[u1];
      if (x > 0.0f && u01f(w[k]) < 1.0f - cm_expf(nb2 * x)) join(parent, q, u1);
    }
  }
  for (int u = 0; u < n; ++u) parent[u] = find_root(parent, u);
  if (algo == 4) stats[1] = stats[2] = 0;
  if (algo == 3) {
    uint32_t w[4];
    const uint32_t ctr[4] = {0u, sweep, 0x09u, 0u};
    oracle_philox(ctr, key, w);
    const int seed = (int)(((uint64_t)w[0] * (uint64_t)n) >> 32);
    for (int u = 0; u < n; ++u)
      if (parent[u] == parent[seed]) {
        flip[u] = 1;
        ++stats[0];
      }
  } else {
    for (int u = 0; u < n; ++u) ++size[parent[u]];
    for (int u = 0; u < n; ++u) {
      if (parent[u] == u) {
        stats[1] += (int64_t)size[u] * size[u];
        ++stats[2];
      }
      uint32_t w[4];
      const uint32_t ctr[4] = {(uint32_t)parent[u], sweep, 0x08u, 0u};
      oracle_philox(ctr, key, w);
      flip[u] = (int8_t)(w[0] >> 31);
    }
  }
  for (int u = 0; u < n; ++u) {
    if (!flip[u]) continue;
    const float tp = 2.0f * proj[u];
    for (int c = 0; c < ncomp; ++c) s[c * n + u] = s[c * n + u] - tp * r[c];
  }
  free(parent);
  free(size);
  free(proj);
  free(flip);
  return 0;
}
