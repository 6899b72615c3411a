// O(n) vector models (XY n = 2, Heisenberg n = 3) with FP32 unit spins:
// checkerboard heat bath (von Mises / exponential-in-cos), over-relaxation and
// Gaussian-step Metropolis.  Two lanes with identical results: one thread
// block per chain running the whole schedule (lattice in shared memory when
// it fits), or many blocks per chain with one launch per colour (large
// lattices, latency), replayed as CUDA graphs.  Per-measurement energy,
// magnetisation and stiffness sums are exact 64-bit fixed-point sums of FP64
// per-site terms.  The elementary functions come from fpmath.h and this file
// is compiled without floating-point contraction, so a CPU replay follows the
// spins and the sums bit for bit.
//
// Replaces critmc src/critmc/kernels/on.py:349-418 (`run`), :113-137
// (`metropolis_sweep`), :141-183 (`overrelax_sweep`), :187-261
// (`_von_mises`, `heatbath_sweep`), :36-87 (measurements, `normalize`).
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "fpmath.h"
#include "geom.cuh"
#include "host_common.h"

namespace critmc {

constexpr int ON_PCHAINS = 1024;
constexpr int ON_MAX_GROUPS = 16;
constexpr int ON_MAX_ROWS = 8;
constexpr int ON_SMEM_MAX = 200 * 1024;
constexpr int ON_MAX_VM_ITER = 64;  // von Mises rejection rounds (acceptance > 0.65 each)

struct OnParams {
  float* spins;
  double* e_out;
  double* m_out;
  double* sc_out;
  double* ss_out;
  long long* aux_out;
  ByteGeom g;
  int n_chains, chain0, chains_per_group, n_meas, n_rows;
  int codes[ON_MAX_ROWS];
  int reps[ON_MAX_ROWS];
  int resident;
  uint32_t sweep0;
  float beta[ON_MAX_GROUPS];
  float step[ON_MAX_GROUPS];
  uint32_t keys[ON_PCHAINS][2];
};

constexpr float ON_PI = 3.14159265358979323846f;

// uniform in [0, 1) and in (0, 1] from 24 random bits
__device__ __forceinline__ float u01(uint32_t w) { return critmc_u01f(w); }
__device__ __forceinline__ float u01o(uint32_t w) { return critmc_u01f_open0(w); }

// Box-Muller pair of standard normals
__device__ __forceinline__ void gauss2(uint32_t a, uint32_t b, float& g0, float& g1) {
  const float rad = sqrtf(-2.0f * cm_logf(u01o(a)));
  float sn, cs;
  cm_sincosf(2.0f * ON_PI * u01(b), &sn, &cs);
  g0 = rad * cs;
  g1 = rad * sn;
}

// neighbour slots in critmc's column order (+x, -x, +y, -y, +z, -z) of the
// site at (r, i) of row (y, z)
template <int Z>
__device__ __forceinline__ void on_neighbours_at(const ByteGeom& g, int c, int r, int i, int y, int z,
                                                 uint32_t* nb) {
  uint32_t raw[Z];
  byte_neighbours_at<Z>(g, c, r, i, y, z, raw);
  const int p = (c + y + z) & 1;
  nb[0] = p ? raw[1] : raw[0];  // +x
  nb[1] = p ? raw[0] : raw[1];  // -x
  if constexpr (Z >= 4) {
    nb[2] = raw[3];  // +y
    nb[3] = raw[2];  // -y
  }
  if constexpr (Z == 6) {
    nb[4] = raw[5];  // +z
    nb[5] = raw[4];  // -z
  }
}

template <int Z>
__device__ __forceinline__ void on_neighbours(const ByteGeom& g, int c, uint32_t s, uint32_t* nb,
                                              int& y, int& z) {
  int r, i;
  byte_row_index(g, s, r, i);
  y = r;
  z = 0;
  if constexpr (Z == 6) {
    y = r % g.ly;
    z = r / g.ly;
  }
  on_neighbours_at<Z>(g, c, r, i, y, z, nb);
}

// Best & Fisher (1979) von Mises sampler, critmc kernels/on.py:187-204, returning
// cos(theta) of the angle theta to the local field (kappa >= 1e-8).  At most
// ON_MAX_VM_ITER rounds; with a per-round acceptance above 0.65 the bound is
// reached with probability below 1e-29, and then the last proposal is kept.
__device__ __forceinline__ float von_mises_cos(float kappa, const critmc_u32x4& r0, uint32_t slot,
                                               uint32_t sweep, uint32_t col, uint32_t k0, uint32_t k1) {
  const float root = sqrtf(1.0f + 4.0f * kappa * kappa);
  const float tau = 1.0f + root;
  const float rho = 2.0f * kappa * tau / ((root + 1.0f) * (tau + sqrtf(2.0f * tau)));
  const float r = (1.0f + rho * rho) / (2.0f * rho);
  float f = 1.0f;
  uint32_t a = r0.v[0], b = r0.v[1];
  for (int it = 0; it < ON_MAX_VM_ITER; ++it) {
    if (it > 0) {
      const critmc_u32x4 x =
          critmc_philox4x32(slot, sweep, CRITMC_TAG_SITE2 | (col << 16), (uint32_t)it, k0, k1);
      a = x.v[0];
      b = x.v[1];
    }
    const float zz = cm_cosf(ON_PI * u01(a));
    f = (1.0f + r * zz) / (r + zz);
    const float c = kappa * (r - f);
    const float u2 = u01(b);
    if (c * (2.0f - c) - u2 > 0.0f || cm_logf(c / u2) + 1.0f - c >= 0.0f) break;
  }
  return fminf(1.0f, fmaxf(-1.0f, f));
}

// Observables are sums of per-site terms, each rounded to a multiple of
// 2^-36 and added as 64-bit integers: exact and independent of how the sites
// are split over threads and blocks (the CPU replay gets the same totals).
constexpr double ON_FIX = 68719476736.0;  // 2^36
constexpr double ON_UNFIX = 1.0 / 68719476736.0;
// round(x 2^36) to nearest even, as llrint does: for |x 2^36| < 2^51, adding
// 1.5 2^52 leaves the rounded integer in the low mantissa bits (one add and an
// integer subtract instead of a conversion instruction).  The terms here are
// dot products and components of unit vectors, |x| <= 3.
constexpr double ON_ROUND_MAGIC = 6755399441055744.0;  // 1.5 * 2^52
__device__ __forceinline__ long long on_fix(double x) {
  const double t = __dadd_rn(x * ON_FIX, ON_ROUND_MAGIC);
  return __double_as_longlong(t) - __double_as_longlong(ON_ROUND_MAGIC);
}

// number of sums per measurement: energy, M[N], stiffness cos/sin [dim], accepted moves
template <int N, int Z>
constexpr int on_nv() { return 2 + N + Z; }

// One update of site s of colour c (one of the three moves); returns 1 for an
// accepted Metropolis move.  lat holds comp[n][colour][slot].
template <int N, int Z>
__device__ __forceinline__ int on_site_nb(float* lat, const ByteGeom& g, int c, uint32_t s, const uint32_t* nb,
                                          int code, uint32_t sweep, float beta, float step, uint32_t k0,
                                          uint32_t k1) {
  float* own[N];
  const float* oth[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    own[k] = lat + ((size_t)k * 2 + c) * g.slots;
    oth[k] = lat + ((size_t)k * 2 + (c ^ 1)) * g.slots;
  }
  float h[N], sv[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    float acc = 0.0f;
#pragma unroll
    for (int q = 0; q < Z; ++q) acc += oth[k][CRITMC_IDX(nb[q], g.slots)];
    h[k] = acc;
    sv[k] = own[k][CRITMC_IDX(s, g.slots)];
  }
  if (code == CRITMC_OVERRELAX) {
    // on.py:141-183: reflect about the local field; keep the spin if h = 0
    float hh = 0.0f, sh = 0.0f;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      hh += h[k] * h[k];
      sh += sv[k] * h[k];
    }
    if (hh != 0.0f) {
      const float f = 2.0f * sh / hh;
#pragma unroll
      for (int k = 0; k < N; ++k) own[k][s] = f * h[k] - sv[k];
    }
    return 0;
  }
  const critmc_u32x4 r0 = critmc_philox4x32(s, sweep, CRITMC_TAG_SITE | ((uint32_t)c << 16), 0u, k0, k1);
  if (code == CRITMC_HEATBATH) {
    float hn = 0.0f;
#pragma unroll
    for (int k = 0; k < N; ++k) hn += h[k] * h[k];
    hn = sqrtf(hn);
    const float kappa = beta * hn;
    if constexpr (N == 2) {
      // new spin = rotation of the field direction by theta (sign from word 2);
      // the same as angle atan2(h) + theta, without the angle
      if (kappa < 1e-8f) {
        float sn, cs;
        cm_sincosf(ON_PI * (2.0f * u01(r0.v[0]) - 1.0f), &sn, &cs);
        own[0][s] = cs;
        own[1][s] = sn;
      } else {
        const float ct = von_mises_cos(kappa, r0, s, sweep, (uint32_t)c, k0, k1);
        float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        if (!(u01(r0.v[2]) < 0.5f)) st = -st;
        const float inv = 1.0f / hn;
        const float hx = h[0] * inv, hy = h[1] * inv;
        own[0][s] = ct * hx - st * hy;
        own[1][s] = ct * hy + st * hx;
      }
    } else {
      if (hn == 0.0f) {
        float g0, g1, g2, g3;
        gauss2(r0.v[0], r0.v[1], g0, g1);
        gauss2(r0.v[2], r0.v[3], g2, g3);
        const float nrm = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
        own[0][s] = g0 / nrm;
        own[1][s] = g1 / nrm;
        own[2][s] = g2 / nrm;
        return 0;
      }
      const float rr = u01(r0.v[0]);
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
      const float phi = 2.0f * ON_PI * u01(r0.v[1]);
      const float w = sqrtf(fmaxf(0.0f, 1.0f - u * u));
      float sp, cp;
      cm_sincosf(phi, &sp, &cp);
      own[0][s] = u * hx + w * (cp * e1x + sp * e2x);
      own[1][s] = u * hy + w * (cp * e1y + sp * e2y);
      own[2][s] = u * hz + w * (cp * e1z + sp * e2z);
    }
    return 0;
  }
  // on.py:113-137: Gaussian step, renormalise, accept exp(-beta dE)
  float gv[4];
  gauss2(r0.v[0], r0.v[1], gv[0], gv[1]);
  uint32_t uacc = r0.v[2];
  if constexpr (N == 3) {
    gauss2(r0.v[2], r0.v[3], gv[2], gv[3]);
    uacc = critmc_philox4x32(s, sweep, CRITMC_TAG_SITE2 | ((uint32_t)c << 16), 0u, k0, k1).v[0];
  }
  float tr[N], nrm = 0.0f;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    tr[k] = sv[k] + step * gv[k];
    nrm += tr[k] * tr[k];
  }
  nrm = sqrtf(nrm);
  float d_e = 0.0f;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    tr[k] /= nrm;
    d_e -= (tr[k] - sv[k]) * h[k];
  }
  if (d_e <= 0.0f || u01(uacc) < cm_expf(-beta * d_e)) {
#pragma unroll
    for (int k = 0; k < N; ++k) own[k][s] = tr[k];
    return 1;
  }
  return 0;
}

template <int N, int Z>
__device__ __forceinline__ int on_site(float* lat, const ByteGeom& g, int c, uint32_t s, int code,
                                       uint32_t sweep, float beta, float step, uint32_t k0, uint32_t k1) {
  uint32_t nb[Z];
  int y, z;
  on_neighbours<Z>(g, c, s, nb, y, z);
  return on_site_nb<N, Z>(lat, g, c, s, nb, code, sweep, beta, step, k0, k1);
}

// on.py:79-87: rescale site j (of 2 slots) to unit length
template <int N>
__device__ __forceinline__ void on_normalize_site(float* lat, size_t n_sites, uint32_t j) {
  float v[N], nrm = 0.0f;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    v[k] = lat[(size_t)k * n_sites + j];
    nrm += v[k] * v[k];
  }
  nrm = sqrtf(nrm);
#pragma unroll
  for (int k = 0; k < N; ++k) lat[(size_t)k * n_sites + j] = v[k] / nrm;
}

// on.py:36-76: add site j's terms (forward bonds) to v[0] energy, v[1..N] M,
// v[1+N+a] stiffness cos, v[1+N+DIM+a] stiffness sin sums
template <int N, int Z>
__device__ __forceinline__ void on_measure_site_nb(const float* lat, const ByteGeom& g, int c, uint32_t s,
                                                   const uint32_t* nb, long long* v) {
  constexpr int DIM = Z / 2;
  double si[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    si[k] = lat[((size_t)k * 2 + c) * g.slots + s];
    v[1 + k] += on_fix(si[k]);
  }
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    double sj[N];
#pragma unroll
    for (int k = 0; k < N; ++k) sj[k] = lat[((size_t)k * 2 + (c ^ 1)) * g.slots + nb[2 * a]];
    double dot = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) dot += si[k] * sj[k];
    v[0] -= on_fix(dot);
    v[1 + N + a] += on_fix(si[0] * sj[0] + si[1] * sj[1]);
    v[1 + N + DIM + a] += on_fix(si[0] * sj[1] - si[1] * sj[0]);
  }
}

template <int N, int Z>
__device__ __forceinline__ void on_measure_site(const float* lat, const ByteGeom& g, uint32_t j, long long* v) {
  const int c = j >= g.slots;
  const uint32_t s = j - c * g.slots;
  uint32_t nb[Z];
  int y, z;
  on_neighbours<Z>(g, c, s, nb, y, z);
  on_measure_site_nb<N, Z>(lat, g, c, s, nb, v);
}

// sum q (of on_nv) of measurement meas, converted back to doubles
template <int N, int Z>
__device__ __forceinline__ void on_write_sum(double* e_out, double* m_out, double* sc_out, double* ss_out,
                                             long long* aux_out, int meas, int q, long long total) {
  constexpr int DIM = Z / 2;
  const size_t o = (size_t)meas;
  const double x = (double)total * ON_UNFIX;
  if (q == 0) {
    e_out[o] = x;
  } else if (q <= N) {
    m_out[o * N + (q - 1)] = x;
  } else if (q <= N + DIM) {
    sc_out[o * DIM + (q - 1 - N)] = x;
  } else if (q <= N + 2 * DIM) {
    ss_out[o * DIM + (q - 1 - N - DIM)] = x;
  } else {
    aux_out[4 * o + 0] = total;
    aux_out[4 * o + 1] = 0;
    aux_out[4 * o + 2] = 0;
    aux_out[4 * o + 3] = 0;
  }
}

// Everything one thread block needs to advance one O(n) chain.
struct OnChain {
  const RunCtl* ctl = nullptr;  // bounded run (work items), polled between measurements
  CtlPoll* poll = nullptr;
  float* gl;          // the chain's spins in HBM
  double* e_out;      // [n_meas]
  double* m_out;      // [n_meas][N]
  double* sc_out;     // [n_meas][dim]
  double* ss_out;     // [n_meas][dim]
  long long* aux_out; // [n_meas][4]
  ByteGeom g;
  int n_meas, n_rows, resident;
  int nt;  // threads that own sites (a multiple of 32)
  const int* codes;
  const int* reps;
  uint32_t sweep0, k0, k1;
  float beta, step;
};

// Threads owning sites for a chain of `slots` sites per colour (the per-chain
// launch uses exactly this many; larger blocks leave the rest idle).
constexpr int ON_THREADS = 1024;
__host__ __device__ inline int on_site_threads(uint32_t slots) {
  const uint32_t t = ((slots + 31) / 32) * 32;
  return (int)(t < 32 ? 32 : (t > (uint32_t)ON_THREADS ? (uint32_t)ON_THREADS : t));
}

// CL == 1: one block, the lattice in shared memory when P.resident.  CL > 1: a
// cluster of CL blocks splits every site loop, the lattice stays in global
// memory (L2-resident at the sizes that use teams), the cluster barrier
// separates the colours, and the blocks' partial sums meet in block 0's
// shared memory.  The site order within a colour does not matter (a colour's
// sites are independent) and the sums are integers, so every CL gives the
// same spins and series.  Block 0's thread 0 alone polls the control and
// passes its answer to all blocks before the barrier that ends a
// measurement, so the whole team stops at the same measurement.
template <int N, int Z, int CL = 1>
__device__ void on_chain_run(const OnChain& P, unsigned char* smem_raw) {
  using T = Team<CL>;
  constexpr int NV = on_nv<N, Z>();
  __shared__ long long red[NV][ON_THREADS / 32];
  __shared__ long long part[CL > 1 ? 2 : 1][CL][NV];  // team: block totals by measurement parity
  __shared__ int s_stop[2];
  const ByteGeom& g = P.g;
  const size_t n_sites = 2 * (size_t)g.slots;
  float* gl = P.gl;
  const bool resident = CL == 1 && P.resident;
  float* lat = resident ? reinterpret_cast<float*>(smem_raw) : gl;
  const int tid = threadIdx.x;
  const unsigned rank = T::rank();
  // one block: idle threads (tid >= nt) start every site loop past its end but
  // take part in the barriers; a team: every thread owns sites
  const uint32_t nt = CL == 1 ? (uint32_t)P.nt : (uint32_t)(CL * blockDim.x);
  const uint32_t t0 = CL == 1 ? (tid < P.nt ? (uint32_t)tid : 0x7fffffffu) : rank * blockDim.x + tid;
  if (resident)
    for (size_t j = t0; j < N * n_sites; j += nt) lat[j] = gl[j];
  if (CL > 1 && tid == 0) s_stop[0] = 0;
  T::sync();
  uint32_t sweep = P.sweep0;

  for (int meas = 0; meas < P.n_meas; ++meas) {
    if constexpr (CL == 1) {
      if (P.ctl) {  // stop between measurements when the budget or a cancel says so
        if (tid == 0) s_stop[0] = P.poll->check(*P.ctl);
        __syncthreads();
        if (s_stop[0]) break;
      }
    } else {
      if (s_stop[meas & 1]) break;  // block 0's answer, written before the last barrier
    }
    long long nacc = 0;
    for (int row = 0; row < P.n_rows; ++row) {
      const int code = P.codes[row];
      for (int rep = 0; rep < P.reps[row]; ++rep) {
        for (int c = 0; c < 2; ++c) {
          SiteCursor cur;
          for (cur.init(g, t0, nt); cur.s < g.slots; cur.next(g)) {
            uint32_t nb[Z];
            on_neighbours_at<Z>(g, c, cur.r, cur.i, cur.y, cur.z, nb);
            nacc += on_site_nb<N, Z>(lat, g, c, cur.s, nb, code, sweep, P.beta, P.step, P.k0, P.k1);
          }
          T::sync();
        }
        ++sweep;
      }
    }
    for (uint32_t j = t0; j < n_sites; j += nt) on_normalize_site<N>(lat, n_sites, j);
    T::sync();
    long long v[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = 0;
    for (int c = 0; c < 2; ++c) {
      SiteCursor cur;
      for (cur.init(g, t0, nt); cur.s < g.slots; cur.next(g)) {
        uint32_t nb[Z];
        on_neighbours_at<Z>(g, c, cur.r, cur.i, cur.y, cur.z, nb);
        on_measure_site_nb<N, Z>(lat, g, c, cur.s, nb, v);
      }
    }
    v[NV - 1] = nacc;
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const long long w = warp_sum(v[q]);
      if (lane == 0) red[q][warp] = w;
    }
    __syncthreads();
    long long total = 0;
    if (tid < NV)
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += red[tid][w];
    if constexpr (CL == 1) {
      if (tid < NV) on_write_sum<N, Z>(P.e_out, P.m_out, P.sc_out, P.ss_out, P.aux_out, meas, tid, total);
    } else {
      if (tid < NV) *T::at(&part[meas & 1][rank][tid], 0) = total;
      if (rank == 0 && tid == 0) {
        const int stop = P.ctl ? P.poll->check(*P.ctl) : 0;
        for (int r = 0; r < CL; ++r) *T::at(&s_stop[(meas + 1) & 1], (unsigned)r) = stop;
      }
    }
    T::sync();
    if constexpr (CL > 1) {
      // block 0 adds the totals; part[meas & 1] is next written two measurements
      // on, after barriers that block 0 only passes once it is done here
      if (rank == 0 && tid < NV) {
        long long sum = 0;
        for (int r = 0; r < CL; ++r) sum += part[meas & 1][r][tid];
        on_write_sum<N, Z>(P.e_out, P.m_out, P.sc_out, P.ss_out, P.aux_out, meas, tid, sum);
      }
    }
  }
  if (resident)
    for (size_t j = t0; j < N * n_sites; j += nt) gl[j] = lat[j];
  T::sync();
}

template <int N, int Z>
__global__ void __launch_bounds__(ON_THREADS) on_run_kernel(const __grid_constant__ OnParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lchain = blockIdx.x;
  const int chain = P.chain0 + lchain;
  const int group = chain / P.chains_per_group;
  constexpr int DIM = Z / 2;
  OnChain a;
  a.g = P.g;
  a.gl = P.spins + (size_t)chain * N * 2 * P.g.slots;
  a.e_out = P.e_out + (size_t)chain * P.n_meas;
  a.m_out = P.m_out + (size_t)chain * P.n_meas * N;
  a.sc_out = P.sc_out + (size_t)chain * P.n_meas * DIM;
  a.ss_out = P.ss_out + (size_t)chain * P.n_meas * DIM;
  a.aux_out = P.aux_out + (size_t)chain * P.n_meas * 4;
  a.n_meas = P.n_meas;
  a.n_rows = P.n_rows;
  a.resident = P.resident;
  a.nt = blockDim.x;
  a.codes = P.codes;
  a.reps = P.reps;
  a.sweep0 = P.sweep0;
  a.k0 = P.keys[lchain][0];
  a.k1 = P.keys[lchain][1];
  a.beta = P.beta[group];
  a.step = P.step[group];
  on_chain_run<N, Z>(a, smem_raw);
}

// ---------------------------------------------------------------------------
// Multi-block lane: one launch per colour of each sweep, then a normalisation
// and a measurement launch per measurement; sums go to int64 accumulators
// acc[chain][meas][NV] with atomics (exact, so the order does not matter).
// ---------------------------------------------------------------------------
constexpr int ON_GRID_THREADS = 256;
constexpr int ON_GPCHAINS = 256;

struct OnGridParams {
  float* spins;
  unsigned long long* acc;  // [n_meas][n_chains][NV]
  const uint32_t* cursor;   // device (sweep base, meas base) for graph replay, or null
  ByteGeom g;
  int n_chains, chain0, chains_per_group, nv;
  int code, col;
  uint32_t sweep, meas;     // absolute, or relative to the cursor
  float beta[ON_MAX_GROUPS];
  float step[ON_MAX_GROUPS];
  uint32_t keys[ON_GPCHAINS][2];
};

template <int N, int Z>
__global__ void __launch_bounds__(ON_GRID_THREADS) on_colour_kernel(const __grid_constant__ OnGridParams P) {
  const int lchain = blockIdx.y, chain = P.chain0 + lchain;
  const int group = chain / P.chains_per_group;
  const uint32_t sweep = (P.cursor ? P.cursor[0] : 0u) + P.sweep;
  const uint32_t meas = (P.cursor ? P.cursor[1] : 0u) + P.meas;
  float* lat = P.spins + (size_t)chain * N * 2 * P.g.slots;
  long long nacc = 0;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P.g.slots; s += gridDim.x * blockDim.x)
    nacc += on_site<N, Z>(lat, P.g, P.col, s, P.code, sweep, P.beta[group], P.step[group], P.keys[lchain][0],
                          P.keys[lchain][1]);
  if (P.code == CRITMC_METROPOLIS) {
    nacc = warp_sum(nacc);
    if ((threadIdx.x & 31) == 0 && nacc)
      atomicAdd(P.acc + ((size_t)meas * P.n_chains + chain) * P.nv + (P.nv - 1), as_ull(nacc));
  }
}

template <int N>
__global__ void __launch_bounds__(ON_GRID_THREADS) on_normalize_kernel(const __grid_constant__ OnGridParams P) {
  const int chain = P.chain0 + blockIdx.y;
  const size_t n_sites = 2 * (size_t)P.g.slots;
  float* lat = P.spins + (size_t)chain * N * n_sites;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_sites; j += gridDim.x * blockDim.x)
    on_normalize_site<N>(lat, n_sites, j);
}

template <int N, int Z>
__global__ void __launch_bounds__(ON_GRID_THREADS) on_measure_kernel(const __grid_constant__ OnGridParams P) {
  constexpr int NV = on_nv<N, Z>();
  const int chain = P.chain0 + blockIdx.y;
  const uint32_t meas = (P.cursor ? P.cursor[1] : 0u) + P.meas;
  const size_t n_sites = 2 * (size_t)P.g.slots;
  const float* lat = P.spins + (size_t)chain * N * n_sites;
  long long v[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = 0;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_sites; j += gridDim.x * blockDim.x)
    on_measure_site<N, Z>(lat, P.g, j, v);
  unsigned long long* acc = P.acc + ((size_t)meas * P.n_chains + chain) * NV;
#pragma unroll
  for (int q = 0; q < NV - 1; ++q) {
    const long long w = warp_sum(v[q]);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(acc + q, as_ull(w));
  }
}

template <int N, int Z>
__global__ void on_grid_finalize(const unsigned long long* acc, int n_chains, int n_meas, double* e_out,
                                 double* m_out, double* sc_out, double* ss_out, long long* aux_out) {
  constexpr int NV = on_nv<N, Z>();
  constexpr int DIM = Z / 2;
  const size_t total = (size_t)n_chains * n_meas * NV;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int q = (int)(i % NV);
    const size_t mc = i / NV;  // meas * n_chains + chain
    const size_t chain = mc % n_chains;
    const int meas = (int)(mc / n_chains);
    on_write_sum<N, Z>(e_out + chain * n_meas, m_out + chain * n_meas * N, sc_out + chain * n_meas * DIM,
                       ss_out + chain * n_meas * DIM, aux_out + chain * n_meas * 4, meas, q,
                       (long long)acc[i]);
  }
}

__global__ void on_cursor_set(uint32_t* cursor, uint32_t sweep, uint32_t meas) {
  cursor[0] = sweep;
  cursor[1] = meas;
}

__global__ void on_cursor_bump(uint32_t* cursor, uint32_t sweeps, uint32_t meas) {
  cursor[0] += sweeps;
  cursor[1] += meas;
}

template <int N, int Z>
static int on_grid_launches(OnGridParams& P, const int* codes, const int* reps, int n_rows, int n_meas,
                            uint32_t sweep0, int n_chains, int blocks, uint32_t* cursor,
                            unsigned long long* acc, double* e_out, double* m_out, double* sc_out,
                            double* ss_out, long long* aux_out, const uint32_t* keys, cudaStream_t s) {
  long long per_meas = 0;
  for (int r = 0; r < n_rows; ++r) per_meas += reps[r];
  P.acc = acc;
  if (cudaMemsetAsync(acc, 0, (size_t)n_chains * n_meas * P.nv * 8, s) != cudaSuccess) return cuda_fail("memset");
  for (int c0 = 0; c0 < n_chains; c0 += ON_GPCHAINS) {
    const int nc = std::min(ON_GPCHAINS, n_chains - c0);
    P.chain0 = c0;
    std::memset(P.keys, 0, sizeof(P.keys));
    std::memcpy(P.keys, keys + 2 * (size_t)c0, sizeof(uint32_t) * 2 * nc);
    const dim3 grid_c((unsigned)blocks, (unsigned)nc);
    const uint32_t site_blocks = (uint32_t)std::min<size_t>(2 * (size_t)blocks, (2 * (size_t)P.g.slots + ON_GRID_THREADS - 1) / ON_GRID_THREADS);
    const dim3 grid_s(std::max(1u, site_blocks), (unsigned)nc);
    auto launch_meas = [&](uint32_t sweep_rel, uint32_t meas_rel, const uint32_t* cur) {
      P.cursor = cur;
      P.meas = meas_rel;
      uint32_t sw = sweep_rel;
      for (int r = 0; r < n_rows; ++r) {
        P.code = codes[r];
        for (int rep = 0; rep < reps[r]; ++rep) {
          P.sweep = sw;
          for (int c = 0; c < 2; ++c) {
            P.col = c;
            on_colour_kernel<N, Z><<<grid_c, ON_GRID_THREADS, 0, s>>>(P);
          }
          ++sw;
        }
      }
      on_normalize_kernel<N><<<grid_s, ON_GRID_THREADS, 0, s>>>(P);
      on_measure_kernel<N, Z><<<grid_s, ON_GRID_THREADS, 0, s>>>(P);
    };
    // a graph of G measurements replayed with a device cursor (cached across
    // calls with the same parameters), the rest launched directly
    const long long launches = 2 * per_meas + 2;
    const int G = (int)std::max<long long>(1, std::min<long long>(n_meas, 512 / launches));
    const int n_graph = n_meas / G;
    int done = 0;
    if (n_graph > 1) {
      on_cursor_set<<<1, 1, 0, s>>>(cursor, sweep0, 0);
      P.cursor = cursor;
      P.sweep = P.meas = 0;
      P.code = P.col = 0;
      int dev = 0;
      cudaGetDevice(&dev);
      GraphKey key;
      key.add(0x4f4e4752u).add(dev).add(N).add(Z).add(G).add(n_rows).add(grid_c).add(grid_s).add(P);
      key.add_bytes(codes, sizeof(int) * n_rows).add_bytes(reps, sizeof(int) * n_rows);
      cudaGraphExec_t exec = graph_cache_find(key);
      if (!exec) {
        cudaGraph_t graph;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return cuda_fail("capture");
        for (int m = 0; m < G; ++m) launch_meas((uint32_t)(m * per_meas), (uint32_t)m, cursor);
        on_cursor_bump<<<1, 1, 0, s>>>(cursor, (uint32_t)(G * per_meas), (uint32_t)G);
        if (cudaStreamEndCapture(s, &graph) != cudaSuccess) return cuda_fail("end capture");
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return cuda_fail("instantiate");
        graph_cache_insert(key, exec);
      }
      for (int i = 0; i < n_graph; ++i) cudaGraphLaunch(exec, s);
      done = n_graph * G;
    }
    for (int m = done; m < n_meas; ++m)
      launch_meas((uint32_t)(sweep0 + (uint32_t)(m * per_meas)), (uint32_t)m, nullptr);
  }
  const size_t total = (size_t)n_chains * n_meas * P.nv;
  const int fb = (int)std::min<size_t>(1184, (total + 255) / 256);
  on_grid_finalize<N, Z><<<std::max(1, fb), 256, 0, s>>>(acc, n_chains, n_meas, e_out, m_out, sc_out, ss_out,
                                                         aux_out);
  if (int e_ = cuda_check("launch")) return e_;
  return CRITMC_OK;
}

static thread_local OnParams g_on;

}  // namespace critmc

using namespace critmc;

extern "C" int32_t critmc_on_run(float* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                 int32_t n, int32_t n_chains, const uint32_t* keys,
                                 const double* betas, const double* steps, int32_t n_groups,
                                 uint32_t sweep0, const int64_t* schedule, int32_t n_rows,
                                 int32_t n_meas, double* e_out, double* m_out, double* stiff_c_out,
                                 double* stiff_s_out, int64_t* aux_out, void* stream) {
  clear_error();
  OnParams& P = g_on;
  int st = byte_geom(dim, lx, ly, lz, P.g);
  if (st) return st;
  if (n != 2 && n != 3) return fail(CRITMC_ERR_UNSUPPORTED, "O(n) kernels handle n = 2 and n = 3");
  if (!spins || !keys || !betas || !steps || !e_out || !m_out || !stiff_c_out || !stiff_s_out || !aux_out)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_groups < 1 || n_groups > ON_MAX_GROUPS || n_chains % n_groups)
    return fail(CRITMC_ERR_INVALID, "need n_chains >= 1 and 1 <= n_groups <= 16 dividing n_chains");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  if (!schedule || n_rows < 1 || n_rows > ON_MAX_ROWS) return fail(CRITMC_ERR_INVALID, "schedule must have 1..8 rows");
  long long per_meas = 0;
  for (int r = 0; r < n_rows; ++r) {
    const int64_t code = schedule[2 * r], reps = schedule[2 * r + 1];
    if (code != CRITMC_METROPOLIS && code != CRITMC_HEATBATH && code != CRITMC_OVERRELAX)
      return fail(CRITMC_ERR_UNSUPPORTED, "O(n) kernels run metropolis, heatbath and overrelax rows");
    // a row of 0 repetitions is allowed: a schedule of only such rows measures
    if (reps < 0 || reps > (1 << 20)) return fail(CRITMC_ERR_INVALID, "schedule repetitions must be in [0, 2^20]");
    P.codes[r] = (int)code;
    P.reps[r] = (int)reps;
    per_meas += reps;
  }
  if ((long long)sweep0 + per_meas * n_meas > 0xFFFFFFFFLL)
    return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");
  if (n_meas == 0) return CRITMC_OK;
  for (int gi = 0; gi < n_groups; ++gi) {
    if (!std::isfinite(betas[gi]) || !std::isfinite(steps[gi]))
      return fail(CRITMC_ERR_INVALID, "betas and steps must be finite");
    P.beta[gi] = (float)betas[gi];
    P.step[gi] = (float)steps[gi];
  }
  P.spins = spins;
  P.e_out = e_out;
  P.m_out = m_out;
  P.sc_out = stiff_c_out;
  P.ss_out = stiff_s_out;
  P.aux_out = (long long*)aux_out;
  P.n_rows = n_rows;
  P.n_chains = n_chains;
  P.chains_per_group = n_chains / n_groups;
  P.n_meas = n_meas;
  P.sweep0 = sweep0;
  const size_t lat_bytes = (size_t)n * 2 * P.g.slots * sizeof(float);
  P.resident = lat_bytes <= (size_t)ON_SMEM_MAX;
  const size_t smem = P.resident ? lat_bytes : 0;
  const int threads = on_site_threads(P.g.slots);
  cudaStream_t s = (cudaStream_t)stream;
  for (int c0 = 0; c0 < n_chains; c0 += ON_PCHAINS) {
    const int nc = std::min(ON_PCHAINS, n_chains - c0);
    P.chain0 = c0;
    std::memcpy(P.keys, keys + 2 * (size_t)c0, sizeof(uint32_t) * 2 * nc);
    auto launch = [&](auto kern) {
      if (smem > 0) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  // static + dynamic may pass 48 KiB
      kern<<<nc, threads, smem, s>>>(P);
    };
    const int key = n * 10 + dim;
    switch (key) {
      case 21: launch(on_run_kernel<2, 2>); break;
      case 22: launch(on_run_kernel<2, 4>); break;
      case 23: launch(on_run_kernel<2, 6>); break;
      case 31: launch(on_run_kernel<3, 2>); break;
      case 32: launch(on_run_kernel<3, 4>); break;
      default: launch(on_run_kernel<3, 6>); break;
    }
    if (int e_ = cuda_check("launch")) return e_;
  }
  return CRITMC_OK;
}

// ---------------------------------------------------------------------------
// O(n) chains as work items (persistent kernel, queue of items).
// ---------------------------------------------------------------------------
#include "items_host.h"

extern "C" int64_t critmc_on_grid_scratch_bytes(int32_t n_chains, int32_t n_meas, int32_t n, int32_t dim) {
  if (n_chains < 0 || n_meas < 0 || n < 2 || n > 3 || dim < 1 || dim > 3) return -1;
  return 256 + (int64_t)n_chains * n_meas * (2 + n + 2 * dim) * 8;
}

extern "C" int32_t critmc_on_run_grid(float* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                      int32_t n, int32_t n_chains, const uint32_t* keys,
                                      const double* betas, const double* steps, int32_t n_groups,
                                      uint32_t sweep0, const int64_t* schedule, int32_t n_rows,
                                      int32_t n_meas, double* e_out, double* m_out, double* stiff_c_out,
                                      double* stiff_s_out, int64_t* aux_out, void* scratch,
                                      int32_t blocks_per_chain, void* stream) {
  clear_error();
  static thread_local OnGridParams P;
  int st = byte_geom(dim, lx, ly, lz, P.g);
  if (st) return st;
  if (n != 2 && n != 3) return fail(CRITMC_ERR_UNSUPPORTED, "O(n) kernels handle n = 2 and n = 3");
  if (!spins || !keys || !betas || !steps || !e_out || !m_out || !stiff_c_out || !stiff_s_out || !aux_out ||
      !scratch)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_groups < 1 || n_groups > ON_MAX_GROUPS || n_chains % n_groups)
    return fail(CRITMC_ERR_INVALID, "need n_chains >= 1 and 1 <= n_groups <= 16 dividing n_chains");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  if (!schedule || n_rows < 1 || n_rows > ON_MAX_ROWS) return fail(CRITMC_ERR_INVALID, "schedule must have 1..8 rows");
  if (blocks_per_chain < 0 || blocks_per_chain > 65535) return fail(CRITMC_ERR_INVALID, "blocks_per_chain out of range");
  int codes[ON_MAX_ROWS], reps[ON_MAX_ROWS];
  long long per_meas = 0;
  for (int r = 0; r < n_rows; ++r) {
    const int64_t code = schedule[2 * r], rp = schedule[2 * r + 1];
    if (code != CRITMC_METROPOLIS && code != CRITMC_HEATBATH && code != CRITMC_OVERRELAX)
      return fail(CRITMC_ERR_UNSUPPORTED, "O(n) kernels run metropolis, heatbath and overrelax rows");
    if (rp < 0 || rp > (1 << 20)) return fail(CRITMC_ERR_INVALID, "schedule repetitions must be in [0, 2^20]");
    codes[r] = (int)code;
    reps[r] = (int)rp;
    per_meas += rp;
  }
  if ((long long)sweep0 + per_meas * n_meas > 0xFFFFFFFFLL)
    return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");
  if (n_meas == 0) return CRITMC_OK;
  for (int gi = 0; gi < n_groups; ++gi) {
    if (!std::isfinite(betas[gi]) || !std::isfinite(steps[gi]))
      return fail(CRITMC_ERR_INVALID, "betas and steps must be finite");
    P.beta[gi] = (float)betas[gi];
    P.step[gi] = (float)steps[gi];
  }
  P.spins = spins;
  P.n_chains = n_chains;
  P.chains_per_group = n_chains / n_groups;
  P.nv = 2 + n + 2 * dim;
  int blocks = blocks_per_chain;
  if (blocks == 0) {
    // one site per thread while that keeps the GPU's blocks resident at once
    const int by_sites = (int)((P.g.slots + ON_GRID_THREADS - 1) / ON_GRID_THREADS);
    const int by_gpu = std::max(1, 148 * 8 / std::min(n_chains, ON_GPCHAINS));
    blocks = std::max(1, std::min(by_sites, by_gpu));
  }
  CaptureStream cs;
  if ((st = cs.begin(stream))) return st;
  uint32_t* cursor = (uint32_t*)scratch;
  unsigned long long* acc = (unsigned long long*)((char*)scratch + 256);
  switch (n * 10 + dim) {
    case 21: st = on_grid_launches<2, 2>(P, codes, reps, n_rows, n_meas, sweep0, n_chains, blocks, cursor, acc, e_out, m_out, stiff_c_out, stiff_s_out, (long long*)aux_out, keys, cs.work); break;
    case 22: st = on_grid_launches<2, 4>(P, codes, reps, n_rows, n_meas, sweep0, n_chains, blocks, cursor, acc, e_out, m_out, stiff_c_out, stiff_s_out, (long long*)aux_out, keys, cs.work); break;
    case 23: st = on_grid_launches<2, 6>(P, codes, reps, n_rows, n_meas, sweep0, n_chains, blocks, cursor, acc, e_out, m_out, stiff_c_out, stiff_s_out, (long long*)aux_out, keys, cs.work); break;
    case 31: st = on_grid_launches<3, 2>(P, codes, reps, n_rows, n_meas, sweep0, n_chains, blocks, cursor, acc, e_out, m_out, stiff_c_out, stiff_s_out, (long long*)aux_out, keys, cs.work); break;
    case 32: st = on_grid_launches<3, 4>(P, codes, reps, n_rows, n_meas, sweep0, n_chains, blocks, cursor, acc, e_out, m_out, stiff_c_out, stiff_s_out, (long long*)aux_out, keys, cs.work); break;
    default: st = on_grid_launches<3, 6>(P, codes, reps, n_rows, n_meas, sweep0, n_chains, blocks, cursor, acc, e_out, m_out, stiff_c_out, stiff_s_out, (long long*)aux_out, keys, cs.work); break;
  }
  if (st) return st;
  return cs.finish();
}

namespace critmc {

// One kernel per (n, dimension): the variants' register needs differ, and a
// kernel holding all of them would be held to the largest.  CL > 1: each item
// is advanced by a cluster of CL blocks (block 0 takes the item from the queue
// and hands its index to the others).
template <int N, int Z, int CL>
__global__ void __launch_bounds__(ON_THREADS) on_items_kernel(const critmc_item* items, int n,
                                                              unsigned* queue, size_t smem, RunCtl ctl) {
  using T = Team<CL>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int cur;
  CtlPoll poll;
  poll.start();
  const unsigned rank = T::rank();
  for (;;) {
    if (rank == 0 && threadIdx.x == 0) {
      const int v = poll.check(ctl) ? n : (int)atomicAdd(queue, 1u);
      for (int r = 0; r < CL; ++r) *T::at(&cur, (unsigned)r) = v;
    }
    T::sync();
    const int i = cur;
    T::sync();
    if (i >= n) break;
    const critmc_item& it = items[i];
    OnChain a;
    if (ctl.status) {
      a.ctl = &ctl;
      a.poll = &poll;
    }
    a.g.dim = it.dim;
    a.g.lx = it.lx;
    a.g.ly = it.dim >= 2 ? it.ly : 1;
    a.g.lz = it.dim >= 3 ? it.lz : 1;
    a.g.hx = it.lx / 2;
    a.g.rows = a.g.ly * a.g.lz;
    a.g.slots = (uint32_t)(a.g.rows * a.g.hx);
    a.gl = reinterpret_cast<float*>(it.spins);
    a.e_out = reinterpret_cast<double*>(it.e_out);
    a.m_out = reinterpret_cast<double*>(it.vec_out);
    a.sc_out = it.sc_out;
    a.ss_out = it.ss_out;
    a.aux_out = reinterpret_cast<long long*>(it.aux_out);
    a.n_meas = it.n_meas;
    a.n_rows = it.n_rows;
    a.resident = (size_t)N * 2 * a.g.slots * sizeof(float) <= smem;
    a.nt = on_site_threads(a.g.slots);
    a.codes = it.codes;
    a.reps = it.reps;
    a.sweep0 = it.sweep0;
    a.k0 = it.key[0];
    a.k1 = it.key[1];
    a.beta = it.beta;
    a.step = it.step;
    on_chain_run<N, Z, CL>(a, smem_raw);
  }
}

template <int N, int Z>
static int on_items_launch_nz(const critmc_item* items, int n, unsigned* queue, size_t smem, int team,
                              const RunCtl& ctl, cudaStream_t s) {
  switch (team) {
    case 2: return launch_team(on_items_kernel<N, Z, 2>, 2, ON_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    case 4: return launch_team(on_items_kernel<N, Z, 4>, 4, ON_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    case 8: return launch_team(on_items_kernel<N, Z, 8>, 8, ON_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    case 16: return launch_team(on_items_kernel<N, Z, 16>, 16, ON_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    default: break;
  }
  auto kern = on_items_kernel<N, Z, 1>;
  if (smem > 0 &&  // static + dynamic may pass 48 KiB
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return cuda_fail("shared memory attribute");
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ON_THREADS, smem);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, std::min(n, std::max(1, per_sm) * sms));
  kern<<<grid, ON_THREADS, smem, s>>>(items, n, queue, smem, ctl);
  if (int e_ = cuda_check("launch")) return e_;
  return CRITMC_OK;
}

template <int N, int Z>
static int on_items_team_clusters_nz(int team) {
  switch (team) {
    case 2: return team_clusters(on_items_kernel<N, Z, 2>, 2, ON_THREADS);
    case 4: return team_clusters(on_items_kernel<N, Z, 4>, 4, ON_THREADS);
    case 8: return team_clusters(on_items_kernel<N, Z, 8>, 8, ON_THREADS);
    case 16: return team_clusters(on_items_kernel<N, Z, 16>, 16, ON_THREADS);
    default: return fail(CRITMC_ERR_INVALID, "team size must be 2, 4, 8 or 16");
  }
}

int on_items_team_clusters(int n_comp, int dim, int team) {
  switch (n_comp * 10 + dim) {
    case 21: return on_items_team_clusters_nz<2, 2>(team);
    case 22: return on_items_team_clusters_nz<2, 4>(team);
    case 23: return on_items_team_clusters_nz<2, 6>(team);
    case 31: return on_items_team_clusters_nz<3, 2>(team);
    case 32: return on_items_team_clusters_nz<3, 4>(team);
    case 33: return on_items_team_clusters_nz<3, 6>(team);
    default: return fail(CRITMC_ERR_INVALID, "O(n) items need n = 2 or 3 and dim 1..3");
  }
}

int on_items_launch(const critmc_item* items, int n, int n_comp, int dim, unsigned* queue, size_t smem, int team,
                    const RunCtl& ctl, cudaStream_t s) {
  switch (n_comp * 10 + dim) {
    case 21: return on_items_launch_nz<2, 2>(items, n, queue, smem, team, ctl, s);
    case 22: return on_items_launch_nz<2, 4>(items, n, queue, smem, team, ctl, s);
    case 23: return on_items_launch_nz<2, 6>(items, n, queue, smem, team, ctl, s);
    case 31: return on_items_launch_nz<3, 2>(items, n, queue, smem, team, ctl, s);
    case 32: return on_items_launch_nz<3, 4>(items, n, queue, smem, team, ctl, s);
    case 33: return on_items_launch_nz<3, 6>(items, n, queue, smem, team, ctl, s);
    default: return fail(CRITMC_ERR_INVALID, "O(n) items need n = 2 or 3 and dim 1..3");
  }
}

}  // namespace critmc
