// Edwards-Anderson +-J spin glasses with parallel tempering, one thread block
// per disorder sample, both replica sets resident in shared memory.
//
// Replica multi-spin coding: the word of a site holds one bit per temperature
// (bit k = configuration at temperature index k, hot -> cold).  A sweep updates
// all temperatures of a replica set at once with the bit-sliced MSB-first
// acceptance of the Ising kernels; each lane compares with the threshold of
// its own temperature (per-lane threshold planes, kernel parameters).  An
// accepted replica exchange moves configurations between lanes, so after the
// swap pass the words are permuted (one warp ballot per word); critmc's perm
// array survives as conf_at for the round-trip bookkeeping.
//
// Replaces critmc src/critmc/kernels/glass.py:81-163 (`pt_run`), :42-53
// (`metropolis_sweep`), :34-38 (`energy`), :57-77 (`_measure`).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "geom.cuh"
#include "host_common.h"
#include "msc_ising.cuh"

namespace critmc {

constexpr int EA_THREADS = 256;
constexpr int EA_MAX_SITES = 4096;
constexpr int EA_MAX_L = 64;
constexpr int EA_NOBS = 7;  // e, q_l, |q|, q^2, q^4, |q(kmin)|^2, count (critmc glass.py:24-31)
constexpr int EA_PSAMPLES = 512;
constexpr int EA_FIXCAP = 64;

// Temperature set and step counts shared by every sample of a call.
struct EaCommon {
  const uint32_t* swap_thr;
  int m, n_steps, n_bins, sweeps_per_step, swap_width;
  uint32_t t0;
  uint32_t planes[3][32];  // lane masks of the threshold bits, classes v = 0..z/2-1
};

// One lattice size: its samples' device arrays and geometry.
struct EaSet {
  uint32_t* words;
  const uint8_t* jneg;
  uint8_t* conf_at;
  uint8_t* labels;
  double* acc;
  long long* swap_acc;
  long long* swap_try;
  long long* label_hist;
  long long* trips;
  const uint32_t* keys;  // device [n_samples][2][2] (campaign), or null (keys in parameters)
  ByteGeom g;
  int n_samples;
  int ext[3];
  double cosx[EA_MAX_L], sinx[EA_MAX_L];  // cos/sin(2 pi x / L) per axis extent (same L per axis)
};

struct EaParams {
  EaCommon C;
  EaSet S;
  int sample0;
  uint32_t keys[EA_PSAMPLES][2][2];
};

// Bit-sliced (vertical) counters: v[p] holds bit p of one count per lane.
// Add a 0..7 count given as bit planes c.
template <int NP>
__device__ __forceinline__ void vadd3(uint32_t (&v)[NP], const Count3& c) {
  uint32_t carry = 0;
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const uint32_t x = p == 0 ? c.b0 : (p == 1 ? c.b1 : (p == 2 ? c.b2 : 0u));
    const uint32_t a = v[p];
    v[p] = a ^ x ^ carry;
    carry = (a & x) | (carry & (a ^ x));
  }
}

// Add one bit per lane.
template <int NP>
__device__ __forceinline__ void vadd1(uint32_t (&v)[NP], uint32_t x) {
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const uint32_t a = v[p];
    v[p] = a ^ x;
    x &= a;
  }
}

// Sum of the warp's vertical counters for count lane `lane` (every lane of the
// warp takes part; each gets the total of its own lane index).
// Transpose the warp's 32x32 bit matrix: bit i of the result in lane k is bit
// k of lane i's word (recursive swap of off-diagonal blocks).
__device__ __forceinline__ uint32_t transpose32(uint32_t x, int lane) {
  const uint32_t lo[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    const int j = 16 >> t;
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~lo[t]) | ((y & ~lo[t]) >> j)) : ((x & lo[t]) | ((y & lo[t]) << j));
  }
  return x;
}

// Sum of the warp's vertical counters for count lane `lane` (every lane of the
// warp takes part; each gets the total of its own lane index): after the
// transpose, lane k holds bit k of every lane's plane.
template <int NP>
__device__ __forceinline__ int vreduce(const uint32_t (&v)[NP], int lane) {
  int mine = 0;
#pragma unroll
  for (int p = 0; p < NP; ++p) mine += __popc(transpose32(v[p], lane)) << p;
  return mine;
}

// threshold bit plane for the undecided lanes (counts 0 .. z/2-1)
template <int Z>
__device__ __forceinline__ uint32_t ea_tbits(const EaCommon& C, const Count3& c, int q) {
  const uint32_t lo = mux(c.b0, C.planes[1][q], C.planes[0][q]);
  if constexpr (Z == 6) return mux(c.b1, C.planes[2][q], lo);
  return lo;
}

struct EaFix {
  uint32_t idx, U, D;  // idx = set * words + colour * slots + slot
};

template <int Z>
__device__ __forceinline__ void ea_site(const ByteGeom& g, const uint32_t* lat, const uint8_t* jn,
                                        int set, int c, uint32_t s, uint32_t& w_s, Count3& cnt) {
  int r, i;
  byte_row_index(g, s, r, i);
  uint32_t nb[Z];
  byte_neighbours<Z>(g, c, r, i, nb);
  const uint32_t* base = lat + (size_t)set * 2 * g.slots;
  const uint32_t* own = base + (size_t)c * g.slots;
  const uint32_t* oth = base + (size_t)(c ^ 1) * g.slots;
  const uint32_t jb = jn[(size_t)c * g.slots + s];
  w_s = own[s];
  uint32_t x[Z];
#pragma unroll
  for (int q = 0; q < Z; ++q) x[q] = w_s ^ oth[nb[q]] ^ (0u - ((jb >> q) & 1u));
  cnt = count_bits<Z>(x);  // unsatisfied bonds per lane
}

template <int Z>
__device__ __forceinline__ void ea_planes(const EaCommon& C, const Count3& cnt, uint32_t k0,
                                          uint32_t k1, uint32_t slot, uint32_t sweep, uint32_t col,
                                          int g_begin, int g_end, uint32_t& D, uint32_t& U) {
  for (int grp = g_begin; grp < g_end && U; ++grp) {
    const critmc_u32x4 r = critmc_philox4x32(
        slot, sweep, CRITMC_TAG_PLANES | ((uint32_t)grp << 8) | (col << 16), 0u, k0, k1);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t t = ea_tbits<Z>(C, cnt, 4 * grp + q);
      D |= U & t & ~r.v[q];
      U &= ~(r.v[q] ^ t);
    }
  }
}

// Threads per block for a sample of this geometry (64, 128 or 256): every
// thread may hold at most 63 / z sites of one colour, the capacity of the
// 6-plane vertical counters of the energy and link-overlap sums.  Fewer
// threads per small sample let more samples share an SM (registers bound the
// blocks per SM), which pays on small lattices, where a step is dominated by
// its serial phases (swap walk, measurement) rather than by the sweep.
inline int ea_threads_for(const ByteGeom& g, int z) {
  // measured per size alone (3D, 512 samples): 64 threads gave +29 % at L = 6 and
  // +10 % at L = 8 but -9 % at L = 10, where the sweep outweighs the serial phases
  if (g.slots <= 256u && (g.slots + 63u) / 64u * (uint32_t)z <= 63u) return 64;
  if ((g.slots + 127u) / 128u * (uint32_t)z <= 63u) return 128;
  return EA_THREADS;
}

// Dynamic shared memory of one sample's block.
inline size_t ea_smem_bytes(const ByteGeom& g, int dim, int lx) {
  return (size_t)(2 * g.slots) * (2 * 4 + 4 + 1) + (size_t)dim * lx * 32 * 4;
}

// All PT steps of one sample by one thread block of T threads (64, 128 or 256;
// the vertical counters of a thread hold at most 63, so T must give every
// thread at most 63 / z sites of a colour: ea_threads_for).  key[set] =
// Philox key of replica set.
template <int Z, int T = EA_THREADS>
__device__ void ea_sample_run(const EaCommon& C, const EaSet& S, int sample, const uint32_t (&key)[2][2],
                              unsigned char* smem_raw, const RunCtl& ctl, CtlPoll& poll) {
  constexpr int DIM = Z / 2;
  const ByteGeom& g = S.g;
  const uint32_t n_sites = 2 * g.slots;
  uint32_t* lat = reinterpret_cast<uint32_t*>(smem_raw);  // [2 sets][2 colours][slots]
  uint32_t* qw = lat + 2 * n_sites;                      // overlap words [2][slots]
  int* splane = reinterpret_cast<int*>(qw + n_sites);    // [DIM][L][32] overlap per plane and lane
  uint8_t* jn = reinterpret_cast<uint8_t*>(splane + DIM * S.ext[0] * 32);  // [2][slots]
  __shared__ EaFix fix[(T / 32)][EA_FIXCAP];
  __shared__ int ecnt[2][32];  // unsatisfied bonds per set and temperature
  __shared__ int qlcnt[32];    // agreeing bonds of the overlap field
  __shared__ int sigma[2][32];
  __shared__ int es[2][32];         // energies per set and temperature slot during the swaps
  __shared__ uint32_t swu[2][32];   // swap uniforms of the step
  __shared__ int conf[2][32], lab[2][32];
  __shared__ double acc_s[32][EA_NOBS];
  __shared__ unsigned long long sw_acc[32], sw_try[32], lhist[32][2], trip[2];
  __shared__ int s_stop;
  __shared__ uint32_t s_acc_mask[2];  // swaps accepted in the step's walk, by set
  __shared__ uint32_t thr_s[31][32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m = C.m;
  const int ext = S.ext[0];  // every extent (equal extents are required)
  // the first 32 swap thresholds of each pair (energy gaps below 128, the common
  // case) in shared memory; the walk reads wider gaps from global memory
  for (int i = tid; i < (m - 1) * 32; i += T) {
    const int k = i >> 5, j = i & 31;
    thr_s[k][j] = j < C.swap_width ? C.swap_thr[(size_t)k * C.swap_width + j] : 0u;
  }
  uint32_t* gw = S.words + (size_t)sample * 2 * n_sites;
  for (uint32_t j = tid; j < 2 * n_sites; j += T) lat[j] = gw[j];
  for (uint32_t j = tid; j < n_sites; j += T) jn[j] = S.jneg[(size_t)sample * n_sites + j];
  if (tid < 64) {
    const int r = tid >> 5, k = tid & 31;
    if (k < m) {
      conf[r][k] = S.conf_at[((size_t)sample * 2 + r) * m + k];
      lab[r][k] = S.labels[((size_t)sample * 2 + r) * m + k];
    }
  }
  if (tid < 32) {
    sw_acc[tid] = sw_try[tid] = 0;
    lhist[tid][0] = lhist[tid][1] = 0;
    for (int o = 0; o < EA_NOBS; ++o) acc_s[tid][o] = 0.0;
  }
  if (tid < 2) trip[tid] = 0;
  __syncthreads();

  const uint32_t lt_mask = (1u << lane) - 1u;
  int bin = 0;
  long long next_edge = 1;
  for (int t = 0; t < C.n_steps; ++t) {
    if (ctl.status) {  // bounded run: stop between steps when the budget or a cancel says so
      if (tid == 0) s_stop = poll.check(ctl);
      __syncthreads();
      if (s_stop) break;
    }
    if (t >= next_edge) {
      // flush the finished bin (critmc glass.py:114-122)
      if (tid < m)
        for (int o = 0; o < EA_NOBS; ++o) {
          S.acc[(((size_t)sample * C.n_bins + bin) * m + tid) * EA_NOBS + o] = acc_s[tid][o];
          acc_s[tid][o] = 0.0;
        }
      ++bin;
      next_edge = (1LL << (bin + 1)) - 1;
    }
    const uint32_t step = C.t0 + (uint32_t)t;
    // ---- sweeps of every temperature of both sets --------------------------
    for (int sw = 0; sw < C.sweeps_per_step; ++sw) {
      const uint32_t sweep = step * (uint32_t)C.sweeps_per_step + (uint32_t)sw;
      for (int c = 0; c < 2; ++c) {
        int nf = 0;
        const uint32_t work = 2 * g.slots;  // both sets, one colour
        auto flush = [&]() {
          __syncwarp();
          for (int e = lane; e < nf; e += 32) {
            const EaFix f = fix[warp][e];
            const int set = f.idx >= n_sites;
            const uint32_t s = f.idx - set * n_sites - (uint32_t)c * g.slots;
            uint32_t w_s;
            Count3 cnt;
            ea_site<Z>(g, lat, jn, set, c, s, w_s, cnt);
            uint32_t D2 = f.D, U2 = f.U;
            ea_planes<Z>(C, cnt, key[set][0], key[set][1], s, sweep, (uint32_t)c, 2, 8, D2, U2);
            lat[f.idx] = w_s ^ D2;
          }
          __syncwarp();
          nf = 0;
        };
        auto defer = [&](uint32_t U, uint32_t D, uint32_t idx) {
          const uint32_t need = __ballot_sync(0xffffffffu, U != 0);
          if (need) {
            const int cntn = __popc(need);
            if (nf + cntn > EA_FIXCAP) flush();
            if (U != 0) fix[warp][nf + __popc(need & lt_mask)] = EaFix{idx, U, D};
            nf += cntn;
          }
        };
        // two work items per loop step: their site loads, Philox planes and
        // comparisons are independent and interleave (+1 to +3 % per size);
        // an item past the end is computed on slot 0 and discarded
        const uint32_t rounds = (work + 2 * T - 1) / (2 * T);
        for (uint32_t it = 0; it < rounds; ++it) {
          const uint32_t jA = it * 2 * T + tid, jB = jA + T;
          const bool vA = jA < work, vB = jB < work;
          const uint32_t jAc = vA ? jA : 0u, jBc = vB ? jB : 0u;
          const int setA = jAc >= g.slots, setB = jBc >= g.slots;
          const uint32_t sA = jAc - setA * g.slots, sB = jBc - setB * g.slots;
          uint32_t wA, wB;
          Count3 cA, cB;
          ea_site<Z>(g, lat, jn, setA, c, sA, wA, cA);
          ea_site<Z>(g, lat, jn, setB, c, sB, wB, cB);
          const uint32_t alwA = (Z == 6) ? (cA.b2 | (cA.b1 & cA.b0)) : (cA.b1 | cA.b2);
          const uint32_t alwB = (Z == 6) ? (cB.b2 | (cB.b1 & cB.b0)) : (cB.b1 | cB.b2);
          uint32_t DA = alwA, UA = vA ? ~alwA : 0u, DB = alwB, UB = vB ? ~alwB : 0u;
          ea_planes<Z>(C, cA, key[setA][0], key[setA][1], sA, sweep, (uint32_t)c, 0, 2, DA, UA);
          ea_planes<Z>(C, cB, key[setB][0], key[setB][1], sB, sweep, (uint32_t)c, 0, 2, DB, UB);
          const uint32_t idxA = (uint32_t)setA * n_sites + (uint32_t)c * g.slots + sA;
          const uint32_t idxB = (uint32_t)setB * n_sites + (uint32_t)c * g.slots + sB;
          if (vA && UA == 0) lat[idxA] = wA ^ DA;
          if (vB && UB == 0) lat[idxB] = wB ^ DB;
          defer(UA, DA, idxA);
          defer(UB, DB, idxB);
        }
        flush();
        __syncthreads();
      }
    }
    // ---- energies per set and temperature (unsatisfied bonds) ---------------
    if (tid < 64) ecnt[tid >> 5][tid & 31] = 0;
    __syncthreads();
    {
      // colour-0 sites see every bond once; at most 63 / z sites per thread (ea_threads_for)
      uint32_t va[6] = {0, 0, 0, 0, 0, 0}, vb[6] = {0, 0, 0, 0, 0, 0};
      for (uint32_t s = tid; s < g.slots; s += T) {
        uint32_t w_s;
        Count3 cnt;
        ea_site<Z>(g, lat, jn, 0, 0, s, w_s, cnt);
        vadd3(va, cnt);
        ea_site<Z>(g, lat, jn, 1, 0, s, w_s, cnt);
        vadd3(vb, cnt);
      }
      atomicAdd(&ecnt[0][lane], vreduce(va, lane));
      atomicAdd(&ecnt[1][lane], vreduce(vb, lane));
    }
    __syncthreads();
    // ---- replica exchange, one warp per set (critmc glass.py:128-152): its lanes
    // draw the swap uniforms, lane 0 walks k = 0..m-2 in order ---------------
    if (warp < 2) {
      const int r = warp;
      const int n_bonds = (int)n_sites * DIM;
      if (lane < m) {
        es[r][lane] = -(n_bonds - 2 * ecnt[r][lane]);
        sigma[r][lane] = lane;
      }
      if (lane < m - 1)
        swu[r][lane] = critmc_philox4x32((uint32_t)lane, step, CRITMC_TAG_SWAP | ((uint32_t)r << 16), 0u,
                                         key[r][0], key[r][1]).v[0];
      if (lane < m - 1) atomicAdd(&sw_try[lane], 1ULL);  // every pair is tried once per set and step
      __syncwarp();
      if (lane == 0) {
        // The walk swaps positions k and k+1 in order k = 0 .. m-2, so position k
        // is final after step k and position k+1 is still untouched: carry the
        // entry moving up (energy, configuration, permutation) in registers and
        // write each position once.  Accepted pairs go to a bit mask that the
        // lanes count afterwards, off the serial chain.
        int cur_e = es[r][0], cur_c = conf[r][0], cur_s = sigma[r][0];
        uint32_t accm = 0;
        for (int k = 0; k < m - 1; ++k) {
          const int ne = es[r][k + 1], nc = conf[r][k + 1], ns = sigma[r][k + 1];
          // betas ascend hot -> cold, so x = (b_k - b_k+1)(E_k - E_k+1) >= 0 iff E_k <= E_k+1
          const int de = cur_e - ne;
          bool ok = de <= 0;
          if (!ok) {
            int j = de / 4;
            if (j > C.swap_width - 1) j = C.swap_width - 1;
            ok = swu[r][k] < (j < 32 ? thr_s[k][j] : C.swap_thr[(size_t)k * C.swap_width + j]);
          }
          if (ok) {  // the carried entry moves on to k+1
            accm |= 1u << k;
            es[r][k] = ne;
            conf[r][k] = nc;
            sigma[r][k] = ns;
          } else {
            es[r][k] = cur_e;
            conf[r][k] = cur_c;
            sigma[r][k] = cur_s;
            cur_e = ne;
            cur_c = nc;
            cur_s = ns;
          }
        }
        es[r][m - 1] = cur_e;
        conf[r][m - 1] = cur_c;
        sigma[r][m - 1] = cur_s;
        s_acc_mask[r] = accm;
        const int hot = conf[r][0], cold = cur_c;
        // labels are indexed by configuration: lab[r][c] for configuration c
        if (lab[r][hot] == 2) atomicAdd(&trip[r], 1ULL);
        lab[r][hot] = 1;
        if (lab[r][cold] == 1) atomicAdd(&trip[r], 1ULL);
        lab[r][cold] = 2;
      }
      __syncwarp();
      if (lane < m - 1 && ((s_acc_mask[r] >> lane) & 1u)) atomicAdd(&sw_acc[lane], 1ULL);
      if (lane < m) {
        ecnt[r][lane] = (es[r][lane] + n_bonds) / 2;  // permuted counts
        const int l = lab[r][conf[r][lane]];
        if (l == 1) atomicAdd(&lhist[lane][0], 1ULL);
        else if (l == 2) atomicAdd(&lhist[lane][1], 1ULL);
      }
    }
    __syncthreads();
    // ---- move configurations between lanes: new bit k = old bit sigma[k] ----
    // (32 words per warp: transpose, take row sigma[k] into row k, transpose back)
    for (int r = 0; r < 2; ++r) {
      const int src = lane < m ? sigma[r][lane] : lane;
      for (uint32_t base = (uint32_t)warp * 32; base < n_sites; base += T) {
        const uint32_t i = base + (uint32_t)lane;
        uint32_t x = i < n_sites ? lat[(size_t)r * n_sites + i] : 0u;
        x = transpose32(x, lane);
        const uint32_t y = __shfl_sync(0xffffffffu, x, src);
        x = transpose32(lane < m ? y : 0u, lane);
        if (i < n_sites) lat[(size_t)r * n_sites + i] = x;
      }
    }
    __syncthreads();
    // ---- measurement (critmc glass.py:57-77, :153-163) -----------------------
    for (uint32_t j = tid; j < n_sites; j += T) qw[j] = ~(lat[j] ^ lat[n_sites + j]);
    if (tid < 32) qlcnt[tid] = 0;
    __syncthreads();
    {
      uint32_t vq[6] = {0, 0, 0, 0, 0, 0};  // agreeing bonds, at most 63 per lane (ea_threads_for)
      for (uint32_t s = tid; s < g.slots; s += T) {
        int r, i;
        byte_row_index(g, s, r, i);
        uint32_t nb[Z];
        byte_neighbours<Z>(g, 0, r, i, nb);
        const uint32_t qs = qw[s];
        uint32_t x[Z];
#pragma unroll
        for (int q = 0; q < Z; ++q) x[q] = ~(qs ^ qw[g.slots + nb[q]]);
        vadd3(vq, count_bits<Z>(x));
      }
      atomicAdd(&qlcnt[lane], vreduce(vq, lane));
    }
    // per-plane overlap counts: warp w handles planes (d, x) = w, w + WARPS, ...;
    // its lanes split the plane's sites (at most 256 / 32 = 8 each)
    // (equal extents: ext = lx for every direction; coordinates in registers)
    for (int pl = warp; pl < DIM * ext; pl += (T / 32)) {
      const int d = pl / ext, x0 = pl - d * ext;
      const int n_pl = DIM == 3 ? ext * ext : ext;
      uint32_t vp[4] = {0, 0, 0, 0};
      for (int idx = lane; idx < n_pl; idx += 32) {
        const int a = idx % ext, b = DIM == 3 ? idx / ext : 0;
        const int x = d == 0 ? x0 : a;
        const int y = d == 0 ? a : (d == 1 ? x0 : b);
        const int z = d == 2 ? x0 : b;
        const int col = (x + y + z) & 1;
        const uint32_t slot = (uint32_t)((y + g.ly * z) * g.hx + x / 2);
        vadd1(vp, qw[(size_t)col * g.slots + slot]);
      }
      splane[(d * ext + x0) * 32 + lane] = vreduce(vp, lane);
    }
    __syncthreads();
    if (tid < m) {
      const int k = tid;
      const double n = (double)n_sites;
      const double nb = n * DIM;
      int qs = 0;
      for (int x = 0; x < ext; ++x) qs += splane[x * 32 + k];
      const double q = (2.0 * qs - n) / n;
      const double ql = (2.0 * qlcnt[k] - nb) / nb;
      double qk2 = 0.0;
      for (int d = 0; d < DIM; ++d) {
        const double per = n / ext;
        double re = 0.0, im = 0.0;
        for (int x = 0; x < ext; ++x) {
          const double sx = 2.0 * splane[(d * ext + x) * 32 + k] - per;
          re += S.cosx[x] * sx;
          im += S.sinx[x] * sx;
        }
        qk2 += (re * re + im * im) / (n * n);
      }
      qk2 /= DIM;
      const double ea = -(nb - 2.0 * ecnt[0][k]), eb = -(nb - 2.0 * ecnt[1][k]);
      acc_s[k][0] += 0.5 * (ea + eb) / n;
      acc_s[k][1] += ql;
      acc_s[k][2] += fabs(q);
      acc_s[k][3] += q * q;
      acc_s[k][4] += q * q * q * q;
      acc_s[k][5] += qk2;
      acc_s[k][6] += 1.0;
    }
    __syncthreads();
  }
  // ---- write back ------------------------------------------------------------
  if (tid < m)
    for (int o = 0; o < EA_NOBS; ++o)
      S.acc[(((size_t)sample * C.n_bins + bin) * m + tid) * EA_NOBS + o] = acc_s[tid][o];
  for (uint32_t j = tid; j < 2 * n_sites; j += T) gw[j] = lat[j];
  if (tid < 64) {
    const int r = tid >> 5, k = tid & 31;
    if (k < m) {
      S.conf_at[((size_t)sample * 2 + r) * m + k] = (uint8_t)conf[r][k];
      S.labels[((size_t)sample * 2 + r) * m + k] = (uint8_t)lab[r][k];
    }
  }
  if (tid < m - 1) {
    S.swap_acc[(size_t)sample * (m - 1) + tid] += (long long)sw_acc[tid];
    S.swap_try[(size_t)sample * (m - 1) + tid] += (long long)sw_try[tid];
  }
  if (tid < m) {
    S.label_hist[((size_t)sample * m + tid) * 2 + 0] += (long long)lhist[tid][0];
    S.label_hist[((size_t)sample * m + tid) * 2 + 1] += (long long)lhist[tid][1];
  }
  if (tid < 2) S.trips[(size_t)sample * 2 + tid] += (long long)trip[tid];
}


template <int Z>
__global__ void __launch_bounds__(EA_THREADS) ea_pt_kernel(const __grid_constant__ EaParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lsample = blockIdx.x;
  const uint32_t key[2][2] = {{P.keys[lsample][0][0], P.keys[lsample][0][1]},
                              {P.keys[lsample][1][0], P.keys[lsample][1][1]}};
  CtlPoll poll;
  poll.start();
  ea_sample_run<Z>(P.C, P.S, P.sample0 + lsample, key, smem_raw, RunCtl{nullptr, nullptr, 0ull}, poll);
}

// A campaign: samples of several lattice sizes in one persistent launch.  Work
// item w is (set, sample) = work[w] (set << 24 | sample), largest lattices
// first; blocks take items from *queue until the list is done.
struct EaCampaignParams {
  EaCommon C;
  const EaSet* sets;
  const uint32_t* work;
  unsigned* queue;
  int n_work;
  RunCtl ctl;  // bounded run (null words: unbounded)
};

// T threads per block (ea_threads_for: the largest need of the campaign's sizes);
// 80 registers a thread allow 3 blocks of 256, 6 of 128 or 12 of 64 per SM.
template <int Z, int T>
__global__ void __launch_bounds__(T, T == 256 ? 3 : (T == 128 ? 6 : 12))
    ea_campaign_kernel(const __grid_constant__ EaCampaignParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int cur;
  CtlPoll poll;
  poll.start();
  for (;;) {
    if (threadIdx.x == 0) cur = poll.check(P.ctl) ? P.n_work : (int)atomicAdd(P.queue, 1u);
    __syncthreads();
    const int w = cur;
    __syncthreads();
    if (w >= P.n_work) break;
    const EaSet& S = P.sets[P.work[w] >> 24];
    const int sample = (int)(P.work[w] & 0xFFFFFFu);
    const uint32_t* k = S.keys + (size_t)sample * 4;
    const uint32_t key[2][2] = {{k[0], k[1]}, {k[2], k[3]}};
    ea_sample_run<Z, T>(P.C, S, sample, key, smem_raw, P.ctl, poll);
    __syncthreads();
  }
}

static thread_local EaParams g_ea;

}  // namespace critmc

using namespace critmc;

extern "C" int32_t critmc_pt_swap_table(int32_t m, const double* betas, int32_t width, uint32_t* out) {
  clear_error();
  if (!betas || !out || m < 2 || m > 32 || width < 2) return fail(CRITMC_ERR_INVALID, "need 2 <= m <= 32, width >= 2");
  for (int k = 0; k + 1 < m; ++k) {
    const double db = betas[k] - betas[k + 1];
    if (!(db < 0.0)) return fail(CRITMC_ERR_INVALID, "betas must increase strictly (temperatures hot -> cold)");
    for (int j = 0; j < width; ++j) {
      // energies of +-J configurations differ by multiples of 4: dE = 4 j
      const double p = j == 0 ? 1.0 : std::exp(db * 4.0 * j);
      const double t = std::nearbyint(std::ldexp(p, 32));
      out[(size_t)k * width + j] = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
    }
    if (out[(size_t)k * width + width - 1] != 0)
      return fail(CRITMC_ERR_INVALID, "swap table too narrow for these temperatures");
  }
  return CRITMC_OK;
}

extern "C" int32_t critmc_ea_coupling_bits(int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                           const double* couplings, uint8_t* jneg) {
  clear_error();
  ByteGeom g;
  int st = byte_geom(dim, lx, ly, lz, g);
  if (st) return st;
  if (dim < 2) return fail(CRITMC_ERR_UNSUPPORTED, "EA samples need dim 2 or 3");
  if (!couplings || !jneg) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  const int n = lx * g.ly * g.lz;
  auto site = [&](int x, int y, int z) { return x + lx * (y + g.ly * z); };
  // critmc lattice.py:147-149: bond index a*N + i is (i, i + e_a)
  auto jval = [&](int a, int i) { return couplings[(size_t)a * n + i]; };
  for (int c = 0; c < 2; ++c)
    for (uint32_t s = 0; s < g.slots; ++s) {
      const int r = (int)(s / g.hx), i = (int)(s % g.hx);
      const int y = r % g.ly, z = r / g.ly, p = (c + y + z) & 1, x = 2 * i + p;
      const int xp = (x + 1) % lx, xm = (x + lx - 1) % lx;
      const int yp = (y + 1) % g.ly, ym = (y + g.ly - 1) % g.ly;
      const int zp = (z + 1) % g.lz, zm = (z + g.lz - 1) % g.lz;
      const int me = site(x, y, z);
      // neighbour order of the colour-major layout: (x-side, other x-side, y-1, y+1, z-1, z+1)
      double jj[6];
      jj[0] = p ? jval(0, site(xm, y, z)) : jval(0, me);  // slot i: -x if p else +x
      jj[1] = p ? jval(0, me) : jval(0, site(xm, y, z));
      jj[2] = jval(1, site(x, ym, z));
      jj[3] = jval(1, me);
      jj[4] = dim == 3 ? jval(2, site(x, y, zm)) : 1.0;
      jj[5] = dim == 3 ? jval(2, me) : 1.0;
      (void)xp;
      (void)yp;
      (void)zp;
      uint8_t b = 0;
      for (int q = 0; q < 2 * dim; ++q) {
        if (jj[q] != 1.0 && jj[q] != -1.0) return fail(CRITMC_ERR_UNSUPPORTED, "couplings must be +-1");
        if (jj[q] < 0) b |= (uint8_t)(1u << q);
      }
      jneg[(size_t)c * g.slots + s] = b;
    }
  return CRITMC_OK;
}

namespace critmc {

// Validate the temperature set and step counts; fill the per-lane threshold planes.
static int ea_common(EaCommon& C, int dim, int m, const double* betas, const uint32_t* swap_thr,
                     int swap_width, uint32_t t0, int n_steps, int n_bins, int sweeps_per_step) {
  if (!betas || !swap_thr) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (dim < 2 || dim > 3) return fail(CRITMC_ERR_UNSUPPORTED, "EA samples need dim 2 or 3");
  if (m < 2 || m > 32) return fail(CRITMC_ERR_INVALID, "need 2 <= m <= 32 temperatures");
  if (n_steps < 0 || n_bins < 1 || n_bins > 31 || (long long)n_steps > (1LL << n_bins) - 1)
    return fail(CRITMC_ERR_INVALID, "need 0 <= n_steps <= 2^n_bins - 1 and 1 <= n_bins <= 31");
  if (sweeps_per_step < 1) return fail(CRITMC_ERR_INVALID, "sweeps_per_step must be >= 1");
  if (swap_width < 2) return fail(CRITMC_ERR_INVALID, "swap_width must be >= 2");
  if (((long long)t0 + n_steps) * sweeps_per_step > 0xFFFFFFFFLL)
    return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");
  for (int k = 0; k + 1 < m; ++k)
    if (!(betas[k] < betas[k + 1])) return fail(CRITMC_ERR_INVALID, "betas must increase (hot -> cold)");
  const int z = 2 * dim;
  // per-lane Metropolis thresholds exp(-beta_k (2z - 4v)), v = 0..z/2-1 unsatisfied bonds
  std::memset(C.planes, 0, sizeof(C.planes));
  for (int v = 0; v < z / 2; ++v)
    for (int k = 0; k < m; ++k) {
      if (!std::isfinite(betas[k]) || betas[k] <= 0.0) return fail(CRITMC_ERR_INVALID, "betas must be positive");
      const double p = std::exp(-betas[k] * (2.0 * z - 4.0 * v));
      const double tt = std::nearbyint(std::ldexp(p, 32));
      const uint32_t thr = tt >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)tt;
      for (int q = 0; q < 32; ++q)
        if ((thr >> (31 - q)) & 1u) C.planes[v][q] |= 1u << k;
    }
  C.swap_thr = swap_thr;
  C.m = m;
  C.n_steps = n_steps;
  C.n_bins = n_bins;
  C.sweeps_per_step = sweeps_per_step;
  C.swap_width = swap_width;
  C.t0 = t0;
  return CRITMC_OK;
}

// Validate one lattice size and fill its set (device pointers as given).
static int ea_set(EaSet& S, int dim, int lx, int ly, int lz, int n_samples, uint32_t* words,
                  const uint8_t* jneg, uint8_t* conf_at, uint8_t* labels, double* acc, int64_t* swap_acc,
                  int64_t* swap_try, int64_t* label_hist, int64_t* trips) {
  int st = byte_geom(dim, lx, ly, lz, S.g);
  if (st) return st;
  if (dim < 2) return fail(CRITMC_ERR_UNSUPPORTED, "EA samples need dim 2 or 3");
  if (2 * S.g.slots > (uint32_t)EA_MAX_SITES) return fail(CRITMC_ERR_UNSUPPORTED, "at most 4096 sites per sample");
  if (lx > EA_MAX_L || S.g.ly > EA_MAX_L || S.g.lz > EA_MAX_L) return fail(CRITMC_ERR_UNSUPPORTED, "extent too large");
  if (lx != S.g.ly || (dim == 3 && lx != S.g.lz))
    return fail(CRITMC_ERR_UNSUPPORTED, "EA samples use equal extents (one k_min table)");
  if (!words || !jneg || !conf_at || !labels || !acc || !swap_acc || !swap_try || !label_hist || !trips)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_samples < 1 || n_samples > (1 << 24)) return fail(CRITMC_ERR_INVALID, "need 1 <= n_samples <= 2^24");
  for (int x = 0; x < lx; ++x) {
    S.cosx[x] = std::cos(2.0 * M_PI * x / lx);
    S.sinx[x] = std::sin(2.0 * M_PI * x / lx);
  }
  S.ext[0] = lx;
  S.ext[1] = S.g.ly;
  S.ext[2] = S.g.lz;
  S.words = words;
  S.jneg = jneg;
  S.conf_at = conf_at;
  S.labels = labels;
  S.acc = acc;
  S.swap_acc = (long long*)swap_acc;
  S.swap_try = (long long*)swap_try;
  S.label_hist = (long long*)label_hist;
  S.trips = (long long*)trips;
  S.n_samples = n_samples;
  S.keys = nullptr;
  return CRITMC_OK;
}

}  // namespace critmc

extern "C" int32_t critmc_ea_pt_run(uint32_t* words, const uint8_t* jneg, int32_t dim, int32_t lx,
                                    int32_t ly, int32_t lz, int32_t m, int32_t n_samples,
                                    const uint32_t* keys, const double* betas,
                                    const uint32_t* swap_thr, int32_t swap_width, uint8_t* conf_at,
                                    uint8_t* labels, uint32_t t0, int32_t n_steps, int32_t n_bins,
                                    int32_t sweeps_per_step, double* acc, int64_t* swap_acc,
                                    int64_t* swap_try, int64_t* label_hist, int64_t* trips,
                                    void* stream) {
  clear_error();
  EaParams& P = g_ea;
  if (!keys) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  int st = ea_set(P.S, dim, lx, ly, lz, n_samples, words, jneg, conf_at, labels, acc, swap_acc, swap_try,
                  label_hist, trips);
  if (st) return st;
  if ((st = ea_common(P.C, dim, m, betas, swap_thr, swap_width, t0, n_steps, n_bins, sweeps_per_step)))
    return st;
  if (n_steps == 0) return CRITMC_OK;
  const size_t smem = ea_smem_bytes(P.S.g, dim, lx);
  cudaStream_t s = (cudaStream_t)stream;
  for (int c0 = 0; c0 < n_samples; c0 += EA_PSAMPLES) {
    const int nc = std::min(EA_PSAMPLES, n_samples - c0);
    P.sample0 = c0;
    std::memcpy(P.keys, keys + (size_t)c0 * 4, sizeof(uint32_t) * 4 * nc);
    auto launch = [&](auto kern) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      kern<<<nc, EA_THREADS, smem, s>>>(P);
    };
    if (dim == 2) launch(ea_pt_kernel<4>);
    else launch(ea_pt_kernel<6>);
    if (int e_ = cuda_check("launch")) return e_;
  }
  return CRITMC_OK;
}

extern "C" int64_t critmc_ea_campaign_buffer_bytes(int32_t n_sizes, int64_t total_samples) {
  if (n_sizes < 1 || total_samples < 1) return -1;
  return 256 + (int64_t)n_sizes * (int64_t)sizeof(EaSet) + 4 * total_samples;
}

extern "C" int32_t critmc_ea_campaign_run(const critmc_ea_size* sizes, int32_t n_sizes, int32_t dim, int32_t m,
                                          const double* betas, const uint32_t* swap_thr, int32_t swap_width,
                                          uint32_t t0, int32_t n_steps, int32_t n_bins, int32_t sweeps_per_step,
                                          void* buffer, int64_t buffer_bytes, void* staging, void* stream) {
  return critmc_ea_campaign_run_ctl(sizes, n_sizes, dim, m, betas, swap_thr, swap_width, t0, n_steps, n_bins,
                                    sweeps_per_step, buffer, buffer_bytes, staging, nullptr, stream);
}

extern "C" int32_t critmc_ea_campaign_run_ctl(const critmc_ea_size* sizes, int32_t n_sizes, int32_t dim,
                                              int32_t m, const double* betas, const uint32_t* swap_thr,
                                              int32_t swap_width, uint32_t t0, int32_t n_steps, int32_t n_bins,
                                              int32_t sweeps_per_step, void* buffer, int64_t buffer_bytes,
                                              void* staging, critmc_control* ctl, void* stream) {
  clear_error();
  if (!sizes || n_sizes < 1 || n_sizes > 255) return fail(CRITMC_ERR_INVALID, "need 1..255 lattice sizes");
  if (!buffer) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  EaCampaignParams P;
  P.ctl = control_device(ctl);
  int st = ea_common(P.C, dim, m, betas, swap_thr, swap_width, t0, n_steps, n_bins, sweeps_per_step);
  if (st) return st;
  std::vector<EaSet> sets(n_sizes);
  long long total = 0;
  size_t smem = 0;
  int threads = 64;
  for (int i = 0; i < n_sizes; ++i) {
    const critmc_ea_size& z = sizes[i];
    if (!z.keys) return fail(CRITMC_ERR_INVALID, "null pointer argument");
    if ((st = ea_set(sets[i], dim, z.lx, z.ly, z.lz, z.n_samples, z.words, z.jneg, z.conf_at, z.labels, z.acc,
                     z.swap_acc, z.swap_try, z.label_hist, z.trips)))
      return st;
    sets[i].keys = z.keys;
    total += z.n_samples;
    smem = std::max(smem, ea_smem_bytes(sets[i].g, dim, z.lx));
    threads = std::max(threads, ea_threads_for(sets[i].g, 2 * dim));
  }
  if (buffer_bytes < critmc_ea_campaign_buffer_bytes(n_sizes, total))
    return fail(CRITMC_ERR_INVALID, "campaign buffer too small");
  if (n_steps == 0) return CRITMC_OK;
  // host image of the buffer: [queue | sets | work], work sorted largest lattice first
  const size_t sets_off = 256, work_off = 256 + (size_t)n_sizes * sizeof(EaSet);
  const size_t bytes = work_off + 4 * (size_t)total;
  std::vector<unsigned char> own;
  unsigned char* img = static_cast<unsigned char*>(staging);
  if (!img) {
    own.resize(bytes);
    img = own.data();
  }
  std::memset(img, 0, sets_off);
  std::memcpy(img + sets_off, sets.data(), (size_t)n_sizes * sizeof(EaSet));
  std::vector<int> order(n_sizes);
  for (int i = 0; i < n_sizes; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sets[a].g.slots > sets[b].g.slots; });
  uint32_t* work = reinterpret_cast<uint32_t*>(img + work_off);
  size_t w = 0;
  for (int i : order)
    for (int smp = 0; smp < sets[i].n_samples; ++smp) work[w++] = ((uint32_t)i << 24) | (uint32_t)smp;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* dev = static_cast<unsigned char*>(buffer);
  if (cudaMemcpyAsync(dev, img, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return cuda_fail("copy campaign");
  P.queue = reinterpret_cast<unsigned*>(dev);
  P.sets = reinterpret_cast<const EaSet*>(dev + sets_off);
  P.work = reinterpret_cast<const uint32_t*>(dev + work_off);
  P.n_work = (int)total;
  auto launch = [&](auto kern, int nthreads) -> int {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return cuda_fail("shared memory attribute");
    int per_sm = 0, dev_id = 0, sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nthreads, smem);
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
    const long long grid = std::max(1LL, std::min<long long>(total, (long long)std::max(1, per_sm) * sms));
    kern<<<(unsigned)grid, nthreads, smem, s>>>(P);
    return cuda_check("launch");
  };
  if (dim == 2) {
    if (threads == 64) return launch(ea_campaign_kernel<4, 64>, 64);
    if (threads == 128) return launch(ea_campaign_kernel<4, 128>, 128);
    return launch(ea_campaign_kernel<4, 256>, 256);
  }
  if (threads == 64) return launch(ea_campaign_kernel<6, 64>, 64);
  if (threads == 128) return launch(ea_campaign_kernel<6, 128>, 128);
  return launch(ea_campaign_kernel<6, 256>, 256);
}
