// Flat-histogram random walks in energy space (Wang-Landau, multicanonical)
// for zero-field Ising and q-state Potts chains, one walker per thread: many
// walkers (seeds, energy windows) advance in one launch.
//
// A walker's moves are sequential, as in critmc: move t picks a random site,
// proposes a flip (Ising) or a different state (Potts), and accepts with
// min(1, w(new) / w(old)) inside its level window [lo, hi]; a move that would
// leave the window is rejected, and the current level is counted as for any
// rejected move.  Levels: Ising idx = (E_b + B) / 4, Potts idx = E + B (B the
// bond count).  Random words of move t of a walker: Philox(t mod 2^32,
// t / 2^32, 0x0A, 0) with the walker's key: word 0 the site ((w0 N) >> 32),
// word 1 the Potts proposal ((w1 (q-1)) >> 32, skipping the old state), words
// 2, 3 the 53-bit uniform u; a move is accepted if ln w(new) >= ln w(old) or
// ln u < ln w(new) - ln w(old), the probability min(1, w(new) / w(old)) of
// critmc's u < exp(ln w(new) - ln w(old)), with the log of fpmath.h, so a CPU
// replay follows bit for bit (this file is compiled without contraction).
//
// Replaces critmc src/critmc/kernels/flathist.py:28-132 (wl_ising, wl_potts,
// muca_ising, muca_potts).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fpmath.h"
#include "host_common.h"
#include "philox.h"

namespace critmc {

constexpr uint32_t TAG_FLATHIST = 0x0Au;
constexpr int FH_THREADS = 64;
constexpr int FH_STAGED_WALKERS = 32;  // walkers (threads) per block of the staged kernel

// Exact quotient i / d for 0 <= i < n by one multiply and shift: with
// 2^k >= n d and m = ceil(2^k / d), m d = 2^k + e (0 <= e < d) and
// i m / 2^k = i / d + i e / (d 2^k), whose second term is below 1/d, so the
// floor is that of i / d.  For n <= 2^24 the product stays below 2^50.
struct FhDiv {
  unsigned m;
  int k;
};

struct FhWalk {
  int8_t* spins;        // [w][N] critmc site order
  long long* idx;       // [w] current level
  long long* order;     // Ising: M [w]; Potts: counts [w][q]
  double* lng;          // [w][levels] WL: ln g (updated); MUCA: ln w (read)
  long long* hist;      // [w][levels]
  const int* window;    // [w][2]
  unsigned long long* trials;  // [w] moves done so far (the RNG counter)
  const double* ln_f;   // [w] WL constant ln f
  const double* n_levels;  // [w] WL 1/t mode: ln f = n_levels / (t0 + t + 1)
  const int* one_over_t;   // [w]
  const unsigned long long* t_base;  // [w] trials at the start of the Wang-Landau run
  const uint32_t* keys;    // [w][2]
  long long* idx_out;   // MUCA [w][n_meas]
  long long* order_out; // MUCA [w][n_meas] (Ising M, Potts sum_k n_k^2)
  int n_walkers, lx, ly, lz, dim, q, levels, n_meas;
  FhDiv div_x, div_y;   // exact division by lx and by ly
  long long moves;      // WL moves per walker; MUCA moves per measurement
  int smem_stride;      // staged kernel: shared-memory bytes per walker
};

static FhDiv fh_div_for(long long n, int d) {
  int k = 0;
  while ((1LL << k) < n * (long long)d) ++k;
  return FhDiv{(unsigned)(((1LL << k) + d - 1) / d), k};
}

__device__ __forceinline__ int fh_div(int i, FhDiv v) {
  return (int)(((unsigned long long)(unsigned)i * v.m) >> v.k);
}

// Single-precision decision of ln u < dw.  The estimate of ln u comes from
// the top 23 bits of word 2 as uf = 1.m - 1 (0 <= u - uf < 2^-23) and the
// hardware base-2 logarithm; it is used for uf >= 2^-12 only, where
// ln u - ln uf < 2^-23 / uf <= 2^-13 (1 + |ln uf|) and the logarithm adds a
// few 2^-22 (1 + |ln uf|).  With dwf = (float)dw (relative error 2^-24) and the
// margin M = 2^-12 (1 + |estimate|): if |estimate - dwf| > M, the errors cannot
// change the sign of ln u - dw (when |dwf| > 2 |estimate| + 2 the gap exceeds
// |dwf| / 2 + 1, far above them), so the float comparison is the decision of
// the double-precision test.  Otherwise (and for uf < 2^-12 or NaN, where the
// estimate is NaN) the move is decided with the double-precision log of
// fpmath.h.  The FP64 pipe is narrow on this part, so the common case keeps
// one subtraction and one conversion in double.
__device__ __forceinline__ float fh_log_estimate(const critmc_u32x4& r) {
  const float uf = __uint_as_float(0x3F800000u | (r.v[2] >> 9)) - 1.0f;
  return uf >= 0.000244140625f ? __log2f(uf) * 0.693147180559945309f : __int_as_float(0x7FC00000);
}

// neighbours of site i (periodic, first coordinate fastest)
template <int DIM>
__device__ __forceinline__ void fh_neighbours(const FhWalk& P, int i, int* nb) {
  const int q1 = fh_div(i, P.div_x);  // i / lx
  const int x = i - q1 * P.lx;
  nb[0] = x + 1 == P.lx ? i - (P.lx - 1) : i + 1;
  nb[1] = x == 0 ? i + (P.lx - 1) : i - 1;
  if (DIM >= 2) {
    const int q2 = fh_div(q1, P.div_y);  // i / (lx ly)
    const int y = q1 - q2 * P.ly;
    nb[2] = y + 1 == P.ly ? i - (P.ly - 1) * P.lx : i + P.lx;
    nb[3] = y == 0 ? i + (P.ly - 1) * P.lx : i - P.lx;
    if (DIM == 3) {
      const int plane = P.lx * P.ly;
      nb[4] = q2 + 1 == P.lz ? i - (P.lz - 1) * plane : i + plane;
      nb[5] = q2 == 0 ? i + (P.lz - 1) * plane : i - plane;
    }
  }
}

// One thread per walker.  The move body has no data-dependent branches, and
// everything that does not depend on the walk (the next move's Philox words,
// ln u and ln f) is computed one move ahead, so the serial chain of a move is
// the site loads, the level change, one load of ln g and one comparison.
// The entry of the current level and its pending visit count stay in
// registers until the walk leaves the level: the additions to ln g(idx) are
// the same, in the same order, as with a store after every move.
// HT, CT: histogram and count types (int64 in global memory; int32 in shared
// memory, where the histogram holds this launch's visits only)
template <int MODE, int POTTS, int DIM, typename HT, typename CT>  // MODE 0 Wang-Landau, 1 multicanonical
__device__ __forceinline__ void fh_walk(const FhWalk& P, int w, int8_t* s, double* lng, HT* hist, CT* counts) {
  constexpr int Z = 2 * DIM;
  const int n = P.lx * P.ly * P.lz;
  const int lo = P.window[2 * w], hi = P.window[2 * w + 1];
  const uint32_t k0 = P.keys[2 * w], k1 = P.keys[2 * w + 1];
  long long idx = P.idx[w];
  // a walker whose window leaves the level range, or whose level lies outside
  // its window, is left untouched (no access outside its arrays)
  if (lo < 0 || hi >= P.levels || lo > hi || idx < lo || idx > hi) return;
  unsigned long long t = P.trials[w];
  long long m = POTTS ? 0 : P.order[w];
  double cur = lng[idx];  // WL: ln g(idx); MUCA: ln w(idx)
  long long pending = 0;
  const bool one_over_t = MODE == 0 && P.one_over_t[w] != 0;
  const double lf_const = MODE == 0 ? P.ln_f[w] : 0.0;
  const double n_lev = MODE == 0 ? P.n_levels[w] : 0.0;
  const unsigned long long t0 = MODE == 0 ? P.t_base[w] : 0ull;
  // 1/t mode (Belardinelli-Pereyra): ln f = n_levels / (trials of this run + 1)
  auto ln_f_at = [&](unsigned long long tt) -> double {
    if (MODE != 0) return 0.0;
    if (one_over_t) return n_lev / ((double)(tt - t0) + 1.0);
    return lf_const;
  };
  critmc_u32x4 r = critmc_philox4x32((uint32_t)t, (uint32_t)(t >> 32), TAG_FLATHIST, 0u, k0, k1);
  float luf = fh_log_estimate(r);
  double lf = ln_f_at(t);
  const long long n_rounds = MODE == 0 ? 1 : P.n_meas;
  for (long long meas = 0; meas < n_rounds; ++meas) {
    for (long long j = 0; j < P.moves; ++j, ++t) {
      const unsigned long long tn = t + 1;
      const critmc_u32x4 rn = critmc_philox4x32((uint32_t)tn, (uint32_t)(tn >> 32), TAG_FLATHIST, 0u, k0, k1);
      const float lufn = fh_log_estimate(rn);
      const double lfn = ln_f_at(tn);
      const int i = (int)(((unsigned long long)r.v[0] * (unsigned)n) >> 32);
      int nb[Z];
      fh_neighbours<DIM>(P, i, nb);
      const int old = s[i];
      int nv, d;
      if (POTTS) {
        int ns = (int)(((unsigned long long)r.v[1] * (unsigned)(P.q - 1)) >> 32);
        ns += ns >= old;
        nv = ns;
        int n_old = 0, n_new = 0;
#pragma unroll
        for (int k = 0; k < Z; ++k) {
          const int v = s[nb[k]];
          n_old += v == old;
          n_new += v == ns;
        }
        d = n_old - n_new;
      } else {
        int field = 0;
#pragma unroll
        for (int k = 0; k < Z; ++k) field += s[nb[k]];
        nv = -old;
        // dE_b = 2 s_i h_i, one level per 4 (s h is even for even z)
        d = (old * field) / 2;
      }
      const long long nidx = idx + d;
      const bool inside = lo <= nidx && nidx <= hi;
      const long long cidx = inside ? nidx : idx;
      const double g_load = lng[cidx];
      const double g_new = cidx == idx ? cur : g_load;
      // ln w = -ln g (Wang-Landau) or the given weights (multicanonical);
      // ln u < ln w(new) - ln w(old) has probability min(1, w(new) / w(old))
      const double w_old = MODE == 0 ? -cur : cur;
      const double w_new = MODE == 0 ? -g_new : g_new;
      const double dw = w_new - w_old;
      const float dwf = (float)dw;
      bool acc = dwf >= 0.0f || luf < dwf;
      if (!(fabsf(luf - dwf) > (1.0f / 4096.0f) * (1.0f + fabsf(luf))))
        acc = w_new >= w_old || cm_log(critmc_u01_53(r.v[2], r.v[3])) < dw;
      acc = acc && inside;
      s[i] = (int8_t)(acc ? nv : old);
      if (POTTS) {
        if (acc && (unsigned)old < (unsigned)P.q) {  // spins outside 0..q-1 are not counted
          --counts[old];
          ++counts[nv];
        }
      } else {
        m += acc ? nv - old : 0;
      }
      const bool moved = acc && nidx != idx;
      if (moved) {
        if (MODE == 0) lng[idx] = cur;
        hist[idx] += (HT)pending;
        pending = 0;
      }
      cur = moved ? g_new : cur;
      idx = moved ? nidx : idx;
      if (MODE == 0) cur += lf;
      ++pending;
      r = rn;
      luf = lufn;
      lf = lfn;
    }
    if (MODE == 1) {
      P.idx_out[(size_t)w * P.n_meas + meas] = idx;
      long long o = m;
      if (POTTS) {
        o = 0;
        for (int k = 0; k < P.q; ++k) o += (long long)counts[k] * counts[k];
      }
      P.order_out[(size_t)w * P.n_meas + meas] = o;
    }
  }
  if (MODE == 0) lng[idx] = cur;
  hist[idx] += (HT)pending;
  P.idx[w] = idx;
  P.trials[w] = t;
  if (!POTTS) P.order[w] = m;
}

template <int MODE, int POTTS, int DIM>
__global__ void __launch_bounds__(FH_THREADS) fh_kernel_global(const __grid_constant__ FhWalk P) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.n_walkers) return;
  const size_t n = (size_t)P.lx * P.ly * P.lz;
  fh_walk<MODE, POTTS, DIM, long long, long long>(P, w, P.spins + w * n, P.lng + (size_t)w * P.levels,
                                                 P.hist + (size_t)w * P.levels,
                                                 POTTS ? P.order + (size_t)w * P.q : nullptr);
}

// The walkers of a block keep their spins, ln g (or ln w), histogram and Potts
// counts in shared memory for the whole launch: loads and stores of the move
// chain then never leave the SM.  Per walker, at a stride that is an odd
// number of 8-byte words (so the lanes of a warp spread over the banks):
// ln g [levels] double | this launch's visits [levels] int32 | counts [q] int32
// | spins [N] int8.  The host keeps a launch below 2^31 moves per walker.
template <int MODE, int POTTS, int DIM>
__global__ void __launch_bounds__(FH_STAGED_WALKERS) fh_kernel_staged(const __grid_constant__ FhWalk P) {
  extern __shared__ __align__(16) unsigned char fh_smem[];
  const int w0 = blockIdx.x * blockDim.x;
  const int nb = min((int)blockDim.x, P.n_walkers - w0);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int n = P.lx * P.ly * P.lz, L = P.levels, Q = POTTS ? P.q : 0;
  const int stride = P.smem_stride;
  const int off_hist = 8 * L, off_counts = 12 * L, off_spins = 12 * L + 4 * Q;
  // cooperative, coalesced copies of the block's contiguous span of each array
  for (int e = tid; e < nb * L; e += nt) {
    const int ww = e / L, k = e - ww * L;
    unsigned char* base = fh_smem + (size_t)ww * stride;
    reinterpret_cast<double*>(base)[k] = P.lng[(size_t)w0 * L + e];
    reinterpret_cast<int*>(base + off_hist)[k] = 0;
  }
  if constexpr (POTTS != 0) {
    for (int e = tid; e < nb * Q; e += nt) {
      const int ww = e / Q, k = e - ww * Q;
      reinterpret_cast<int*>(fh_smem + (size_t)ww * stride + off_counts)[k] = (int)P.order[(size_t)w0 * Q + e];
    }
  }
  for (int e = tid; e < nb * n; e += nt) {
    const int ww = e / n, k = e - ww * n;
    reinterpret_cast<int8_t*>(fh_smem + (size_t)ww * stride + off_spins)[k] = P.spins[(size_t)w0 * n + e];
  }
  __syncthreads();
  if (tid < nb) {
    unsigned char* base = fh_smem + (size_t)tid * stride;
    fh_walk<MODE, POTTS, DIM, int, int>(P, w0 + tid, reinterpret_cast<int8_t*>(base + off_spins),
                                        reinterpret_cast<double*>(base), reinterpret_cast<int*>(base + off_hist),
                                        POTTS ? reinterpret_cast<int*>(base + off_counts) : nullptr);
  }
  __syncthreads();
  for (int e = tid; e < nb * L; e += nt) {
    const int ww = e / L, k = e - ww * L;
    const unsigned char* base = fh_smem + (size_t)ww * stride;
    if (MODE == 0) P.lng[(size_t)w0 * L + e] = reinterpret_cast<const double*>(base)[k];
    P.hist[(size_t)w0 * L + e] += reinterpret_cast<const int*>(base + off_hist)[k];
  }
  if constexpr (POTTS != 0) {
    for (int e = tid; e < nb * Q; e += nt) {
      const int ww = e / Q, k = e - ww * Q;
      P.order[(size_t)w0 * Q + e] = reinterpret_cast<const int*>(fh_smem + (size_t)ww * stride + off_counts)[k];
    }
  }
  for (int e = tid; e < nb * n; e += nt) {
    const int ww = e / n, k = e - ww * n;
    P.spins[(size_t)w0 * n + e] = reinterpret_cast<const int8_t*>(fh_smem + (size_t)ww * stride + off_spins)[k];
  }
}

// Greedy descent into the window (critmc flathist.py:96-130, on the device):
// step j draws Philox(j mod 2^32, j / 2^32, 0x0C, 0) with the walker's key
// (word 0 the site, word 1 the Potts proposal, as for the walk) and keeps a
// move when the level does not move away from the window.  steps_out gets the
// number of steps taken, or -1 if the window was not reached in max_steps.
constexpr uint32_t TAG_DESCEND = 0x0Cu;

template <int POTTS, int DIM>
__global__ void __launch_bounds__(FH_THREADS) fh_descend_kernel(const __grid_constant__ FhWalk P,
                                                                long long* steps_out) {
  constexpr int Z = 2 * DIM;
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= P.n_walkers) return;
  const int n = P.lx * P.ly * P.lz;
  int8_t* s = P.spins + (size_t)w * n;
  const int lo = P.window[2 * w], hi = P.window[2 * w + 1];
  const uint32_t k0 = P.keys[2 * w], k1 = P.keys[2 * w + 1];
  long long idx = P.idx[w];
  long long m = POTTS ? 0 : P.order[w];
  long long* counts = POTTS ? P.order + (size_t)w * P.q : nullptr;
  long long used = -1;
  for (long long j = 0; j <= P.moves; ++j) {
    if (lo <= idx && idx <= hi) {
      used = j;
      break;
    }
    if (j == P.moves) break;
    const critmc_u32x4 r = critmc_philox4x32((uint32_t)j, (uint32_t)(j >> 32), TAG_DESCEND, 0u, k0, k1);
    const int i = (int)(((unsigned long long)r.v[0] * (unsigned)n) >> 32);
    int nb[Z];
    fh_neighbours<DIM>(P, i, nb);
    const int old = s[i];
    int nv, d;
    if (POTTS) {
      int ns = (int)(((unsigned long long)r.v[1] * (unsigned)(P.q - 1)) >> 32);
      ns += ns >= old;
      nv = ns;
      int n_old = 0, n_new = 0;
      for (int k = 0; k < Z; ++k) {
        const int v = s[nb[k]];
        n_old += v == old;
        n_new += v == ns;
      }
      d = n_old - n_new;
    } else {
      int field = 0;
      for (int k = 0; k < Z; ++k) field += s[nb[k]];
      nv = -old;
      d = (old * field) / 2;
    }
    const long long nidx = idx + d;
    if ((idx < lo && nidx >= idx) || (idx > hi && nidx <= idx)) {
      s[i] = (int8_t)nv;
      if (POTTS) {
        if ((unsigned)old < (unsigned)P.q) {
          --counts[old];
          ++counts[nv];
        }
      } else {
        m += nv - old;
      }
      idx = nidx;
    }
  }
  P.idx[w] = idx;
  if (!POTTS) P.order[w] = m;
  steps_out[w] = used;
}

template <int MODE, int POTTS, int DIM>
static int fh_launch(const FhWalk& P, bool staged, int wpb, cudaStream_t s) {
  if (!staged) {
    const int blocks = (P.n_walkers + FH_THREADS - 1) / FH_THREADS;
    fh_kernel_global<MODE, POTTS, DIM><<<blocks, FH_THREADS, 0, s>>>(P);
    return cuda_check("launch");
  }
  const size_t smem = (size_t)wpb * P.smem_stride;
  if (cudaFuncSetAttribute(fh_kernel_staged<MODE, POTTS, DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return cuda_fail("shared memory attribute");
  const int blocks = (P.n_walkers + wpb - 1) / wpb;
  fh_kernel_staged<MODE, POTTS, DIM><<<blocks, wpb, smem, s>>>(P);
  return cuda_check("launch");
}

template <int MODE, int POTTS>
static int fh_launch_dim(const FhWalk& P, bool staged, int wpb, cudaStream_t s) {
  if (P.dim == 1) return fh_launch<MODE, POTTS, 1>(P, staged, wpb, s);
  if (P.dim == 2) return fh_launch<MODE, POTTS, 2>(P, staged, wpb, s);
  return fh_launch<MODE, POTTS, 3>(P, staged, wpb, s);
}

}  // namespace critmc

using namespace critmc;

static int fh_check(int dim, int lx, int ly, int lz, int q, int n_walkers, int levels) {
  if (dim < 1 || dim > 3 || lx < 2 || (dim >= 2 && ly < 2) || (dim == 3 && lz < 2))
    return fail(CRITMC_ERR_INVALID, "bad lattice extents");
  if (q != 0 && (q < 2 || q > 127)) return fail(CRITMC_ERR_INVALID, "q must be 0 (Ising) or 2..127");
  if (n_walkers < 1 || levels < 2) return fail(CRITMC_ERR_INVALID, "need walkers and levels");
  if ((long long)lx * ly * lz > (1LL << 24)) return fail(CRITMC_ERR_INVALID, "at most 2^24 sites per walker");
  return CRITMC_OK;
}

extern "C" int32_t critmc_fh_run(int32_t mode, int8_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                 int32_t q, int32_t n_walkers, const uint32_t* keys, int32_t levels,
                                 int64_t* idx, int64_t* order, double* lng, int64_t* hist, const int32_t* window,
                                 uint64_t* trials, const double* ln_f, const double* n_levels,
                                 const int32_t* one_over_t, const uint64_t* t_base, int64_t moves,
                                 int32_t n_meas, int64_t* idx_out,
                                 int64_t* order_out, void* stream) {
  clear_error();
  if (dim < 2) ly = 1;
  if (dim < 3) lz = 1;
  int st = fh_check(dim, lx, ly, lz, q, n_walkers, levels);
  if (st) return st;
  const bool force_global = (mode & 0x10) != 0, force_shared = (mode & 0x20) != 0;
  mode &= ~0x30;
  if (mode != 0 && mode != 1) return fail(CRITMC_ERR_INVALID, "mode must be 0 (Wang-Landau) or 1 (multicanonical)");
  if (!spins || !keys || !idx || !order || !lng || !hist || !window || !trials)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (mode == 0 && (!ln_f || !n_levels || !one_over_t || !t_base))
    return fail(CRITMC_ERR_INVALID, "Wang-Landau needs ln_f, n_levels, one_over_t, t_base");
  if (mode == 1 && (n_meas < 0 || (n_meas > 0 && (!idx_out || !order_out))))
    return fail(CRITMC_ERR_INVALID, "multicanonical runs need idx_out and order_out");
  if (moves < 0) return fail(CRITMC_ERR_INVALID, "moves must not be negative");
  FhWalk P;
  P.spins = spins;
  P.idx = (long long*)idx;
  P.order = (long long*)order;
  P.lng = lng;
  P.hist = (long long*)hist;
  P.window = window;
  P.trials = (unsigned long long*)trials;
  P.ln_f = ln_f;
  P.n_levels = n_levels;
  P.one_over_t = one_over_t;
  P.t_base = (const unsigned long long*)t_base;
  P.keys = keys;
  P.idx_out = (long long*)idx_out;
  P.order_out = (long long*)order_out;
  P.n_walkers = n_walkers;
  P.lx = lx;
  P.ly = ly;
  P.lz = lz;
  P.dim = dim;
  P.q = q;
  P.levels = levels;
  P.n_meas = mode == 1 ? n_meas : 1;
  P.div_x = fh_div_for((long long)lx * ly * lz, lx);
  P.div_y = fh_div_for((long long)lx * ly * lz, ly);
  P.moves = moves;
  // Stage the walkers in shared memory when they can all be resident at once
  // that way, or when at least 256 fit an SM; otherwise (large lattices, many
  // walkers) the register-limited global-memory kernel keeps more in flight.
  const long long n = (long long)lx * ly * lz;
  long long stride = (12LL * levels + 4LL * (q ? q : 0) + n + 7) / 8 * 8;
  if ((stride / 8) % 2 == 0) stride += 8;
  const long long per_walker_moves = moves * (long long)P.n_meas;
  int dev = 0, smem_max = 0, smem_sm = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return cuda_fail("device attributes");
  const long long fit = smem_max / stride;
  const int wpb = (int)std::min<long long>(FH_STAGED_WALKERS, std::max<long long>(fit, 1));
  // resident walkers per SM: whole blocks, each with 1 KB of shared memory reserved
  const long long per_sm = wpb * (smem_sm / (wpb * stride + 1024));
  const bool can_stage = fit >= 1 && per_walker_moves < (1LL << 31);
  if (force_shared && !can_stage)
    return fail(CRITMC_ERR_INVALID, "a walker does not fit in shared memory, or 2^31 moves or more in one call");
  const bool staged = force_shared || (!force_global && can_stage && (per_sm >= 256 || per_sm * sms >= n_walkers));
  P.smem_stride = (int)std::min<long long>(stride, 1 << 30);
  cudaStream_t s = (cudaStream_t)stream;
  if (mode == 0) return q == 0 ? fh_launch_dim<0, 0>(P, staged, wpb, s) : fh_launch_dim<0, 1>(P, staged, wpb, s);
  return q == 0 ? fh_launch_dim<1, 0>(P, staged, wpb, s) : fh_launch_dim<1, 1>(P, staged, wpb, s);
}

extern "C" int32_t critmc_fh_descend(int8_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz, int32_t q,
                                     int32_t n_walkers, const uint32_t* keys, int32_t levels, int64_t* idx,
                                     int64_t* order, const int32_t* window, int64_t max_steps, int64_t* steps_out,
                                     void* stream) {
  clear_error();
  if (dim < 2) ly = 1;
  if (dim < 3) lz = 1;
  int st = fh_check(dim, lx, ly, lz, q, n_walkers, levels);
  if (st) return st;
  if (!spins || !keys || !idx || !order || !window || !steps_out) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (max_steps < 0) return fail(CRITMC_ERR_INVALID, "max_steps must not be negative");
  FhWalk P;
  std::memset(&P, 0, sizeof(P));
  P.spins = spins;
  P.idx = (long long*)idx;
  P.order = (long long*)order;
  P.window = window;
  P.keys = keys;
  P.n_walkers = n_walkers;
  P.lx = lx;
  P.ly = ly;
  P.lz = lz;
  P.dim = dim;
  P.q = q;
  P.levels = levels;
  P.moves = max_steps;
  P.div_x = fh_div_for((long long)lx * ly * lz, lx);
  P.div_y = fh_div_for((long long)lx * ly * lz, ly);
  const int blocks = (n_walkers + FH_THREADS - 1) / FH_THREADS;
  cudaStream_t s = (cudaStream_t)stream;
  long long* so = (long long*)steps_out;
  if (q == 0) {
    if (dim == 1) fh_descend_kernel<0, 1><<<blocks, FH_THREADS, 0, s>>>(P, so);
    else if (dim == 2) fh_descend_kernel<0, 2><<<blocks, FH_THREADS, 0, s>>>(P, so);
    else fh_descend_kernel<0, 3><<<blocks, FH_THREADS, 0, s>>>(P, so);
  } else {
    if (dim == 1) fh_descend_kernel<1, 1><<<blocks, FH_THREADS, 0, s>>>(P, so);
    else if (dim == 2) fh_descend_kernel<1, 2><<<blocks, FH_THREADS, 0, s>>>(P, so);
    else fh_descend_kernel<1, 3><<<blocks, FH_THREADS, 0, s>>>(P, so);
  }
  return cuda_check("launch");
}
