// Cluster updates (Swendsen-Wang, Wolff) for Ising and q-state Potts chains
// on the byte (int8) and multi-spin-coded (bit) layouts.
//
// Sites are numbered by their colour-major layout index u = colour * slots +
// row * (lx/2) + i (for the bit layout, site u is bit u % 32 of word u / 32).
// A bond is (colour-0 site s, direction q) with q in the neighbour order of
// byte_neighbours; it is active when both ends agree and word q % 4 of
// Philox(s, sweep, 0x07 | (q/4) << 8, 0) is below round(p 2^32), p = 1 - e^{-2 beta}
// (Ising) or 1 - e^{-beta} (Potts).  Clusters are the connected components of
// the active bonds, found with a lock-free union-find that always links the
// larger root under the smaller one, so every cluster's root is its smallest
// site index whatever the thread order.  Swendsen-Wang draws per root r
// Philox(r, sweep, 0x08, 0): Ising flips the cluster if word 0 >= 2^31, Potts
// gives it state (word 0 * q) >> 32.  Wolff picks the seed site
// (word 0 * N) >> 32 of Philox(0, sweep, 0x09, 0) and flips its cluster (Potts:
// new state (old + 1 + ((word 1 * (q - 1)) >> 32)) mod q).  Energy and
// magnetisation (or Potts counts) are updated exactly from the changed bonds
// and sites.
//
// O(n) chains (FP32 unit spins, colour-major structure of arrays) use the
// embedded Ising model of a random axis r: Philox(0, sweep, 0x0B, 0) gives r
// (XY: angle 2 pi u0; Heisenberg: z = 2 u0 - 1 and angle 2 pi u1, uniform on
// the sphere), p_i = S_i . r, a bond is active when p_i p_j > 0 and the 24-bit
// uniform of its word is below 1 - exp(-2 beta p_i p_j), and a flipped
// cluster is reflected, S_i <- S_i - 2 p_i r.  The float arithmetic uses
// fpmath.h and this file is compiled without contraction, so the CPU replay
// follows bit for bit.
//
// Replaces critmc src/critmc/kernels/ising.py:111-171 (wolff_update,
// sw_update), kernels/potts.py:107-168 and kernels/on.py:265-345; statistics
// as critmc's aux columns (kernels/common.py:35-39: summed Wolff size, SW
// sum |C|^2 and cluster count).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "fpmath.h"
#include "geom.cuh"
#include "host_common.h"

namespace critmc {

constexpr int CL_THREADS = 256;
static_assert(CL_THREADS % 32 == 0, "the decide kernel's warp-uniform loop needs whole warps");
constexpr int CL_PCHAINS = 256;
constexpr uint32_t TAG_BOND = 0x07u, TAG_CLFLIP = 0x08u, TAG_WOLFF = 0x09u, TAG_ONAXIS = 0x0Bu;

struct ClParams {
  void* spins;
  int* label;            // [n_chains][N]
  int8_t* newv;          // [n_chains][N]
  int* size;             // [n_chains][N]
  long long* running;    // Ising [n][2] (E_b, M); Potts energy [n]
  long long* counts;     // Potts [n][q]
  long long* stats;      // [n][3]: += Wolff size; = SW sum |C|^2, cluster count
  ByteGeom g;
  uint32_t n;            // sites per chain (2 slots)
  int bits;              // 1: bit layout, 0: int8
  int potts, q, algo, chain0;
  int on_n;              // O(n) chains: components (2, 3); 0 for Ising / Potts
  float* proj;           // O(n): [n_chains][N] projections on the axis
  float nb2;             // O(n): -2 beta
  uint32_t thr, sweep;
  uint32_t keys[CL_PCHAINS][2];
};

__device__ __forceinline__ int cl_val(const ClParams& P, int chain, uint32_t u) {
  if (P.bits) {
    const uint32_t* w = static_cast<const uint32_t*>(P.spins) + (size_t)chain * (P.n >> 5);
    return ((w[u >> 5] >> (u & 31)) & 1u) ? 1 : -1;
  }
  return static_cast<const int8_t*>(P.spins)[(size_t)chain * P.n + u];
}

// root of x with path halving; labels only ever point to smaller indices
__device__ __forceinline__ int cl_find(int* L, int x) {
  for (;;) {
    const int p = L[x];
    if (p == x) return x;
    const int gp = L[p];
    if (gp != p) L[x] = gp;
    x = gp;
  }
}

__device__ __forceinline__ void cl_unite(int* L, int a, int b) {
  for (;;) {  // each pass either finishes or moves b to a strictly smaller root
    a = cl_find(L, a);
    b = cl_find(L, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(&L[b], a);
    if (old == b) return;
    b = old;
  }
}

// the reflection axis of an O(n) chain for this update
__device__ __forceinline__ void cl_axis(const ClParams& P, int lchain, float* r) {
  const critmc_u32x4 w = critmc_philox4x32(0u, P.sweep, TAG_ONAXIS, 0u, P.keys[lchain][0], P.keys[lchain][1]);
  const float two_pi = 6.28318530717958647692f;
  float sn, cs;
  if (P.on_n == 2) {
    cm_sincosf(two_pi * critmc_u01f(w.v[0]), &sn, &cs);
    r[0] = cs;
    r[1] = sn;
    r[2] = 0.0f;
  } else {
    const float z = 2.0f * critmc_u01f(w.v[0]) - 1.0f;
    const float rho = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    cm_sincosf(two_pi * critmc_u01f(w.v[1]), &sn, &cs);
    r[0] = rho * cs;
    r[1] = rho * sn;
    r[2] = z;
  }
}

__device__ __forceinline__ const float* cl_on_spins(const ClParams& P, int chain) {
  return static_cast<const float*>(P.spins) + (size_t)chain * P.on_n * P.n;
}

__global__ void cl_init_kernel(ClParams P) {
  const int lchain = blockIdx.y, chain = P.chain0 + lchain;
  int* L = P.label + (size_t)chain * P.n;
  float r[3];
  if (P.on_n) cl_axis(P, lchain, r);
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < P.n; u += gridDim.x * blockDim.x) {
    L[u] = (int)u;
    if (P.on_n) {
      const float* S = cl_on_spins(P, chain);
      float p = S[u] * r[0] + S[P.n + u] * r[1];
      if (P.on_n == 3) p = p + S[2 * (size_t)P.n + u] * r[2];
      P.proj[(size_t)chain * P.n + u] = p;
    }
  }
}

template <int Z>
__global__ void __launch_bounds__(CL_THREADS) cl_link_kernel(const __grid_constant__ ClParams P) {
  const int lchain = blockIdx.y, chain = P.chain0 + lchain;
  int* L = P.label + (size_t)chain * P.n;
  const uint32_t k0 = P.keys[lchain][0], k1 = P.keys[lchain][1];
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P.g.slots; s += gridDim.x * blockDim.x) {
    int r, i;
    byte_row_index(P.g, s, r, i);
    uint32_t nb[Z];
    byte_neighbours<Z>(P.g, 0, r, i, nb);
    const critmc_u32x4 w0 = critmc_philox4x32(s, P.sweep, TAG_BOND, 0u, k0, k1);
    critmc_u32x4 w1 = w0;
    if constexpr (Z == 6) w1 = critmc_philox4x32(s, P.sweep, TAG_BOND | (1u << 8), 0u, k0, k1);
    if (P.on_n) {
      const float* pr = P.proj + (size_t)chain * P.n;
      const float p0 = pr[s];
#pragma unroll
      for (int q = 0; q < Z; ++q) {
        const uint32_t u1 = P.g.slots + nb[q];
        const uint32_t word = q < 4 ? w0.v[q] : w1.v[q - 4];
        const float x = p0 * pr[u1];
        if (x > 0.0f && critmc_u01f(word) < 1.0f - cm_expf(P.nb2 * x)) cl_unite(L, (int)s, (int)u1);
      }
      continue;
    }
    const int v0 = cl_val(P, chain, s);
#pragma unroll
    for (int q = 0; q < Z; ++q) {
      const uint32_t u1 = P.g.slots + nb[q];
      const uint32_t word = q < 4 ? w0.v[q] : w1.v[q - 4];
      if (word < P.thr && cl_val(P, chain, u1) == v0) cl_unite(L, (int)s, (int)u1);
    }
  }
}

__global__ void cl_flatten_kernel(ClParams P) {
  const int chain = P.chain0 + blockIdx.y;
  int* L = P.label + (size_t)chain * P.n;
  int* S = P.size + (size_t)chain * P.n;
  // read-only walk: a path-halving store here could overwrite another site's
  // final root with an intermediate label after that site's thread wrote it
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < P.n; u += gridDim.x * blockDim.x) {
    int r = (int)u;
    for (int p = L[r]; p != r; p = L[r]) r = p;
    L[u] = r;
    S[u] = 0;
  }
}

// new value of every site; SW cluster sizes; Wolff size
__global__ void __launch_bounds__(CL_THREADS) cl_decide_kernel(const __grid_constant__ ClParams P) {
  const int lchain = blockIdx.y, chain = P.chain0 + lchain;
  const int* L = P.label + (size_t)chain * P.n;
  int8_t* nv = P.newv + (size_t)chain * P.n;
  int* S = P.size + (size_t)chain * P.n;
  const uint32_t k0 = P.keys[lchain][0], k1 = P.keys[lchain][1];
  int root = -1, wnew = 0;
  if (P.algo == CRITMC_WOLFF) {
    const critmc_u32x4 w = critmc_philox4x32(0u, P.sweep, TAG_WOLFF, 0u, k0, k1);
    const uint32_t seed = (uint32_t)(((unsigned long long)w.v[0] * P.n) >> 32);
    root = L[seed];
    if (!P.on_n) {
      const int old = cl_val(P, chain, seed);
      wnew = P.potts ? (old + 1 + (int)(((unsigned long long)w.v[1] * (unsigned)(P.q - 1)) >> 32)) % P.q : -old;
    }
  }
  long long flipped = 0;
  // warp-uniform loop (blockDim is a multiple of 32): every lane takes part in
  // the match below on every pass
  for (uint32_t base = blockIdx.x * blockDim.x; base < P.n; base += gridDim.x * blockDim.x) {
    const uint32_t u = base + threadIdx.x;
    const bool valid = u < P.n;
    const int r = valid ? L[u] : -1;
    if (P.algo == CRITMC_SWENDSEN_WANG) {
      // one atomic per group of lanes with the same root: the root of a giant
      // cluster would otherwise take one atomic per site
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, r);
      if (valid && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&S[r], __popc(peers));
    }
    if (!valid) continue;
    if (P.on_n) {  // O(n): newv is the reflect flag
      int f = 0;
      if (P.algo == CRITMC_WOLFF) {
        f = r == root;
        flipped += f;
      } else {
        f = (int)(critmc_philox4x32((uint32_t)r, P.sweep, TAG_CLFLIP, 0u, k0, k1).v[0] >> 31);
      }
      nv[u] = (int8_t)f;
      continue;
    }
    const int old = cl_val(P, chain, u);
    int v = old;
    if (P.algo == CRITMC_WOLFF) {
      if (r == root) {
        v = wnew;
        ++flipped;
      }
    } else {
      const uint32_t w = critmc_philox4x32((uint32_t)r, P.sweep, TAG_CLFLIP, 0u, k0, k1).v[0];
      v = P.potts ? (int)(((unsigned long long)w * (unsigned)P.q) >> 32) : ((w >> 31) ? -old : old);
    }
    nv[u] = (int8_t)v;
  }
  if (P.algo == CRITMC_WOLFF) {
    flipped = warp_sum(flipped);
    if ((threadIdx.x & 31) == 0 && flipped) atomicAdd(reinterpret_cast<unsigned long long*>(P.stats + 3 * chain), as_ull(flipped));
  }
}

// SW statistics describe the last decomposition: clear them first
__global__ void cl_sw_clear_kernel(long long* stats, int c0, int nc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nc) {
    stats[3 * (size_t)(c0 + c) + 1] = 0;
    stats[3 * (size_t)(c0 + c) + 2] = 0;
  }
}

// block sum of one value per thread (blockDim a multiple of 32, at most 1024);
// the result is valid in thread 0
__device__ __forceinline__ long long cl_block_sum(long long v, long long* red) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  long long t = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

// SW statistics: sum |C|^2 and the number of clusters (roots have L[u] == u);
// one atomic per block and counter (a per-warp atomic on the same two
// addresses serialises thousands of them)
__global__ void cl_sw_stats_kernel(ClParams P) {
  const int chain = P.chain0 + blockIdx.y;
  const int* L = P.label + (size_t)chain * P.n;
  const int* S = P.size + (size_t)chain * P.n;
  long long c2 = 0, ncl = 0;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < P.n; u += gridDim.x * blockDim.x)
    if (L[u] == (int)u) {
      c2 += (long long)S[u] * S[u];
      ++ncl;
    }
  __shared__ long long red[32];
  c2 = cl_block_sum(c2, red);
  ncl = cl_block_sum(ncl, red);
  if (threadIdx.x == 0) {
    unsigned long long* st = reinterpret_cast<unsigned long long*>(P.stats + 3 * chain);
    if (c2) atomicAdd(st + 1, as_ull(c2));
    if (ncl) atomicAdd(st + 2, as_ull(ncl));
  }
}

// energy change over the bonds (colour-0 sites see every bond once)
template <int Z>
__global__ void __launch_bounds__(CL_THREADS) cl_delta_kernel(const __grid_constant__ ClParams P) {
  const int chain = P.chain0 + blockIdx.y;
  const int8_t* nv = P.newv + (size_t)chain * P.n;
  long long de = 0;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P.g.slots; s += gridDim.x * blockDim.x) {
    int r, i;
    byte_row_index(P.g, s, r, i);
    uint32_t nb[Z];
    byte_neighbours<Z>(P.g, 0, r, i, nb);
    const int o0 = cl_val(P, chain, s), n0 = nv[s];
#pragma unroll
    for (int q = 0; q < Z; ++q) {
      const uint32_t u1 = P.g.slots + nb[q];
      const int o1 = cl_val(P, chain, u1), n1 = nv[u1];
      if (P.potts) de += (long long)(o0 == o1) - (long long)(n0 == n1);  // E = -#equal bonds
      else de += (long long)o0 * o1 - (long long)n0 * n1;                // E_b = -sum s s
    }
  }
  __shared__ long long red[32];
  de = cl_block_sum(de, red);  // one atomic per block
  if (threadIdx.x == 0 && de) {
    long long* e = P.potts ? P.running + chain : P.running + 2 * chain;
    atomicAdd(reinterpret_cast<unsigned long long*>(e), as_ull(de));
  }
}

// write the new values; magnetisation (Ising) or counts (Potts) changes
__global__ void __launch_bounds__(CL_THREADS) cl_apply_kernel(const __grid_constant__ ClParams P) {
  const int chain = P.chain0 + blockIdx.y;
  const int8_t* nv = P.newv + (size_t)chain * P.n;
  __shared__ int hist[2][128];
  if (P.potts)
    for (int k = threadIdx.x; k < 2 * 128; k += blockDim.x) (&hist[0][0])[k] = 0;
  __syncthreads();
  long long dm = 0;
  if (P.bits) {  // one thread per word: no two threads touch a word
    uint32_t* w = static_cast<uint32_t*>(P.spins) + (size_t)chain * (P.n >> 5);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < (P.n >> 5); k += gridDim.x * blockDim.x) {
      uint32_t m = 0;
      const uint32_t old = w[k];
      for (int b = 0; b < 32; ++b) {
        const uint32_t bit = nv[32 * k + b] > 0 ? 1u : 0u;
        m |= bit << b;
      }
      dm += 2LL * (__popc(m & ~old) - __popc(old & ~m));
      w[k] = m;
    }
  } else {
    int8_t* s = static_cast<int8_t*>(P.spins) + (size_t)chain * P.n;
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < P.n; u += gridDim.x * blockDim.x) {
      const int o = s[u], v = nv[u];
      if (o == v) continue;
      s[u] = (int8_t)v;
      if (P.potts) {
        atomicSub(&hist[0][o], 1);
        atomicAdd(&hist[1][v], 1);
      } else {
        dm += v - o;
      }
    }
  }
  if (P.potts) {
    __syncthreads();
    long long* c = P.counts + (size_t)chain * P.q;
    for (int k = threadIdx.x; k < P.q; k += blockDim.x) {
      const int d = hist[0][k] + hist[1][k];
      if (d) atomicAdd(reinterpret_cast<unsigned long long*>(c + k), as_ull((long long)d));
    }
  } else {
    dm = warp_sum(dm);
    if ((threadIdx.x & 31) == 0 && dm) atomicAdd(reinterpret_cast<unsigned long long*>(P.running + 2 * chain + 1), as_ull(dm));
  }
}

// O(n): reflect the spins of the flipped clusters, S <- S - 2 p r
__global__ void __launch_bounds__(CL_THREADS) cl_on_apply_kernel(const __grid_constant__ ClParams P) {
  const int lchain = blockIdx.y, chain = P.chain0 + lchain;
  const int8_t* nv = P.newv + (size_t)chain * P.n;
  const float* pr = P.proj + (size_t)chain * P.n;
  float* S = static_cast<float*>(P.spins) + (size_t)chain * P.on_n * P.n;
  float r[3];
  cl_axis(P, lchain, r);
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < P.n; u += gridDim.x * blockDim.x) {
    if (!nv[u]) continue;
    const float tp = 2.0f * pr[u];
    for (int c = 0; c < P.on_n; ++c) S[(size_t)c * P.n + u] = S[(size_t)c * P.n + u] - tp * r[c];
  }
}

static int cl_launch(ClParams& P, int n_chains, const uint32_t* keys, cudaStream_t s) {
  const unsigned bx_sites = std::min<unsigned>(4096, (P.n + CL_THREADS - 1) / CL_THREADS);
  const unsigned bx_slots = std::min<unsigned>(4096, (P.g.slots + CL_THREADS - 1) / CL_THREADS);
  const unsigned bx_words = std::min<unsigned>(4096, ((P.n >> 5) + CL_THREADS - 1) / CL_THREADS);
  for (int c0 = 0; c0 < n_chains; c0 += CL_PCHAINS) {
    const int nc = std::min(CL_PCHAINS, n_chains - c0);
    P.chain0 = c0;
    std::memcpy(P.keys, keys + 2 * (size_t)c0, sizeof(uint32_t) * 2 * nc);
    if (P.algo == CRITMC_SWENDSEN_WANG) cl_sw_clear_kernel<<<(nc + 127) / 128, 128, 0, s>>>(P.stats, c0, nc);
    const dim3 gs(bx_sites, nc), gb(bx_slots, nc), gw(std::max(1u, bx_words), nc);
    // the reductions run on at most 2 blocks per SM: fewer same-address atomics
    const dim3 gs_red(std::min(bx_sites, 296u), nc), gb_red(std::min(bx_slots, 296u), nc);
    cl_init_kernel<<<gs, CL_THREADS, 0, s>>>(P);
    if (P.g.dim == 1) cl_link_kernel<2><<<gb, CL_THREADS, 0, s>>>(P);
    else if (P.g.dim == 2) cl_link_kernel<4><<<gb, CL_THREADS, 0, s>>>(P);
    else cl_link_kernel<6><<<gb, CL_THREADS, 0, s>>>(P);
    cl_flatten_kernel<<<gs, CL_THREADS, 0, s>>>(P);
    cl_decide_kernel<<<gs, CL_THREADS, 0, s>>>(P);
    if (P.algo == CRITMC_SWENDSEN_WANG) cl_sw_stats_kernel<<<gs_red, CL_THREADS, 0, s>>>(P);
    if (P.on_n) {
      cl_on_apply_kernel<<<gs, CL_THREADS, 0, s>>>(P);
    } else {
      if (P.g.dim == 1) cl_delta_kernel<2><<<gb_red, CL_THREADS, 0, s>>>(P);
      else if (P.g.dim == 2) cl_delta_kernel<4><<<gb_red, CL_THREADS, 0, s>>>(P);
      else cl_delta_kernel<6><<<gb_red, CL_THREADS, 0, s>>>(P);
      cl_apply_kernel<<<P.bits ? gw : gs, CL_THREADS, 0, s>>>(P);
    }
    if (int e = cuda_check("launch")) return e;
  }
  return CRITMC_OK;
}

}  // namespace critmc

using namespace critmc;

extern "C" int64_t critmc_cluster_scratch_bytes(int32_t n_chains, int64_t n_sites) {
  if (n_chains < 1 || n_sites < 2) return -1;
  return (int64_t)n_chains * n_sites * (4 + 4 + 4 + 1) + 256;
}

extern "C" int32_t critmc_cluster_update(int32_t bits, void* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                         int32_t q, int32_t n_chains, const uint32_t* keys, double beta, int32_t algo,
                                         uint32_t sweep, int64_t* running, int64_t* counts, int64_t* stats,
                                         void* scratch, void* stream) {
  clear_error();
  static thread_local ClParams P;
  int st = byte_geom(dim, lx, ly, lz, P.g);
  if (st) return st;
  if (!spins || !keys || !running || !stats || !scratch) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (algo != CRITMC_WOLFF && algo != CRITMC_SWENDSEN_WANG) return fail(CRITMC_ERR_INVALID, "algo must be wolff or sw");
  if (n_chains < 1) return fail(CRITMC_ERR_INVALID, "need n_chains >= 1");
  if (!(beta >= 0.0) || !std::isfinite(beta)) return fail(CRITMC_ERR_INVALID, "beta must be finite and >= 0");
  const bool potts = q > 0;
  if (potts && (q < 2 || q > 127 || !counts)) return fail(CRITMC_ERR_INVALID, "Potts needs 2 <= q <= 127 and counts");
  if (potts && bits) return fail(CRITMC_ERR_UNSUPPORTED, "Potts chains use the int8 layout");
  P.n = 2 * P.g.slots;
  if (bits && (P.g.hx % 32)) return fail(CRITMC_ERR_UNSUPPORTED, "bit layout needs lx a multiple of 64");
  if ((long long)P.n * n_chains >= (1LL << 31)) return fail(CRITMC_ERR_UNSUPPORTED, "too many sites");
  const double p = -std::expm1(-(potts ? 1.0 : 2.0) * beta);
  const double t = std::nearbyint(std::ldexp(p, 32));
  P.thr = t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
  P.spins = spins;
  P.bits = bits ? 1 : 0;
  P.potts = potts ? 1 : 0;
  P.q = potts ? q : 2;
  P.algo = algo;
  P.sweep = sweep;
  P.running = (long long*)running;
  P.counts = (long long*)counts;
  P.stats = (long long*)stats;
  char* base = static_cast<char*>(scratch);
  P.label = reinterpret_cast<int*>(base);
  P.size = reinterpret_cast<int*>(base + (size_t)n_chains * P.n * 4);
  P.proj = reinterpret_cast<float*>(base + (size_t)n_chains * P.n * 8);
  P.newv = reinterpret_cast<int8_t*>(base + (size_t)n_chains * P.n * 12);
  P.on_n = 0;
  return cl_launch(P, n_chains, keys, (cudaStream_t)stream);
}

extern "C" int32_t critmc_on_cluster_update(float* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                            int32_t n, int32_t n_chains, const uint32_t* keys, double beta,
                                            int32_t algo, uint32_t sweep, int64_t* stats, void* scratch,
                                            void* stream) {
  clear_error();
  static thread_local ClParams P;
  int st = byte_geom(dim, lx, ly, lz, P.g);
  if (st) return st;
  if (!spins || !keys || !stats || !scratch) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (algo != CRITMC_WOLFF && algo != CRITMC_SWENDSEN_WANG) return fail(CRITMC_ERR_INVALID, "algo must be wolff or sw");
  if (n != 2 && n != 3) return fail(CRITMC_ERR_UNSUPPORTED, "O(n) cluster updates for n = 2, 3");
  if (n_chains < 1) return fail(CRITMC_ERR_INVALID, "need n_chains >= 1");
  if (!(beta >= 0.0) || !std::isfinite(beta)) return fail(CRITMC_ERR_INVALID, "beta must be finite and >= 0");
  P.n = 2 * P.g.slots;
  if ((long long)P.n * n_chains >= (1LL << 31)) return fail(CRITMC_ERR_UNSUPPORTED, "too many sites");
  P.spins = spins;
  P.bits = 0;
  P.potts = 0;
  P.q = 2;
  P.algo = algo;
  P.sweep = sweep;
  P.running = nullptr;
  P.counts = nullptr;
  P.stats = (long long*)stats;
  P.thr = 0;
  P.nb2 = (float)(-2.0 * beta);
  char* base = static_cast<char*>(scratch);
  P.label = reinterpret_cast<int*>(base);
  P.size = reinterpret_cast<int*>(base + (size_t)n_chains * P.n * 4);
  P.proj = reinterpret_cast<float*>(base + (size_t)n_chains * P.n * 8);
  P.newv = reinterpret_cast<int8_t*>(base + (size_t)n_chains * P.n * 12);
  P.on_n = n;
  return cl_launch(P, n_chains, keys, (cudaStream_t)stream);
}
