// Byte lattices: int8 Ising and q-state Potts chains, one thread block per
// chain running the whole schedule (lattice staged in shared memory when it
// fits).  This is also the batched form for many small chains: a launch
// carries up to BYTE_PCHAINS chains, one block each.
//
// Replaces critmc src/critmc/kernels/ising.py:174-237 / potts.py:171-235
// (`run`), ising.py:69-107 and potts.py:45-103 (the sweeps) for checkerboard
// visiting order.
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "geom.cuh"
#include "host_common.h"

namespace critmc {

constexpr int BYTE_PCHAINS = 1024;      // chains per launch (keys in kernel parameters)
constexpr int BYTE_MAX_GROUPS = 16;
constexpr int BYTE_MAX_ROWS = 8;        // schedule rows
constexpr int BYTE_SMEM_MAX = 160 * 1024;
constexpr int MODEL_ISING = 0, MODEL_POTTS = 1;

struct ByteParams {
  int8_t* spins;
  long long* running;   // Ising: [n][2] (E_b, M); Potts: energy [n]
  long long* counts;    // Potts: [n][q]
  long long* e_out;
  long long* m_out;     // Ising only
  long long* counts_out;  // Potts only
  long long* aux_out;
  ByteGeom g;
  int q;
  int n_chains, chain0, chains_per_group, n_meas;
  int n_rows;
  int codes[BYTE_MAX_ROWS];
  int reps[BYTE_MAX_ROWS];
  int resident;
  uint32_t sweep0;
  // Ising: kind/thr per group and algorithm slot; Potts: 64-bit thresholds and weights
  uint32_t kind[BYTE_MAX_GROUPS][2][CRITMC_NCLS];
  uint32_t thr[BYTE_MAX_GROUPS][2][CRITMC_NCLS];
  unsigned long long boltz[BYTE_MAX_GROUPS][8];
  unsigned long long weight[BYTE_MAX_GROUPS][8];
  uint32_t keys[BYTE_PCHAINS][2];
};

// Everything one thread block needs to advance one byte-lattice chain.
struct ByteChain {
  const RunCtl* ctl = nullptr;  // bounded run (work items), polled between measurements
  CtlPoll* poll = nullptr;
  int8_t* gl;            // lattice in HBM, [colour][slot]
  long long* running;    // Ising: (E_b, M); Potts: E
  long long* counts;     // Potts: [q]
  long long* e_out;      // [n_meas]
  long long* m_out;      // Ising: [n_meas]
  long long* counts_out; // Potts: [n_meas][q]
  long long* aux_out;    // [n_meas][4]
  ByteGeom g;
  int q, n_meas, n_rows, resident;
  const int* codes;
  const int* reps;
  uint32_t sweep0, k0, k1;
  const uint32_t* kind;  // [2][16] (Ising)
  const uint32_t* thr;   // [2][16] (Ising)
  const unsigned long long* boltz;   // [8] (Potts)
  const unsigned long long* weight;  // [8] (Potts)
};

// CL == 1: one block, the lattice in shared memory when a.resident.  CL > 1: a
// cluster of CL blocks splits every site loop over the lattice in global
// memory, the cluster barrier separates the colours, and block 0 adds the
// blocks' per-measurement sums (and, for Potts, their running count changes,
// snapshotted at each measurement) from distributed shared memory.  A
// colour's sites are independent and the sums are integers, so every CL
// gives the same spins and series.  Block 0's thread 0 alone polls the
// control and passes its answer to all blocks before the barrier that ends a
// measurement, so the whole team stops at the same measurement.
template <int MODEL, int Z, int CL = 1>
__device__ void byte_chain_run(const ByteChain& a, unsigned char* smem_raw) {
  using T = Team<CL>;
  __shared__ long long red[16];
  __shared__ int cnt[128];  // Potts: counts (CL == 1), this block's count changes (CL > 1)
  __shared__ int s_stop[2];
  __shared__ long long part[CL > 1 ? 2 : 1][CL][3];
  __shared__ int snap[CL > 1 ? 2 : 1][CL > 1 ? 128 : 1];
  __shared__ long long cnt0[CL > 1 ? 128 : 1];
  const ByteGeom& g = a.g;
  const uint32_t k0 = a.k0, k1 = a.k1;
  const size_t n_sites = 2 * (size_t)g.slots;
  int8_t* gl = a.gl;
  const bool resident = CL == 1 && a.resident;
  int8_t* lat = resident ? reinterpret_cast<int8_t*>(smem_raw) : gl;
  const unsigned rank = T::rank();
  const int tid = threadIdx.x, nb_threads = blockDim.x;
  const uint32_t t0 = rank * blockDim.x + tid, nt = CL * blockDim.x;
  if (resident)
    for (size_t j = tid; j < n_sites; j += nb_threads) lat[j] = gl[j];
  const int q = a.q;
  if (MODEL == MODEL_POTTS)
    for (int k = tid; k < q; k += nb_threads) {
      if constexpr (CL == 1) {
        cnt[k] = (int)a.counts[k];
      } else {
        cnt[k] = 0;
        cnt0[k] = a.counts[k];
      }
    }
  if (CL > 1 && tid == 0) s_stop[0] = 0;
  T::sync();

  long long e_run = a.running[0];
  long long m_run = (MODEL == MODEL_ISING) ? a.running[1] : 0;
  uint32_t sweep = a.sweep0;
  for (int meas = 0; meas < a.n_meas; ++meas) {
    if constexpr (CL == 1) {
      if (a.ctl) {  // stop between measurements when the budget or a cancel says so
        if (tid == 0) s_stop[0] = a.poll->check(*a.ctl);
        __syncthreads();
        if (s_stop[0]) break;
      }
    } else {
      if (s_stop[meas & 1]) break;  // block 0's answer, written before the last barrier
    }
    long long dE = 0, dM = 0, nacc = 0;
    for (int row = 0; row < a.n_rows; ++row) {
      const int code = a.codes[row];
      const int slot_alg = (code == CRITMC_HEATBATH) ? 1 : 0;
      for (int rep = 0; rep < a.reps[row]; ++rep) {
        for (int c = 0; c < 2; ++c) {
          int8_t* own = lat + (size_t)c * g.slots;
          const int8_t* other = lat + (size_t)(c ^ 1) * g.slots;
          for (uint32_t s = t0; s < g.slots; s += nt) {
            int r, i;
            byte_row_index(g, s, r, i);
            uint32_t nb[Z];
            byte_neighbours<Z>(g, c, r, i, nb);
            const critmc_u32x4 rnd =
                critmc_philox4x32(s, sweep, CRITMC_TAG_SITE | ((uint32_t)c << 16), 0u, k0, k1);
            const int old = own[CRITMC_IDX(s, g.slots)];
            if constexpr (MODEL == MODEL_ISING) {
              int field = 0;
#pragma unroll
              for (int k = 0; k < Z; ++k) field += other[CRITMC_IDX(nb[k], g.slots)];
              const int sb = old > 0;
              int v;
              if (slot_alg == 0) v = (Z - old * field) / 2;  // anti-aligned neighbours
              else v = (field + Z) / 2;                       // up neighbours
              const int cls = 2 * v + sb;
              const uint32_t kd = a.kind[slot_alg * CRITMC_NCLS + cls];
              const bool dec = kd == CRITMC_KIND_ALWAYS ||
                               (kd == CRITMC_KIND_RANDOM && rnd.v[0] < a.thr[slot_alg * CRITMC_NCLS + cls]);
              const int nw = slot_alg == 0 ? (dec ? -old : old) : (dec ? 1 : -1);
              if (nw != old) {
                own[s] = (int8_t)nw;
                dE += 2 * old * field;
                dM += nw - old;
                ++nacc;
              }
            } else {
              int nbs[Z];
#pragma unroll
              for (int k = 0; k < Z; ++k) nbs[k] = other[CRITMC_IDX(nb[k], g.slots)];
              int nw;
              if (slot_alg == 0) {
                // propose a uniformly chosen different state (potts.py:53-56)
                nw = (int)(((unsigned long long)rnd.v[0] * (unsigned)(q - 1)) >> 32);
                if (nw >= old) ++nw;
                int n_old = 0, n_new = 0;
#pragma unroll
                for (int k = 0; k < Z; ++k) {
                  n_old += nbs[k] == old;
                  n_new += nbs[k] == nw;
                }
                const int delta = n_old - n_new;
                const bool acc = delta <= 0 || (unsigned long long)rnd.v[1] < a.boltz[delta];
                if (acc) {
                  own[s] = (int8_t)nw;
                  atomicSub(&cnt[old], 1);
                  atomicAdd(&cnt[nw], 1);
                  dE += delta;
                  ++nacc;
                }
              } else {
                // heat bath: state k with weight W[#neighbours in k] (potts.py:75-103)
                const unsigned long long u = ((unsigned long long)rnd.v[0] << 32) | rnd.v[1];
                unsigned long long total = 0;
                for (int k = 0; k < q; ++k) {
                  int nk = 0;
#pragma unroll
                  for (int j = 0; j < Z; ++j) nk += nbs[j] == k;
                  total += a.weight[nk];
                }
                const unsigned long long x = __umul64hi(u, total);
                unsigned long long cum = 0;
                nw = q - 1;
                for (int k = 0; k < q; ++k) {
                  int nk = 0;
#pragma unroll
                  for (int j = 0; j < Z; ++j) nk += nbs[j] == k;
                  cum += a.weight[nk];
                  if (x < cum) {
                    nw = k;
                    break;
                  }
                }
                if (nw != old) {
                  int n_old = 0, n_new = 0;
#pragma unroll
                  for (int k = 0; k < Z; ++k) {
                    n_old += nbs[k] == old;
                    n_new += nbs[k] == nw;
                  }
                  own[s] = (int8_t)nw;
                  atomicSub(&cnt[old], 1);
                  atomicAdd(&cnt[nw], 1);
                  dE += n_old - n_new;
                  ++nacc;
                }
              }
            }
          }
          T::sync();
        }
        ++sweep;
      }
    }
    dE = block_sum(dE, red);
    dM = block_sum(dM, red);
    nacc = block_sum(nacc, red);
    if constexpr (CL > 1) {
      if (tid == 0) {
        long long* p = T::at(&part[meas & 1][rank][0], 0);
        p[0] = dE;
        p[1] = dM;
        p[2] = nacc;
      }
      if (MODEL == MODEL_POTTS)
        for (int k = tid; k < q; k += nb_threads) snap[meas & 1][k] = cnt[k];
      if (rank == 0 && tid == 0) {
        const int stop = a.ctl ? a.poll->check(*a.ctl) : 0;
        for (int r = 0; r < CL; ++r) *T::at(&s_stop[(meas + 1) & 1], (unsigned)r) = stop;
      }
      T::sync();
      // block 0 adds the blocks' sums; part and snap of this parity are next
      // written two measurements on, after barriers block 0 passes once done here
      dE = dM = nacc = 0;
      if (rank == 0 && tid == 0)
        for (int r = 0; r < CL; ++r) {
          dE += part[meas & 1][r][0];
          dM += part[meas & 1][r][1];
          nacc += part[meas & 1][r][2];
        }
    }
    e_run += dE;
    m_run += dM;
    if (rank == 0 && tid == 0) {
      a.e_out[meas] = e_run;
      if (MODEL == MODEL_ISING) a.m_out[meas] = m_run;
      a.aux_out[4 * meas + 0] = nacc;
      a.aux_out[4 * meas + 1] = 0;
      a.aux_out[4 * meas + 2] = 0;
      a.aux_out[4 * meas + 3] = 0;
    }
    if (MODEL == MODEL_POTTS && rank == 0)
      for (int k = tid; k < q; k += nb_threads) {
        long long c;
        if constexpr (CL == 1) {
          c = cnt[k];
        } else {
          c = cnt0[k];
          for (int r = 0; r < CL; ++r) c += *T::at(&snap[meas & 1][k], (unsigned)r);
        }
        a.counts_out[(size_t)meas * q + k] = c;
      }
  }
  T::sync();
  if (resident)
    for (size_t j = tid; j < n_sites; j += nb_threads) gl[j] = lat[j];
  if (rank == 0 && tid == 0) {
    a.running[0] = e_run;
    if (MODEL == MODEL_ISING) a.running[1] = m_run;
  }
  if (MODEL == MODEL_POTTS && rank == 0)
    for (int k = tid; k < q; k += nb_threads) {
      long long c;
      if constexpr (CL == 1) {
        c = cnt[k];
      } else {
        c = cnt0[k];
        for (int r = 0; r < CL; ++r) c += *T::at(&cnt[k], (unsigned)r);
      }
      a.counts[k] = c;
    }
  T::sync();
}

template <int MODEL, int Z>
__global__ void __launch_bounds__(512) byte_run_kernel(const __grid_constant__ ByteParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lchain = blockIdx.x;
  const int chain = P.chain0 + lchain;
  const int group = chain / P.chains_per_group;
  ByteChain a;
  a.g = P.g;
  a.gl = P.spins + (size_t)chain * 2 * P.g.slots;
  a.running = P.running + (MODEL == MODEL_ISING ? 2 * (size_t)chain : (size_t)chain);
  a.counts = P.counts ? P.counts + (size_t)chain * P.q : nullptr;
  a.e_out = P.e_out + (size_t)chain * P.n_meas;
  a.m_out = P.m_out ? P.m_out + (size_t)chain * P.n_meas : nullptr;
  a.counts_out = P.counts_out ? P.counts_out + (size_t)chain * P.n_meas * P.q : nullptr;
  a.aux_out = P.aux_out + (size_t)chain * P.n_meas * 4;
  a.q = P.q;
  a.n_meas = P.n_meas;
  a.n_rows = P.n_rows;
  a.resident = P.resident;
  a.codes = P.codes;
  a.reps = P.reps;
  a.sweep0 = P.sweep0;
  a.k0 = P.keys[lchain][0];
  a.k1 = P.keys[lchain][1];
  a.kind = &P.kind[group][0][0];
  a.thr = &P.thr[group][0][0];
  a.boltz = P.boltz[group];
  a.weight = P.weight[group];
  byte_chain_run<MODEL, Z>(a, smem_raw);
}

static int byte_schedule(ByteParams& P, const int64_t* schedule, int n_rows, long long& per_meas) {
  if (!schedule || n_rows < 1 || n_rows > BYTE_MAX_ROWS)
    return fail(CRITMC_ERR_INVALID, "schedule must have 1..8 rows");
  per_meas = 0;
  for (int r = 0; r < n_rows; ++r) {
    const int64_t code = schedule[2 * r], reps = schedule[2 * r + 1];
    if (code != CRITMC_METROPOLIS && code != CRITMC_HEATBATH)
      return fail(CRITMC_ERR_UNSUPPORTED, "byte lattices run checkerboard metropolis and heatbath rows only");
    if (reps < 1 || reps > (1 << 20)) return fail(CRITMC_ERR_INVALID, "schedule repetitions must be in [1, 2^20]");
    P.codes[r] = (int)code;
    P.reps[r] = (int)reps;
    per_meas += reps;
  }
  P.n_rows = n_rows;
  return CRITMC_OK;
}

template <int MODEL>
static int byte_launch(ByteParams& P, const uint32_t* keys, cudaStream_t s) {
  const size_t lat_bytes = 2 * (size_t)P.g.slots;
  P.resident = lat_bytes <= (size_t)BYTE_SMEM_MAX;
  const size_t smem = P.resident ? lat_bytes : 0;
  int threads = (int)std::min<uint32_t>(512, ((P.g.slots + 31) / 32) * 32);
  threads = std::max(threads, 32);
  for (int c0 = 0; c0 < P.n_chains; c0 += BYTE_PCHAINS) {
    const int nc = std::min(BYTE_PCHAINS, P.n_chains - c0);
    P.chain0 = c0;
    std::memcpy(P.keys, keys + 2 * (size_t)c0, sizeof(uint32_t) * 2 * nc);
    auto launch = [&](auto kern) {
      if (smem > 0) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  // static + dynamic may pass 48 KiB
      kern<<<nc, threads, smem, s>>>(P);
    };
    switch (P.g.dim) {
      case 1: launch(byte_run_kernel<MODEL, 2>); break;
      case 2: launch(byte_run_kernel<MODEL, 4>); break;
      default: launch(byte_run_kernel<MODEL, 6>); break;
    }
    if (int e_ = cuda_check("launch")) return e_;
  }
  return CRITMC_OK;
}

static thread_local ByteParams g_params;  // large: kept off the stack, one per calling thread

}  // namespace critmc

using namespace critmc;

extern "C" int32_t critmc_potts_tables(int32_t z, double beta, uint64_t* boltz_thr, uint64_t* hb_weight) {
  clear_error();
  if (!boltz_thr || !hb_weight) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (z < 1 || z > 7 || !std::isfinite(beta)) return fail(CRITMC_ERR_INVALID, "need 1 <= z <= 7 and finite beta");
  for (int d = 0; d < 8; ++d) {
    const double p = std::exp(-beta * d);  // potts.py:192-194 boltz[d]
    if (d == 0 || p >= 1.0) {
      boltz_thr[d] = 1ULL << 32;
    } else {
      const double t = std::nearbyint(std::ldexp(p, 32));
      boltz_thr[d] = t >= 4294967296.0 ? (1ULL << 32) : (uint64_t)t;
    }
  }
  // weight[n] = exp(beta n) (potts.py:192-194), scaled so that the largest is 2^52
  double mx = -INFINITY;
  for (int n = 0; n <= z; ++n) mx = std::max(mx, beta * n);
  for (int n = 0; n < 8; ++n) {
    const double w = n <= z ? std::exp(beta * n - mx) : 0.0;
    hb_weight[n] = (uint64_t)std::nearbyint(std::ldexp(w, 52));
  }
  return CRITMC_OK;
}

extern "C" int32_t critmc_ising_byte_run(int8_t* spins, int32_t dim, int32_t lx, int32_t ly,
                                         int32_t lz, int32_t n_chains, const uint32_t* keys,
                                         const uint32_t* tables, int32_t n_groups, uint32_t sweep0,
                                         const int64_t* schedule, int32_t n_rows, int32_t n_meas,
                                         int64_t* running, int64_t* e_out, int64_t* m_out,
                                         int64_t* aux_out, void* stream) {
  clear_error();
  ByteParams& P = g_params;
  int st = byte_geom(dim, lx, ly, lz, P.g);
  if (st) return st;
  if (!spins || !keys || !tables || !running || !e_out || !m_out || !aux_out)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_groups < 1 || n_groups > BYTE_MAX_GROUPS || n_chains % n_groups)
    return fail(CRITMC_ERR_INVALID, "need n_chains >= 1 and 1 <= n_groups <= 16 dividing n_chains");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  long long per_meas = 0;
  if ((st = byte_schedule(P, schedule, n_rows, per_meas))) return st;
  if ((long long)sweep0 + per_meas * n_meas > 0xFFFFFFFFLL)
    return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");
  if (n_meas == 0) return CRITMC_OK;
  for (int gi = 0; gi < n_groups; ++gi)
    for (int a = 0; a < 2; ++a) {
      std::memcpy(P.kind[gi][a], tables + ((size_t)gi * 4 + 2 * a) * CRITMC_NCLS, CRITMC_NCLS * 4);
      std::memcpy(P.thr[gi][a], tables + ((size_t)gi * 4 + 2 * a + 1) * CRITMC_NCLS, CRITMC_NCLS * 4);
    }
  P.spins = spins;
  P.running = (long long*)running;
  P.e_out = (long long*)e_out;
  P.m_out = (long long*)m_out;
  P.aux_out = (long long*)aux_out;
  P.counts = nullptr;
  P.counts_out = nullptr;
  P.q = 2;
  P.n_chains = n_chains;
  P.chains_per_group = n_chains / n_groups;
  P.n_meas = n_meas;
  P.sweep0 = sweep0;
  return byte_launch<MODEL_ISING>(P, keys, (cudaStream_t)stream);
}

extern "C" int32_t critmc_potts_run(int8_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                    int32_t q, int32_t n_chains, const uint32_t* keys,
                                    const double* betas, int32_t n_groups, uint32_t sweep0,
                                    const int64_t* schedule, int32_t n_rows, int32_t n_meas,
                                    int64_t* energy, int64_t* counts, int64_t* e_out,
                                    int64_t* counts_out, int64_t* aux_out, void* stream) {
  clear_error();
  ByteParams& P = g_params;
  int st = byte_geom(dim, lx, ly, lz, P.g);
  if (st) return st;
  if (!spins || !keys || !betas || !energy || !counts || !e_out || !counts_out || !aux_out)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (q < 2 || q > 127) return fail(CRITMC_ERR_INVALID, "q must be in [2, 127]");
  if (n_chains < 1 || n_groups < 1 || n_groups > BYTE_MAX_GROUPS || n_chains % n_groups)
    return fail(CRITMC_ERR_INVALID, "need n_chains >= 1 and 1 <= n_groups <= 16 dividing n_chains");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  long long per_meas = 0;
  if ((st = byte_schedule(P, schedule, n_rows, per_meas))) return st;
  if ((long long)sweep0 + per_meas * n_meas > 0xFFFFFFFFLL)
    return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");
  if (n_meas == 0) return CRITMC_OK;
  for (int gi = 0; gi < n_groups; ++gi) {
    uint64_t b[8], w[8];
    if ((st = critmc_potts_tables(2 * dim, betas[gi], b, w))) return st;
    for (int d = 0; d < 8; ++d) {
      P.boltz[gi][d] = b[d];
      P.weight[gi][d] = w[d];
    }
  }
  P.spins = spins;
  P.running = (long long*)energy;
  P.counts = (long long*)counts;
  P.e_out = (long long*)e_out;
  P.m_out = nullptr;
  P.counts_out = (long long*)counts_out;
  P.aux_out = (long long*)aux_out;
  P.q = q;
  P.n_chains = n_chains;
  P.chains_per_group = n_chains / n_groups;
  P.n_meas = n_meas;
  P.sweep0 = sweep0;
  return byte_launch<MODEL_POTTS>(P, keys, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Byte-lattice chains as work items (persistent kernel, queue of items).
// ---------------------------------------------------------------------------
#include "items_host.h"

namespace critmc {

__device__ __forceinline__ int byte_geom_device(const critmc_item& it, ByteGeom& g) {
  g.dim = it.dim;
  g.lx = it.lx;
  g.ly = it.dim >= 2 ? it.ly : 1;
  g.lz = it.dim >= 3 ? it.lz : 1;
  g.hx = it.lx / 2;
  g.rows = g.ly * g.lz;
  g.slots = (uint32_t)(g.rows * g.hx);
  return 0;
}

// CL > 1: each item is advanced by a cluster of CL blocks (block 0 takes the
// item from the queue and hands its index to the others).
template <int CL>
__global__ void __launch_bounds__(ITEM_THREADS) byte_items_kernel(const critmc_item* items, int n,
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
    ByteChain a;
    if (ctl.status) {
      a.ctl = &ctl;
      a.poll = &poll;
    }
    byte_geom_device(it, a.g);
    a.gl = reinterpret_cast<int8_t*>(it.spins);
    a.running = reinterpret_cast<long long*>(it.running);
    a.counts = reinterpret_cast<long long*>(it.counts);
    a.e_out = reinterpret_cast<long long*>(it.e_out);
    a.m_out = reinterpret_cast<long long*>(it.vec_out);
    a.counts_out = reinterpret_cast<long long*>(it.vec_out);
    a.aux_out = reinterpret_cast<long long*>(it.aux_out);
    a.q = it.kind == CRITMC_ITEM_POTTS ? it.q_or_n : 2;
    a.n_meas = it.n_meas;
    a.n_rows = it.n_rows;
    a.resident = 2 * (size_t)a.g.slots <= smem;
    a.codes = it.codes;
    a.reps = it.reps;
    a.sweep0 = it.sweep0;
    a.k0 = it.key[0];
    a.k1 = it.key[1];
    a.kind = &it.kind_tab[0][0];
    a.thr = &it.thr_tab[0][0];
    a.boltz = reinterpret_cast<const unsigned long long*>(it.boltz);
    a.weight = reinterpret_cast<const unsigned long long*>(it.weight);
    if (it.kind == CRITMC_ITEM_POTTS) {
      if (it.dim == 1) byte_chain_run<MODEL_POTTS, 2, CL>(a, smem_raw);
      else if (it.dim == 2) byte_chain_run<MODEL_POTTS, 4, CL>(a, smem_raw);
      else byte_chain_run<MODEL_POTTS, 6, CL>(a, smem_raw);
    } else {
      if (it.dim == 1) byte_chain_run<MODEL_ISING, 2, CL>(a, smem_raw);
      else if (it.dim == 2) byte_chain_run<MODEL_ISING, 4, CL>(a, smem_raw);
      else byte_chain_run<MODEL_ISING, 6, CL>(a, smem_raw);
    }
  }
}

int byte_items_team_clusters(int team) {
  switch (team) {
    case 2: return team_clusters(byte_items_kernel<2>, 2, ITEM_THREADS);
    case 4: return team_clusters(byte_items_kernel<4>, 4, ITEM_THREADS);
    case 8: return team_clusters(byte_items_kernel<8>, 8, ITEM_THREADS);
    case 16: return team_clusters(byte_items_kernel<16>, 16, ITEM_THREADS);
    default: return fail(CRITMC_ERR_INVALID, "team size must be 2, 4, 8 or 16");
  }
}

int byte_items_launch(const critmc_item* items, int n, unsigned* queue, size_t smem, int team, const RunCtl& ctl,
                      cudaStream_t s) {
  switch (team) {
    case 2: return launch_team(byte_items_kernel<2>, 2, ITEM_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    case 4: return launch_team(byte_items_kernel<4>, 4, ITEM_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    case 8: return launch_team(byte_items_kernel<8>, 8, ITEM_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    case 16: return launch_team(byte_items_kernel<16>, 16, ITEM_THREADS, n, s, items, n, queue, (size_t)0, ctl);
    default: break;
  }
  auto kern = byte_items_kernel<1>;
  if (smem > 0 &&  // static + dynamic may pass 48 KiB
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return cuda_fail("shared memory attribute");
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ITEM_THREADS, smem);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, std::min(n, std::max(1, per_sm) * sms));
  kern<<<grid, ITEM_THREADS, smem, s>>>(items, n, queue, smem, ctl);
  if (int e_ = cuda_check("launch")) return e_;
  return CRITMC_OK;
}

}  // namespace critmc
