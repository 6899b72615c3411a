// Multi-spin-coded Ising: checkerboard half-sweep kernel over chains held in
// HBM, the scan that turns per-measurement increments into the E_b / M
// series, a from-scratch E_b / M measurement, and the C-ABI driver.
//
// Replaces critmc src/critmc/kernels/ising.py:174-237 (`run`), :69-87
// (`metropolis_sweep`), :91-107 (`heatbath_sweep`) and :32-45
// (`bond_energy`, `magnetization`).
#include <cstdio>
#include <cstring>
#include <vector>

#include "host_common.h"
#include "msc_ising.cuh"
#include "msc_ising_host.h"

namespace critmc {

constexpr int MSC_THREADS = 256;
constexpr int MSC_WPT = 4;  // words per thread per block
constexpr int MSC_WPB = MSC_THREADS * MSC_WPT;

struct MscFix {
  uint32_t w, U, s, D;
};

struct MscHalfArgs {
  uint32_t* spins;
  const uint32_t* keys;
  unsigned long long* acc;  // [meas][chain][3]
  const uint32_t* cursor;   // optional device (sweep base, meas base)
  MscGeom g;
  int n_chains;
  int chains_per_group;
  int col;
  uint32_t sweep;  // absolute sweep (or offset when cursor != null)
  uint32_t meas;   // measurement slot (or offset when cursor != null)
};

template <int Z>
__device__ __forceinline__ void msc_row_coords(const MscGeom& g, uint32_t w, int& y, int& z, int& k) {
  const int r = (int)(w >> g.wc_log2);
  k = (int)(w & (g.wc - 1));
  if constexpr (Z == 6) {
    y = r % g.ly;
    z = r / g.ly;
  } else {
    y = r;
    z = 0;
  }
}

// grid: x = word blocks of one colour plane, y = chain within group, z = group
template <int Z, int RULE, int KG>
__global__ void __launch_bounds__(MSC_THREADS)
    msc_halfsweep_kernel(const MscHalfArgs a, const __grid_constant__ MscTables tabs) {
  __shared__ MscFix fix[MSC_WPB];
  __shared__ int nfix;
  __shared__ int red[3][MSC_THREADS / 32];

  const int group = blockIdx.z;
  const int chain = group * a.chains_per_group + blockIdx.y;
  const int tid = threadIdx.x;
  const MscGeom& g = a.g;
  if (tid == 0) nfix = 0;
  __syncthreads();

  MscRule<Z, RULE> rule{tabs.kind[group], tabs.thr[group]};
  const uint32_t k0 = a.keys[2 * chain], k1 = a.keys[2 * chain + 1];
  const uint32_t sweep = a.cursor ? a.cursor[0] + a.sweep : a.sweep;
  const uint32_t meas = a.cursor ? a.cursor[1] + a.meas : a.meas;
  const uint32_t col = (uint32_t)a.col;

  uint32_t* own = a.spins + (size_t)chain * 2 * g.words + (size_t)col * g.words;
  const uint32_t* other = a.spins + (size_t)chain * 2 * g.words + (size_t)(col ^ 1) * g.words;

  int dE = 0, dM = 0, nacc = 0;
  const uint32_t wbase = blockIdx.x * (uint32_t)MSC_WPB;
#pragma unroll 1
  for (int j = 0; j < MSC_WPT; ++j) {
    const uint32_t widx = wbase + j * MSC_THREADS + tid;
    if (widx >= g.words) break;
    int y, z, k;
    msc_row_coords<Z>(g, widx, y, z, k);
    uint32_t n[Z];
    msc_neighbours<Z>(other, g, (int)col, y, z, k, n);
    MscWord w;
    rule.classify(own[widx], n, w);
#pragma unroll
    for (int grp = 0; grp < KG; ++grp) msc_group<Z, RULE>(rule, w, k0, k1, widx, sweep, col, grp);
    const uint32_t s_new = (RULE == RULE_HB0) ? w.D : (w.s ^ w.D);
    msc_obs<Z>((w.s ^ s_new) & ~w.U, w.s, w.anti, dE, dM, nacc);
    if (w.U == 0) {
      own[widx] = s_new;
    } else {
      const int slot = atomicAdd(&nfix, 1);
      fix[slot] = MscFix{widx, w.U, w.s, w.D};
    }
  }
  __syncthreads();
  // deferred lanes: continue the comparison with the next plane groups
  const int nf = nfix;
  for (int e = tid; e < nf; e += MSC_THREADS) {
    const MscFix f = fix[e];
    int y, z, k;
    msc_row_coords<Z>(g, f.w, y, z, k);
    uint32_t n[Z];
    msc_neighbours<Z>(other, g, (int)col, y, z, k, n);
    MscWord w;
    rule.classify(f.s, n, w);
    w.D = f.D;
    w.U = f.U;
    for (int grp = KG; grp < 8 && w.U != 0; ++grp) msc_group<Z, RULE>(rule, w, k0, k1, f.w, sweep, col, grp);
    const uint32_t s_new = (RULE == RULE_HB0) ? w.D : (f.s ^ w.D);
    msc_obs<Z>((f.s ^ s_new) & f.U, f.s, w.anti, dE, dM, nacc);
    own[f.w] = s_new;
  }
  // block reduction of the observable increments
  dE = warp_sum(dE);
  dM = warp_sum(dM);
  nacc = warp_sum(nacc);
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = dE;
    red[1][tid >> 5] = dM;
    red[2][tid >> 5] = nacc;
  }
  __syncthreads();
  if (tid < 3 && a.acc) {
    long long v = 0;
    for (int q = 0; q < MSC_THREADS / 32; ++q) v += red[tid][q];
    atomicAdd(a.acc + ((size_t)meas * a.n_chains + chain) * 3 + tid, as_ull(v));
  }
}

// per-chain scan of the increments into the absolute series
__global__ void msc_finalize_kernel(const long long* __restrict__ acc, long long* running,
                                    long long* e_out, long long* m_out, long long* aux_out,
                                    int n_chains, int n_meas) {
  const int chain = blockIdx.x;
  const int tid = threadIdx.x;
  const int nt = blockDim.x;
  __shared__ long long se[256], sm[256];
  const int per = (n_meas + nt - 1) / nt;
  const int b = tid * per, e = min(n_meas, b + per);
  long long le = 0, lm = 0;
  for (int i = b; i < e; ++i) {
    le += acc[((size_t)i * n_chains + chain) * 3 + 0];
    lm += acc[((size_t)i * n_chains + chain) * 3 + 1];
  }
  se[tid] = le;
  sm[tid] = lm;
  __syncthreads();
  if (tid == 0) {
    long long ce = running[2 * chain], cm = running[2 * chain + 1];
    for (int q = 0; q < nt; ++q) {
      const long long te = se[q], tm = sm[q];
      se[q] = ce;
      sm[q] = cm;
      ce += te;
      cm += tm;
    }
    running[2 * chain] = ce;
    running[2 * chain + 1] = cm;
  }
  __syncthreads();
  long long ce = se[tid], cm = sm[tid];
  for (int i = b; i < e; ++i) {
    const size_t src = ((size_t)i * n_chains + chain) * 3;
    ce += acc[src + 0];
    cm += acc[src + 1];
    const size_t dst = (size_t)chain * n_meas + i;
    e_out[dst] = ce;
    m_out[dst] = cm;
    aux_out[dst * 4 + 0] = acc[src + 2];
    aux_out[dst * 4 + 1] = 0;
    aux_out[dst * 4 + 2] = 0;
    aux_out[dst * 4 + 3] = 0;
  }
}

__global__ void msc_cursor_set(uint32_t* cursor, uint32_t sweep, uint32_t meas) {
  cursor[0] = sweep;
  cursor[1] = meas;
}
__global__ void msc_cursor_bump(uint32_t* cursor, uint32_t sweeps, uint32_t meas) {
  cursor[0] += sweeps;
  cursor[1] += meas;
}

// E_b and M from scratch: every bond has exactly one colour-0 endpoint.
template <int Z>
__global__ void msc_measure_kernel(const uint32_t* __restrict__ spins, MscGeom g,
                                   unsigned long long* out) {
  const int chain = blockIdx.y;
  const uint32_t* c0 = spins + (size_t)chain * 2 * g.words;
  const uint32_t* c1 = c0 + g.words;
  long long unsat = 0, up = 0;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < g.words; w += gridDim.x * blockDim.x) {
    int y, z, k;
    msc_row_coords<Z>(g, w, y, z, k);
    uint32_t n[Z];
    msc_neighbours<Z>(c1, g, 0, y, z, k, n);
    const uint32_t s = c0[w];
#pragma unroll
    for (int q = 0; q < Z; ++q) unsat += __popc(s ^ n[q]);
    up += __popc(s) + __popc(c1[w]);
  }
  unsat = warp_sum(unsat);
  up = warp_sum(up);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out + 2 * chain, as_ull(unsat));
    atomicAdd(out + 2 * chain + 1, as_ull(up));
  }
}

__global__ void msc_measure_final(unsigned long long* io, int n_chains, long long n_sites, int z) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_chains) return;
  const long long unsat = (long long)io[2 * c], up = (long long)io[2 * c + 1];
  const long long bonds = n_sites * z / 2;
  io[2 * c] = (unsigned long long)(-(bonds - 2 * unsat));
  io[2 * c + 1] = (unsigned long long)(2 * up - n_sites);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int msc_geom(int dim, int lx, int ly, int lz, MscGeom& g) {
  if (dim != 2 && dim != 3) return fail(CRITMC_ERR_UNSUPPORTED, "MSC Ising supports dim 2 and 3");
  if (dim == 2) lz = 1;
  if (lx < 64 || lx % 64 != 0) return fail(CRITMC_ERR_UNSUPPORTED, "MSC Ising needs lx % 64 == 0");
  const int wc = lx / 64;
  if ((wc & (wc - 1)) != 0) return fail(CRITMC_ERR_UNSUPPORTED, "MSC Ising needs lx/64 a power of two");
  if (ly < 2 || ly % 2 != 0) return fail(CRITMC_ERR_UNSUPPORTED, "checkerboard needs even ly");
  if (dim == 3 && (lz < 2 || lz % 2 != 0)) return fail(CRITMC_ERR_UNSUPPORTED, "checkerboard needs even lz");
  g.dim = dim;
  g.lx = lx;
  g.ly = ly;
  g.lz = lz;
  g.wc = wc;
  g.wc_log2 = 0;
  while ((1 << g.wc_log2) < wc) ++g.wc_log2;
  g.rows = ly * lz;
  const long long words = (long long)g.rows * wc;
  if (words >= (1LL << 31)) return fail(CRITMC_ERR_UNSUPPORTED, "lattice too large");
  g.words = (uint32_t)words;
  return CRITMC_OK;
}

// Pick the cheapest rule that reproduces the table's decisions exactly.
int msc_pick_rule(const uint32_t* kind, const uint32_t* thr, int z, int algo, int n_groups) {
  bool spin_indep = true, metro0 = (algo == CRITMC_METROPOLIS), hb0 = (algo == CRITMC_HEATBATH);
  for (int gi = 0; gi < n_groups; ++gi) {
    const uint32_t* kd = kind + gi * CRITMC_NCLS;
    const uint32_t* th = thr + gi * CRITMC_NCLS;
    for (int v = 0; v <= z; ++v) {
      if (kd[2 * v] != kd[2 * v + 1] || th[2 * v] != th[2 * v + 1]) spin_indep = false;
      const uint32_t k = kd[2 * v];
      // NEVER behaves as RANDOM with thr = 0 (u < 0 is never true)
      const bool rnd = (k == CRITMC_KIND_RANDOM) || (k == CRITMC_KIND_NEVER && th[2 * v] == 0);
      if (2 * v < z) {
        if (!rnd) metro0 = false;
      } else if (k != CRITMC_KIND_ALWAYS) {
        metro0 = false;
      }
      if (!rnd) hb0 = false;
    }
  }
  if (!spin_indep) return RULE_GENSPIN;
  if (metro0) return RULE_METRO0;
  if (hb0) return RULE_HB0;
  return RULE_GEN;
}

template <int Z, int RULE>
static void launch_half_kg(const MscHalfArgs& a, const MscTables& t, int n_groups, int kg,
                           cudaStream_t st) {
  const dim3 grid((a.g.words + MSC_WPB - 1) / MSC_WPB, a.chains_per_group, n_groups);
  if (kg == 1) msc_halfsweep_kernel<Z, RULE, 1><<<grid, MSC_THREADS, 0, st>>>(a, t);
  else msc_halfsweep_kernel<Z, RULE, 2><<<grid, MSC_THREADS, 0, st>>>(a, t);
}

template <int Z>
static void launch_half_z(const MscHalfArgs& a, const MscTables& t, int n_groups, int rule, int kg,
                          cudaStream_t st) {
  switch (rule) {
    case RULE_METRO0: launch_half_kg<Z, RULE_METRO0>(a, t, n_groups, kg, st); break;
    case RULE_HB0: launch_half_kg<Z, RULE_HB0>(a, t, n_groups, kg, st); break;
    case RULE_GEN: launch_half_kg<Z, RULE_GEN>(a, t, n_groups, kg, st); break;
    default: launch_half_kg<Z, RULE_GENSPIN>(a, t, n_groups, kg, st); break;
  }
}

void msc_launch_half(const MscHalfArgs& a, const MscTables& t, int n_groups, int rule, int kg,
                     cudaStream_t st) {
  if (a.g.dim == 2) launch_half_z<4>(a, t, n_groups, rule, kg, st);
  else launch_half_z<6>(a, t, n_groups, rule, kg, st);
}

}  // namespace critmc

using namespace critmc;

extern "C" int64_t critmc_ising_msc_scratch_bytes(int32_t n_chains, int32_t n_meas) {
  return 16 + (int64_t)n_chains * n_meas * 3 * 8;
}

extern "C" int32_t critmc_ising_msc_run(uint32_t* spins, int32_t dim, int32_t lx, int32_t ly,
                                        int32_t lz, int32_t n_chains, const uint32_t* keys,
                                        const uint32_t* tables, int32_t n_groups, uint32_t sweep0,
                                        const int64_t* schedule, int32_t n_rows, int32_t n_meas,
                                        int64_t* running, int64_t* e_out, int64_t* m_out,
                                        int64_t* aux_out, void* scratch, int32_t mode,
                                        int32_t k_inline, void* stream) {
  clear_error();
  MscGeom g;
  int st = msc_geom(dim, lx, ly, lz, g);
  if (st) return st;
  if (!spins || !keys || !tables || !running || !e_out || !m_out || !aux_out || !scratch)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_chains > 65535) return fail(CRITMC_ERR_INVALID, "n_chains must be in [1, 65535]");
  if (n_groups < 1 || n_groups > MSC_MAX_GROUPS || n_chains % n_groups != 0)
    return fail(CRITMC_ERR_INVALID, "n_groups must be in [1, 16] and divide n_chains");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  if (!schedule || n_rows < 1) return fail(CRITMC_ERR_INVALID, "empty schedule");
  if (k_inline != 4 && k_inline != 8) return fail(CRITMC_ERR_INVALID, "k_inline must be 4 or 8");
  long long sweeps_per_meas = 0;
  for (int r = 0; r < n_rows; ++r) {
    const int64_t code = schedule[2 * r], reps = schedule[2 * r + 1];
    if (code != CRITMC_METROPOLIS && code != CRITMC_HEATBATH)
      return fail(CRITMC_ERR_UNSUPPORTED, "MSC Ising runs checkerboard metropolis and heatbath rows only");
    if (reps < 1) return fail(CRITMC_ERR_INVALID, "schedule repetitions must be positive");
    sweeps_per_meas += reps;
  }
  if (mode == 0) mode = 3;
  if (mode != 1 && mode != 3) return fail(CRITMC_ERR_UNSUPPORTED, "mode must be 0, 1 or 3");
  if (n_meas == 0) return CRITMC_OK;
  const long long total_sweeps = sweeps_per_meas * (long long)n_meas;
  if ((long long)sweep0 + total_sweeps > 0xFFFFFFFFLL)
    return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");

  // per-algorithm uniform tables and rules
  MscTables tabs[2];
  int rule[2];
  for (int slot = 0; slot < 2; ++slot) {
    std::memset(&tabs[slot], 0, sizeof(MscTables));
    for (int gi = 0; gi < n_groups; ++gi) {
      const uint32_t* src = tables + (size_t)gi * 4 * CRITMC_NCLS + slot * 2 * CRITMC_NCLS;
      std::memcpy(tabs[slot].kind[gi], src, CRITMC_NCLS * 4);
      std::memcpy(tabs[slot].thr[gi], src + CRITMC_NCLS, CRITMC_NCLS * 4);
    }
    rule[slot] = msc_pick_rule(&tabs[slot].kind[0][0], &tabs[slot].thr[0][0], 2 * dim,
                               slot ? CRITMC_HEATBATH : CRITMC_METROPOLIS, n_groups);
  }

  CaptureStream cs;
  if ((st = cs.begin(stream))) return st;
  cudaStream_t s = cs.work;
  uint32_t* cursor = (uint32_t*)scratch;
  unsigned long long* acc = (unsigned long long*)((char*)scratch + 16);
  if (cudaMemsetAsync(acc, 0, (size_t)n_chains * n_meas * 3 * 8, s) != cudaSuccess)
    return cuda_fail("memset");

  MscHalfArgs a;
  a.spins = spins;
  a.keys = keys;
  a.acc = acc;
  a.g = g;
  a.n_chains = n_chains;
  a.chains_per_group = n_chains / n_groups;
  const int kg = k_inline / 4;

  auto launch_meas = [&](uint32_t sweep_rel, uint32_t meas_rel, const uint32_t* cur) {
    a.cursor = cur;
    uint32_t sw = sweep_rel;
    for (int r = 0; r < n_rows; ++r) {
      const int slot = schedule[2 * r] == CRITMC_HEATBATH ? 1 : 0;
      for (int64_t rep = 0; rep < schedule[2 * r + 1]; ++rep) {
        a.sweep = sw;
        a.meas = meas_rel;
        a.col = 0;
        msc_launch_half(a, tabs[slot], n_groups, rule[slot], kg, s);
        a.col = 1;
        msc_launch_half(a, tabs[slot], n_groups, rule[slot], kg, s);
        ++sw;
      }
    }
  };

  if (mode == 1) {
    uint32_t sw = sweep0;
    for (int m = 0; m < n_meas; ++m) {
      launch_meas(sw, (uint32_t)m, nullptr);
      sw += (uint32_t)sweeps_per_meas;
    }
  } else {
    // a graph of G measurements replayed with a device cursor
    const int G = (int)std::max<long long>(
        1, std::min<long long>(n_meas, 256 / std::max<long long>(1, sweeps_per_meas)));
    msc_cursor_set<<<1, 1, 0, s>>>(cursor, sweep0, 0);
    const int n_graph = n_meas / G;
    if (n_graph > 1) {
      cudaGraph_t graph;
      cudaGraphExec_t exec;
      if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return cuda_fail("capture");
      for (int m = 0; m < G; ++m) launch_meas((uint32_t)(m * sweeps_per_meas), (uint32_t)m, cursor);
      msc_cursor_bump<<<1, 1, 0, s>>>(cursor, (uint32_t)(G * sweeps_per_meas), (uint32_t)G);
      if (cudaStreamEndCapture(s, &graph) != cudaSuccess) return cuda_fail("end capture");
      if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_fail("instantiate");
      }
      for (int i = 0; i < n_graph; ++i) cudaGraphLaunch(exec, s);
      cudaGraphExecDestroy(exec);
      cudaGraphDestroy(graph);
    }
    const int done = n_graph > 1 ? n_graph * G : 0;
    for (int m = done; m < n_meas; ++m)
      launch_meas((uint32_t)(sweep0 + (uint32_t)(m * sweeps_per_meas)), (uint32_t)m, nullptr);
  }
  msc_finalize_kernel<<<n_chains, 256, 0, s>>>((const long long*)acc, (long long*)running,
                                                (long long*)e_out, (long long*)m_out,
                                                (long long*)aux_out, n_chains, n_meas);
  if (cudaGetLastError() != cudaSuccess) return cuda_fail("launch");
  return cs.finish();
}

extern "C" int32_t critmc_ising_msc_measure(const uint32_t* spins, int32_t dim, int32_t lx,
                                            int32_t ly, int32_t lz, int32_t n_chains, int64_t* out,
                                            void* stream) {
  clear_error();
  MscGeom g;
  int st = msc_geom(dim, lx, ly, lz, g);
  if (st) return st;
  if (!spins || !out) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_chains > 65535) return fail(CRITMC_ERR_INVALID, "n_chains must be in [1, 65535]");
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(out, 0, (size_t)n_chains * 2 * 8, s) != cudaSuccess) return cuda_fail("memset");
  const dim3 grid(std::min<uint32_t>(1024, (g.words + 255) / 256), n_chains);
  if (dim == 2) msc_measure_kernel<4><<<grid, 256, 0, s>>>(spins, g, (unsigned long long*)out);
  else msc_measure_kernel<6><<<grid, 256, 0, s>>>(spins, g, (unsigned long long*)out);
  const long long n_sites = (long long)lx * ly * (dim == 3 ? lz : 1);
  msc_measure_final<<<(n_chains + 127) / 128, 128, 0, s>>>((unsigned long long*)out, n_chains, n_sites, 2 * dim);
  if (cudaGetLastError() != cudaSuccess) return cuda_fail("launch");
  return CRITMC_OK;
}
