// Multi-spin-coded Ising: checkerboard half-sweep kernel over chains held in
// HBM, the scan that turns per-measurement increments into the E_b / M
// series, a from-scratch E_b / M measurement, and the C-ABI driver.
//
// Replaces critmc src/critmc/kernels/ising.py:174-237 (`run`), :69-87
// (`metropolis_sweep`), :91-107 (`heatbath_sweep`) and :32-45
// (`bond_energy`, `magnetization`).
#include <cuda.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "host_common.h"
#include "msc_ising.cuh"
#include "msc_ising_host.h"

namespace critmc {

constexpr int MSC_THREADS = 256;
constexpr int MSC_WARPS = MSC_THREADS / 32;
constexpr int MSC_FIXCAP = 64;     // deferred words per warp before a flush
constexpr int MSC_PCHAINS = 256;   // chains per launch (their keys travel as kernel parameters)

// Kernel parameters: keys and tables live in the constant bank, so the Philox
// key schedule and the threshold broadcasts run on the uniform datapath.
struct MscParams {
  uint32_t* spins;
  unsigned long long* acc;  // [meas][n_chains][3]
  const uint32_t* cursor;   // optional device (sweep base, meas base)
  MscGeom g;
  int n_chains;             // chains of the call (stride of acc)
  int chain0;               // first chain of this launch
  int chains_per_group;
  int col;
  int run;                  // rows walked by one thread
  uint32_t sweep;           // absolute sweep (or offset when cursor != null)
  uint32_t meas;            // measurement slot (or offset when cursor != null)
  uint32_t keys[MSC_PCHAINS][2];
  MscTables tabs;
  // batches of separately allocated chains (critmc_ising_msc_run_batch): the
  // lattice and table group of each chain of the launch, and a device array of
  // their sweep bases; batch_sweep == null for the contiguous chains of
  // critmc_ising_msc_run
  const uint32_t* batch_sweep;
  uint32_t* batch_spins[CRITMC_MSC_BATCH_MAX];
  uint32_t batch_group[CRITMC_MSC_BATCH_MAX];
};

struct MscFix {
  uint32_t w, U, D;
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

// Finish one deferred word: continue the MSB-first comparison plane group by
// plane group until every lane is decided, then store it.
template <int Z, int RULE, int KG, int PR>
__device__ __forceinline__ void msc_fixup(const MscRule<Z, RULE>& rule, const MscGeom& g,
                                          const MscFix f, uint32_t* own, const uint32_t* other,
                                          uint32_t col, uint32_t k0, uint32_t k1, uint32_t sweep,
                                          int& dE, int& dM, int& nacc) {
  int y, z, k;
  msc_row_coords<Z>(g, f.w, y, z, k);
  uint32_t n[Z];
  msc_neighbours<Z>(other, g, (int)col, y, z, k, n);
  MscWord w;
  rule.classify(own[CRITMC_IDX(f.w, g.words)], n, w);
  w.D = f.D;
  w.U = f.U;
  for (int grp = KG; grp < 8 && w.U != 0; ++grp) msc_group<Z, RULE, PR>(rule, w, k0, k1, f.w, sweep, col, grp);
  const uint32_t s_new = (RULE == RULE_HB0) ? w.D : (w.s ^ w.D);
  msc_obs<Z>((w.s ^ s_new) & f.U, w.s, w.anti, dE, dM, nacc);
  own[CRITMC_IDX(f.w, g.words)] = s_new;
}

// Finish the deferred words of a warp's list, all lanes on different words;
// returns the (E, M, accepted) increments.  Out of line on purpose: inlined,
// this path's state made the main loop below hold more registers and
// rematerialise its uniform values (measured: 318 -> 271 instructions per
// word, 2,580 -> 2,820 site updates/ns at L = 4096 with the bound below).
template <int Z, int RULE, int KG, int PR>
__device__ __noinline__ int3 msc_flush(const MscRule<Z, RULE> rule, const MscGeom g, const MscFix* list, int nf,
                                       uint32_t* own, const uint32_t* other, uint32_t col, uint32_t k0, uint32_t k1,
                                       uint32_t sweep) {
  int dE = 0, dM = 0, nacc = 0;
  const int lane = threadIdx.x & 31;
  __syncwarp();
  for (int e = lane; e < nf; e += 32)
    msc_fixup<Z, RULE, KG, PR>(rule, g, list[e], own, other, col, k0, k1, sweep, dE, dM, nacc);
  __syncwarp();
  return make_int3(dE, dM, nacc);
}

// One colour of one sweep.  grid: x = column/run tiles, y = chain of the launch.
// Thread t walks `run` consecutive rows of column k = t mod wc.  PR: Philox
// rounds of the acceptance planes (10, or 7 when the caller asks for it).
// BATCH: the chains of the launch are separately allocated (batch_* fields).
// The kernel is issue bound.  2D: each loop step updates two rows, whose
// loads, Philox evaluations and comparisons are independent and interleave,
// at two blocks per SM (up to 128 registers a thread, nothing rematerialised):
// +5 % over one row per step at three blocks per SM (85 registers).  3D: one
// row per step, three blocks per SM, except for the general (field) rules,
// which spilled at 85 registers: two blocks per SM, +3 % measured.
template <int Z, int RULE, int KG, int PR, bool BATCH>
__global__ void __launch_bounds__(MSC_THREADS, (Z == 4 || RULE >= RULE_GEN) ? 2 : 3)
    msc_halfsweep_kernel(const __grid_constant__ MscParams P) {
  __shared__ MscFix fix[MSC_WARPS][MSC_FIXCAP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lchain = blockIdx.y;
  const int chain = P.chain0 + lchain;
  const int group = BATCH ? (int)P.batch_group[lchain] : chain / P.chains_per_group;
  const MscGeom& g = P.g;
  const MscRule<Z, RULE> rule{P.tabs.kind[group], P.tabs.thr[group]};
  const uint32_t k0 = P.keys[lchain][0], k1 = P.keys[lchain][1];
  const uint32_t sweep = (P.cursor ? P.cursor[0] + P.sweep : P.sweep) + (BATCH ? P.batch_sweep[chain] : 0u);
  const uint32_t meas = P.cursor ? P.cursor[1] + P.meas : P.meas;
  const uint32_t col = (uint32_t)P.col;
  uint32_t* const lat = BATCH ? P.batch_spins[lchain] : P.spins + (size_t)chain * 2 * g.words;
  uint32_t* own = lat + (size_t)col * g.words;
  const uint32_t* other = lat + (size_t)(col ^ 1) * g.words;

  const uint32_t t = blockIdx.x * MSC_THREADS + threadIdx.x;
  const int k = (int)(t & (g.wc - 1));
  const int r0 = (int)(t >> g.wc_log2) * P.run;
  const uint32_t lt_mask = (1u << lane) - 1u;
  int nf = 0;  // entries in this warp's list (warp-uniform)
  int dE = 0, dM = 0, nacc = 0;
  // uniform part of the plane stream and, for the rules with few threshold
  // classes, the broadcast threshold bits of the inline planes
  critmc_plane_stream ps;
  critmc_plane_stream_init(&ps, k0, k1, sweep, col, KG);
  constexpr int NR = MscRule<Z, RULE>::NR;
  constexpr bool PRE = NR > 0 && NR <= 2;
  uint32_t pre[4 * KG][PRE ? NR : 1];
  if constexpr (PRE) rule.template prepare<KG>(pre);

  auto flush = [&]() {
    const int3 d = msc_flush<Z, RULE, KG, PR>(rule, g, fix[warp], nf, own, other, col, k0, k1, sweep);
    dE += d.x;
    dM += d.y;
    nacc += d.z;
    nf = 0;
  };

  auto defer = [&](const MscWord& w, uint32_t widx) {  // a word with undecided lanes goes on the list
    const uint32_t need = __ballot_sync(0xffffffffu, w.U != 0);
    if (need) {
      const int cnt = __popc(need);
      if (nf + cnt > MSC_FIXCAP) flush();
      if (w.U != 0) fix[warp][nf + __popc(need & lt_mask)] = MscFix{widx, w.U, w.D};
      nf += cnt;
    }
  };

  if constexpr (Z == 4) {
    // sliding window down the column over the other colour: rows r-1 (o_m) and r (o_c)
    uint32_t o_m = 0, o_c = 0;
    if (r0 < g.rows) {
      const int ym = (r0 == 0) ? g.ly - 1 : r0 - 1;
      o_m = other[CRITMC_IDX((size_t)ym * g.wc + k, g.words)];
      o_c = other[CRITMC_IDX((size_t)r0 * g.wc + k, g.words)];
    }
    const int kplus = (k == g.wc - 1) ? 0 : k + 1, kminus = (k == 0) ? g.wc - 1 : k - 1;
#pragma unroll 1
    for (int i = 0; i < P.run; i += 2) {  // rows a = r0 + i and b = a + 1
      const int ra = r0 + i, rb = ra + 1;
      const bool va = ra < g.rows, vb = (i + 1 < P.run) && (rb < g.rows);
      const uint32_t wa = (uint32_t)ra * g.wc + k, wb = (uint32_t)rb * g.wc + k;
      const int pa = (P.col + ra) & 1, pb = pa ^ 1;
      uint32_t o_p1 = 0, o_p2 = 0, adjA = 0, adjB = 0, ownA = 0, ownB = 0;
      if (va) {
        const int yp = (ra == g.ly - 1) ? 0 : ra + 1;
        o_p1 = other[CRITMC_IDX((size_t)yp * g.wc + k, g.words)];
        adjA = other[CRITMC_IDX((size_t)ra * g.wc + (pa ? kplus : kminus), g.words)];
        ownA = own[CRITMC_IDX(wa, g.words)];
      }
      if (vb) {
        const int yp = (rb == g.ly - 1) ? 0 : rb + 1;
        o_p2 = other[CRITMC_IDX((size_t)yp * g.wc + k, g.words)];
        adjB = other[CRITMC_IDX((size_t)rb * g.wc + (pb ? kplus : kminus), g.words)];
        ownB = own[CRITMC_IDX(wb, g.words)];
      }
      uint32_t nA[4], nB[4];
      nA[0] = o_c;
      nA[1] = pa ? __funnelshift_r(o_c, adjA, 1) : __funnelshift_l(adjA, o_c, 1);
      nA[2] = o_m;
      nA[3] = o_p1;
      nB[0] = o_p1;
      nB[1] = pb ? __funnelshift_r(o_p1, adjB, 1) : __funnelshift_l(adjB, o_p1, 1);
      nB[2] = o_c;
      nB[3] = o_p2;
      o_m = o_p1;
      o_c = o_p2;
      MscWord A, B;
      rule.classify(ownA, nA, A);
      rule.classify(ownB, nB, B);
      const critmc_plane_word_t pwa = critmc_plane_word(&ps, wa);
      const critmc_plane_word_t pwb = critmc_plane_word(&ps, wb);
#pragma unroll
      for (int grp = 0; grp < KG; ++grp) {
        const critmc_u32x4 xa = critmc_plane_group_rounds(&ps, pwa, grp, PR);
        const critmc_u32x4 xb = critmc_plane_group_rounds(&ps, pwb, grp, PR);
        msc_resolve<Z, RULE>(rule, A, xa, grp, PRE ? &pre[4 * grp][0] : nullptr);
        msc_resolve<Z, RULE>(rule, B, xb, grp, PRE ? &pre[4 * grp][0] : nullptr);
      }
      if (!va) A.U = 0;
      if (!vb) B.U = 0;
      const uint32_t sa = (RULE == RULE_HB0) ? A.D : (A.s ^ A.D);
      const uint32_t sb = (RULE == RULE_HB0) ? B.D : (B.s ^ B.D);
      if (va) {
        msc_obs<Z>((A.s ^ sa) & ~A.U, A.s, A.anti, dE, dM, nacc);
        if (A.U == 0) own[CRITMC_IDX(wa, g.words)] = sa;
      }
      if (vb) {
        msc_obs<Z>((B.s ^ sb) & ~B.U, B.s, B.anti, dE, dM, nacc);
        if (B.U == 0) own[CRITMC_IDX(wb, g.words)] = sb;
      }
      defer(A, wa);
      defer(B, wb);
    }
  } else {
#pragma unroll 1
    for (int i = 0; i < P.run; ++i) {
      const int r = r0 + i;
      const bool valid = r < g.rows;
      const uint32_t widx = (uint32_t)r * g.wc + k;
      MscWord w;
      w.U = 0;
      if (valid) {
        uint32_t n[Z];
        int y, z, kk;
        msc_row_coords<Z>(g, widx, y, z, kk);
        msc_neighbours<Z>(other, g, (int)col, y, z, k, n);
        rule.classify(own[CRITMC_IDX(widx, g.words)], n, w);
        const critmc_plane_word_t pw = critmc_plane_word(&ps, widx);
#pragma unroll
        for (int grp = 0; grp < KG; ++grp)
          msc_resolve<Z, RULE>(rule, w, critmc_plane_group_rounds(&ps, pw, grp, PR), grp,
                               PRE ? &pre[4 * grp][0] : nullptr);
        const uint32_t s_new = (RULE == RULE_HB0) ? w.D : (w.s ^ w.D);
        msc_obs<Z>((w.s ^ s_new) & ~w.U, w.s, w.anti, dE, dM, nacc);
        if (w.U == 0) own[CRITMC_IDX(widx, g.words)] = s_new;
      }
      defer(w, widx);
    }
  }
  if (nf) flush();
  // observable increments: warp reduction, one atomic per quantity and warp
  dE = warp_sum(dE);
  dM = warp_sum(dM);
  nacc = warp_sum(nacc);
  if (lane == 0 && P.acc) {
    unsigned long long* dst = P.acc + ((size_t)meas * P.n_chains + chain) * 3;
    if (dE) atomicAdd(dst + 0, as_ull(dE));
    if (dM) atomicAdd(dst + 1, as_ull(dM));
    if (nacc) atomicAdd(dst + 2, as_ull(nacc));
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

// Output pointers of the chains of a batch (critmc_ising_msc_run_batch).
struct MscBatchOut {
  long long* running[CRITMC_MSC_BATCH_MAX];
  long long* e_out[CRITMC_MSC_BATCH_MAX];
  long long* m_out[CRITMC_MSC_BATCH_MAX];
  long long* aux_out[CRITMC_MSC_BATCH_MAX];
};

// msc_finalize_kernel for separately allocated chains: block c scans chain c's
// increments into its own series and running sums.
__global__ void msc_finalize_batch_kernel(const long long* __restrict__ acc, const __grid_constant__ MscBatchOut O,
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
  long long* running = O.running[chain];
  if (tid == 0) {
    long long ce = running[0], cm = running[1];
    for (int q = 0; q < nt; ++q) {
      const long long te = se[q], tm = sm[q];
      se[q] = ce;
      sm[q] = cm;
      ce += te;
      cm += tm;
    }
    running[0] = ce;
    running[1] = cm;
  }
  __syncthreads();
  long long ce = se[tid], cm = sm[tid];
  long long *e_out = O.e_out[chain], *m_out = O.m_out[chain], *aux_out = O.aux_out[chain];
  for (int i = b; i < e; ++i) {
    const size_t src = ((size_t)i * n_chains + chain) * 3;
    ce += acc[src + 0];
    cm += acc[src + 1];
    e_out[i] = ce;
    m_out[i] = cm;
    aux_out[(size_t)i * 4 + 0] = acc[src + 2];
    aux_out[(size_t)i * 4 + 1] = 0;
    aux_out[(size_t)i * 4 + 2] = 0;
    aux_out[(size_t)i * 4 + 3] = 0;
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

// Hot (random) or cold start of MSC chains from the Philox init stream:
// word w of colour c = word 0 of Philox(w, 0, TAG_INIT | c << 16, 0).
__global__ void msc_init_kernel(uint32_t* spins, MscGeom g, const uint32_t* __restrict__ keys,
                                int start) {
  const int chain = blockIdx.y;
  const uint32_t k0 = keys[2 * chain], k1 = keys[2 * chain + 1];
  uint32_t* base = spins + (size_t)chain * 2 * g.words;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * g.words; i += gridDim.x * blockDim.x) {
    const uint32_t col = i >= g.words, w = i - col * g.words;
    uint32_t v;
    if (start == 0) v = critmc_philox4x32(w, 0u, CRITMC_TAG_INIT | (col << 16), 0u, k0, k1).v[0];
    else v = start > 0 ? ~0u : 0u;
    base[i] = v;
  }
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

template <int Z, int RULE, int PR>
static void launch_half_kg(const MscParams& P, int kg, cudaStream_t st) {
  const long long threads = (long long)P.g.wc * ((P.g.rows + P.run - 1) / P.run);
  const dim3 grid((unsigned)((threads + MSC_THREADS - 1) / MSC_THREADS), P.n_chains - P.chain0 < MSC_PCHAINS ? P.n_chains - P.chain0 : MSC_PCHAINS);
  if constexpr (PR == CRITMC_PHILOX_ROUNDS) {
    if (P.batch_sweep) {  // batches: 8 inline planes, default stream only
      msc_halfsweep_kernel<Z, RULE, 2, PR, true><<<grid, MSC_THREADS, 0, st>>>(P);
      return;
    }
  }
  if (kg == 1) msc_halfsweep_kernel<Z, RULE, 1, PR, false><<<grid, MSC_THREADS, 0, st>>>(P);
  else msc_halfsweep_kernel<Z, RULE, 2, PR, false><<<grid, MSC_THREADS, 0, st>>>(P);
}

template <int Z, int PR>
static void launch_half_z(const MscParams& P, int rule, int kg, cudaStream_t st) {
  switch (rule) {
    case RULE_METRO0: launch_half_kg<Z, RULE_METRO0, PR>(P, kg, st); break;
    case RULE_HB0: launch_half_kg<Z, RULE_HB0, PR>(P, kg, st); break;
    case RULE_GEN: launch_half_kg<Z, RULE_GEN, PR>(P, kg, st); break;
    default: launch_half_kg<Z, RULE_GENSPIN, PR>(P, kg, st); break;
  }
}

// One half-sweep of every chain, in launches of at most MSC_PCHAINS chains.
// pr: Philox rounds of the acceptance planes (10, or 7 on request).
void msc_launch_half(MscParams& P, const uint32_t* keys, int rule, int kg, int pr, cudaStream_t st) {
  for (int c0 = 0; c0 < P.n_chains; c0 += MSC_PCHAINS) {
    P.chain0 = c0;
    const int nc = std::min(MSC_PCHAINS, P.n_chains - c0);
    std::memcpy(P.keys, keys + 2 * (size_t)c0, sizeof(uint32_t) * 2 * nc);
    if (pr == 7) {
      if (P.g.dim == 2) launch_half_z<4, 7>(P, rule, kg, st);
      else launch_half_z<6, 7>(P, rule, kg, st);
    } else {
      if (P.g.dim == 2) launch_half_z<4, CRITMC_PHILOX_ROUNDS>(P, rule, kg, st);
      else launch_half_z<6, CRITMC_PHILOX_ROUNDS>(P, rule, kg, st);
    }
  }
}

// Launch the half-sweeps of n_meas schedule applications on stream s: one
// launch per half-sweep (mode 1), or CUDA graphs of G measurements replayed
// with a device cursor (mode 3; the graph is cached by its parameters).
// sweep0 is the first sweep of the call (contiguous chains) or 0 (batches,
// whose per-chain bases the kernels add).
static int msc_launch_schedule(MscParams (&P)[2], const int (&rule)[2], const uint32_t* keys, int n_chains,
                               const int64_t* schedule, int n_rows, long long sweeps_per_meas, int n_meas,
                               uint32_t sweep0, int mode, int kg, int pr, uint32_t* cursor, cudaStream_t s) {
  auto launch_meas = [&](uint32_t sweep_rel, uint32_t meas_rel, const uint32_t* cur) {
    uint32_t sw = sweep_rel;
    for (int r = 0; r < n_rows; ++r) {
      const int slot = schedule[2 * r] == CRITMC_HEATBATH ? 1 : 0;
      MscParams& q = P[slot];
      q.cursor = cur;
      for (int64_t rep = 0; rep < schedule[2 * r + 1]; ++rep) {
        q.sweep = sw;
        q.meas = meas_rel;
        q.col = 0;
        msc_launch_half(q, keys, rule[slot], kg, pr, s);
        q.col = 1;
        msc_launch_half(q, keys, rule[slot], kg, pr, s);
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
      // the graph depends on the parameters below only: reuse it across calls
      int dev = 0;
      cudaGetDevice(&dev);
      GraphKey key;
      key.add(0x4d534347u).add(dev).add(G).add(n_rows).add(rule).add(kg).add(pr);
      key.add_bytes(schedule, sizeof(int64_t) * 2 * n_rows).add_bytes(keys, sizeof(uint32_t) * 2 * n_chains);
      for (int slot = 0; slot < 2; ++slot) {
        MscParams& q = P[slot];
        q.cursor = cursor;
        q.sweep = q.meas = 0;
        q.col = q.chain0 = 0;
        std::memset(q.keys, 0, sizeof(q.keys));
        key.add(q);
      }
      cudaGraphExec_t exec = graph_cache_find(key);
      if (!exec) {
        cudaGraph_t graph;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
          return cuda_fail("capture");
        for (int m = 0; m < G; ++m) launch_meas((uint32_t)(m * sweeps_per_meas), (uint32_t)m, cursor);
        msc_cursor_bump<<<1, 1, 0, s>>>(cursor, (uint32_t)(G * sweeps_per_meas), (uint32_t)G);
        if (cudaStreamEndCapture(s, &graph) != cudaSuccess) return cuda_fail("end capture");
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return cuda_fail("instantiate");
        graph_cache_insert(key, exec);
      }
      for (int i = 0; i < n_graph; ++i) cudaGraphLaunch(exec, s);
    }
    const int done = n_graph > 1 ? n_graph * G : 0;
    for (int m = done; m < n_meas; ++m)
      launch_meas((uint32_t)(sweep0 + (uint32_t)(m * sweeps_per_meas)), (uint32_t)m, nullptr);
  }
  return CRITMC_OK;
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
  const int run_code = (mode >> 8) & 0xF;  // tuning: rows walked per thread, 2^(code-1); 0 = automatic
  if ((mode & ~0x1FFF) || run_code > 6)
    return fail(CRITMC_ERR_INVALID, "mode: bits 8..11 must be 0..6, bit 12 selects Philox4x32-7, no higher bits");
  const int pr = (mode & CRITMC_MSC_PHILOX7) ? 7 : CRITMC_PHILOX_ROUNDS;  // a stream choice, not a tuning knob
  mode &= 0xFF;
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

  // rows walked per thread: long runs reuse the sliding window, short runs
  // keep enough threads in flight when few chains are batched
  const long long col_threads = (long long)n_chains * g.wc * g.rows;
  int run = 8;
  while (run > 1 && col_threads / run < 148LL * 1536) run /= 2;
  if (run_code) run = 1 << (run_code - 1);

  static thread_local MscParams P[2];
  for (int slot = 0; slot < 2; ++slot) {
    MscParams& q = P[slot];
    q.spins = spins;
    q.acc = acc;
    q.batch_sweep = nullptr;
    q.g = g;
    q.n_chains = n_chains;
    q.chains_per_group = n_chains / n_groups;
    q.run = run;
    q.tabs = tabs[slot];
  }
  const int kg = k_inline / 4;
  if ((st = msc_launch_schedule(P, rule, keys, n_chains, schedule, n_rows, sweeps_per_meas, n_meas, sweep0, mode, kg,
                                pr, cursor, s)))
    return st;
  msc_finalize_kernel<<<n_chains, 256, 0, s>>>((const long long*)acc, (long long*)running,
                                                (long long*)e_out, (long long*)m_out,
                                                (long long*)aux_out, n_chains, n_meas);
  if (int e_ = cuda_check("launch")) return e_;
  return cs.finish();
}

extern "C" int64_t critmc_ising_msc_batch_scratch_bytes(int32_t n_chains, int32_t n_meas) {
  return 256 + (int64_t)n_chains * n_meas * 3 * 8;
}

extern "C" int32_t critmc_ising_msc_run_batch(const critmc_msc_chain* chains, int32_t n_chains, int32_t dim,
                                              int32_t lx, int32_t ly, int32_t lz, const uint32_t* tables,
                                              int32_t n_tables, const int64_t* schedule, int32_t n_rows,
                                              int32_t n_meas, void* scratch, int32_t mode, void* stream) {
  clear_error();
  MscGeom g;
  int st = msc_geom(dim, lx, ly, lz, g);
  if (st) return st;
  if (!chains || !tables || !scratch || !schedule) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_chains > CRITMC_MSC_BATCH_MAX)
    return fail(CRITMC_ERR_INVALID, "a batch holds 1..CRITMC_MSC_BATCH_MAX (16) chains");
  if (n_tables < 1 || n_tables > MSC_MAX_GROUPS) return fail(CRITMC_ERR_INVALID, "n_tables must be in [1, 16]");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  if (n_rows < 1) return fail(CRITMC_ERR_INVALID, "empty schedule");
  long long sweeps_per_meas = 0;
  for (int r = 0; r < n_rows; ++r) {
    const int64_t code = schedule[2 * r], reps = schedule[2 * r + 1];
    if (code != CRITMC_METROPOLIS && code != CRITMC_HEATBATH)
      return fail(CRITMC_ERR_UNSUPPORTED, "MSC Ising runs checkerboard metropolis and heatbath rows only");
    if (reps < 1) return fail(CRITMC_ERR_INVALID, "schedule repetitions must be positive");
    sweeps_per_meas += reps;
  }
  const int run_code = (mode >> 8) & 0xF;
  if ((mode & ~0xFFF) || run_code > 6) return fail(CRITMC_ERR_INVALID, "mode: bits 8..11 must be 0..6, no higher bits");
  mode &= 0xFF;
  if (mode == 0) mode = 3;
  if (mode != 1 && mode != 3) return fail(CRITMC_ERR_UNSUPPORTED, "mode must be 0, 1 or 3");
  std::vector<uint32_t> keys(2 * (size_t)n_chains), sweeps(n_chains);
  for (int c = 0; c < n_chains; ++c) {
    const critmc_msc_chain& ch = chains[c];
    if (!ch.spins || !ch.running || !ch.e_out || !ch.m_out || !ch.aux_out)
      return fail(CRITMC_ERR_INVALID, "batch chain with a null pointer");
    if (ch.table < 0 || ch.table >= n_tables) return fail(CRITMC_ERR_INVALID, "batch chain table out of range");
    if ((long long)ch.sweep0 + sweeps_per_meas * (long long)n_meas > 0xFFFFFFFFLL)
      return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");
    keys[2 * c] = ch.key[0];
    keys[2 * c + 1] = ch.key[1];
    sweeps[c] = ch.sweep0;
  }
  if (n_meas == 0) return CRITMC_OK;

  MscTables tabs[2];
  int rule[2];
  for (int slot = 0; slot < 2; ++slot) {
    std::memset(&tabs[slot], 0, sizeof(MscTables));
    for (int gi = 0; gi < n_tables; ++gi) {
      const uint32_t* src = tables + (size_t)gi * 4 * CRITMC_NCLS + slot * 2 * CRITMC_NCLS;
      std::memcpy(tabs[slot].kind[gi], src, CRITMC_NCLS * 4);
      std::memcpy(tabs[slot].thr[gi], src + CRITMC_NCLS, CRITMC_NCLS * 4);
    }
    rule[slot] = msc_pick_rule(&tabs[slot].kind[0][0], &tabs[slot].thr[0][0], 2 * dim,
                               slot ? CRITMC_HEATBATH : CRITMC_METROPOLIS, n_tables);
  }

  CaptureStream cs;
  if ((st = cs.begin(stream))) return st;
  cudaStream_t s = cs.work;
  uint32_t* cursor = (uint32_t*)scratch;
  uint32_t* sweep_dev = (uint32_t*)((char*)scratch + 16);
  unsigned long long* acc = (unsigned long long*)((char*)scratch + 256);
  if (cudaMemcpyAsync(sweep_dev, sweeps.data(), 4 * (size_t)n_chains, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return cuda_fail("copy sweep bases");
  if (cudaMemsetAsync(acc, 0, (size_t)n_chains * n_meas * 3 * 8, s) != cudaSuccess) return cuda_fail("memset");

  const long long col_threads = (long long)n_chains * g.wc * g.rows;
  int run = 8;
  while (run > 1 && col_threads / run < 148LL * 1536) run /= 2;
  if (run_code) run = 1 << (run_code - 1);

  static thread_local MscParams P[2];
  for (int slot = 0; slot < 2; ++slot) {
    MscParams& q = P[slot];
    std::memset(&q, 0, sizeof(MscParams));
    q.acc = acc;
    q.batch_sweep = sweep_dev;
    for (int c = 0; c < n_chains; ++c) {
      q.batch_spins[c] = chains[c].spins;
      q.batch_group[c] = (uint32_t)chains[c].table;
    }
    q.g = g;
    q.n_chains = n_chains;
    q.chains_per_group = 1;
    q.run = run;
    q.tabs = tabs[slot];
  }
  if ((st = msc_launch_schedule(P, rule, keys.data(), n_chains, schedule, n_rows, sweeps_per_meas, n_meas, 0u, mode,
                                2, CRITMC_PHILOX_ROUNDS, cursor, s)))
    return st;
  MscBatchOut out;
  std::memset(&out, 0, sizeof(out));
  for (int c = 0; c < n_chains; ++c) {
    out.running[c] = (long long*)chains[c].running;
    out.e_out[c] = (long long*)chains[c].e_out;
    out.m_out[c] = (long long*)chains[c].m_out;
    out.aux_out[c] = (long long*)chains[c].aux_out;
  }
  msc_finalize_batch_kernel<<<n_chains, 256, 0, s>>>((const long long*)acc, out, n_chains, n_meas);
  if (int e_ = cuda_check("launch")) return e_;
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
  if (int e_ = cuda_check("launch")) return e_;
  return CRITMC_OK;
}

extern "C" int32_t critmc_ising_msc_init(uint32_t* spins, int32_t dim, int32_t lx, int32_t ly,
                                         int32_t lz, int32_t n_chains, const uint32_t* keys,
                                         int32_t start, void* stream) {
  clear_error();
  MscGeom g;
  int st = msc_geom(dim, lx, ly, lz, g);
  if (st) return st;
  if (!spins || !keys) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_chains > 65535) return fail(CRITMC_ERR_INVALID, "n_chains must be in [1, 65535]");
  if (start < -1 || start > 1) return fail(CRITMC_ERR_INVALID, "start must be 0 (random), 1 (up) or -1 (down)");
  cudaStream_t s = (cudaStream_t)stream;
  const dim3 grid(std::min<uint32_t>(2048, (2 * g.words + 255) / 256), n_chains);
  msc_init_kernel<<<grid, 256, 0, s>>>(spins, g, keys, start);
  if (int e_ = cuda_check("launch")) return e_;
  return CRITMC_OK;
}

// ---------------------------------------------------------------------------
// Variant of critmc_ising_msc_run that allocates nothing.
//
// Some callers cannot allocate device memory where they run the sampler: a
// plugin inside a host application whose framework owns the device allocator
// (a caching allocator or a memory pool with a fixed budget), code that must
// not call cudaMalloc because it would synchronise the device and stall other
// work, or an embedded host that forbids allocation after start-up.  This
// entry point takes its scratch (the measurement accumulators) from a
// file-scope device array instead of a caller buffer.
// ---------------------------------------------------------------------------
namespace critmc {

constexpr size_t MSC_NOALLOC_SCRATCH_BYTES = 1u << 20;  // 1 MiB on every device that loads the library
static __device__ __align__(256) unsigned char g_msc_noalloc_scratch[MSC_NOALLOC_SCRATCH_BYTES];

// Device address of the array on each device.  In host code the array's name
// is only a stand-in for the symbol, never a device address, so it is resolved
// with cudaGetSymbolAddress while that device is current.  The address is
// cached per device together with the unique id of the context it belongs to:
// a lookup that failed is retried on the next call, and after a
// cudaDeviceReset (which unloads the module, so the array may come back at
// another address) the new context's id differs and the address is looked
// up again instead of being written through stale.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);

struct NoallocSlot {
  void* addr = nullptr;
  unsigned long long ctx_id = 0;
  bool valid = false;
};
static NoallocSlot g_noalloc[64];
static std::mutex g_noalloc_mu;

// unique id of the calling thread's current context (0 if unavailable)
static unsigned long long current_context_id() {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (PfnCtxGetCurrent)fn;
    fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (PfnCtxGetId)fn;
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

static int noalloc_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return cuda_fail("cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(CRITMC_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocSlot& slot = g_noalloc[dev];
  const unsigned long long ctx_id = current_context_id();
  if (!slot.valid || ctx_id == 0 || slot.ctx_id != ctx_id) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_msc_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      slot.valid = false;  // not cached: the next call looks it up again
      set_error(cudaGetErrorString(e));
      return CRITMC_ERR_CUDA;
    }
    slot.addr = addr;
    slot.ctx_id = current_context_id();  // the lookup has made the context current if it was not
    slot.valid = slot.ctx_id != 0;
  }
  *out = slot.addr;
  return CRITMC_OK;
}

}  // namespace critmc

extern "C" int64_t critmc_ising_msc_noalloc_max_scratch_bytes(void) {
  return (int64_t)MSC_NOALLOC_SCRATCH_BYTES;
}

extern "C" int32_t critmc_ising_msc_run_noalloc(uint32_t* spins, int32_t dim, int32_t lx, int32_t ly,
                                                int32_t lz, int32_t n_chains, const uint32_t* keys,
                                                const uint32_t* tables, int32_t n_groups,
                                                uint32_t sweep0, const int64_t* schedule,
                                                int32_t n_rows, int32_t n_meas, int64_t* running,
                                                int64_t* e_out, int64_t* m_out, int64_t* aux_out,
                                                int32_t k_inline, void* stream) {
  clear_error();
  MscGeom g;
  int st = msc_geom(dim, lx, ly, lz, g);
  if (st) return st;
  if (!spins || !keys || !tables || !running || !e_out || !m_out || !aux_out)
    return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n_chains > 65535) return fail(CRITMC_ERR_INVALID, "n_chains must be in [1, 65535]");
  if (n_groups < 1 || n_groups > MSC_MAX_GROUPS || n_chains % n_groups != 0)
    return fail(CRITMC_ERR_INVALID, "n_groups must be in [1, 16] and divide n_chains");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  if (!schedule || n_rows < 1) return fail(CRITMC_ERR_INVALID, "empty schedule");
  if (k_inline != 4 && k_inline != 8) return fail(CRITMC_ERR_INVALID, "k_inline must be 4 or 8");
  if (critmc_ising_msc_scratch_bytes(n_chains, n_meas) > (int64_t)MSC_NOALLOC_SCRATCH_BYTES)
    return fail(CRITMC_ERR_INVALID,
                "n_chains * n_meas too large for the built-in 1 MiB scratch (at most 43690); "
                "split the call or use critmc_ising_msc_run with caller scratch");
  long long sweeps_per_meas = 0;
  for (int r = 0; r < n_rows; ++r) {
    const int64_t code = schedule[2 * r], reps = schedule[2 * r + 1];
    if (code != CRITMC_METROPOLIS && code != CRITMC_HEATBATH)
      return fail(CRITMC_ERR_UNSUPPORTED, "MSC Ising runs checkerboard metropolis and heatbath rows only");
    if (reps < 1) return fail(CRITMC_ERR_INVALID, "schedule repetitions must be positive");
    sweeps_per_meas += reps;
  }
  if ((long long)sweep0 + sweeps_per_meas * (long long)n_meas > 0xFFFFFFFFLL)
    return fail(CRITMC_ERR_INVALID, "sweep counter would pass 2^32");
  if (n_meas == 0) return CRITMC_OK;
  void* scratch = nullptr;
  if ((st = noalloc_scratch(&scratch))) return st;

  static thread_local MscTables tabs[2];
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
  cudaStream_t s = (cudaStream_t)stream;
  // the array keeps the previous call's contents: clear the accumulators
  unsigned long long* acc = (unsigned long long*)((char*)scratch + 16);
  if (cudaMemsetAsync(acc, 0, (size_t)n_chains * n_meas * 3 * 8, s) != cudaSuccess)
    return cuda_fail("memset");
  const long long col_threads = (long long)n_chains * g.wc * g.rows;
  int run = 8;
  while (run > 1 && col_threads / run < 148LL * 1536) run /= 2;
  static thread_local MscParams P[2];
  for (int slot = 0; slot < 2; ++slot) {
    MscParams& q = P[slot];
    q.spins = spins;
    q.acc = acc;
    q.batch_sweep = nullptr;
    q.cursor = nullptr;
    q.g = g;
    q.n_chains = n_chains;
    q.chains_per_group = n_chains / n_groups;
    q.run = run;
    q.tabs = tabs[slot];
  }
  uint32_t sw = sweep0;
  for (int meas = 0; meas < n_meas; ++meas)
    for (int r = 0; r < n_rows; ++r) {
      const int slot = schedule[2 * r] == CRITMC_HEATBATH ? 1 : 0;
      for (int64_t rep = 0; rep < schedule[2 * r + 1]; ++rep) {
        P[slot].sweep = sw;
        P[slot].meas = (uint32_t)meas;
        P[slot].col = 0;
        msc_launch_half(P[slot], keys, rule[slot], k_inline / 4, CRITMC_PHILOX_ROUNDS, s);
        P[slot].col = 1;
        msc_launch_half(P[slot], keys, rule[slot], k_inline / 4, CRITMC_PHILOX_ROUNDS, s);
        ++sw;
      }
    }
  msc_finalize_kernel<<<n_chains, 256, 0, s>>>((const long long*)acc, (long long*)running,
                                                (long long*)e_out, (long long*)m_out,
                                                (long long*)aux_out, n_chains, n_meas);
  if (int e_ = cuda_check("launch")) return e_;
  return CRITMC_OK;
}

// ---------------------------------------------------------------------------
// Resident MSC chains as work items: the whole lattice of a chain sits in
// shared memory while its block applies the schedule n_meas times.  Same
// random stream as the half-sweep kernel (word index, sweep, colour).
// ---------------------------------------------------------------------------
#include "items_host.h"

namespace critmc {

constexpr int MSCI_WARPS = ITEM_THREADS / 32;

// one colour of one sweep (CL > 1: the words are split over the team's blocks)
template <int Z, int RULE, int CL>
__device__ void msci_colour(const MscRule<Z, RULE>& rule, const MscGeom& g, uint32_t* lat, int c,
                            uint32_t sweep, uint32_t k0, uint32_t k1, MscFix (*fix)[64],
                            long long& dE, long long& dM, long long& nacc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt_mask = (1u << lane) - 1u;
  uint32_t* own = lat + (size_t)c * g.words;
  const uint32_t* other = lat + (size_t)(c ^ 1) * g.words;
  int idE = 0, idM = 0, inacc = 0;
  int nf = 0;
  auto flush = [&]() {
    __syncwarp();
    for (int e = lane; e < nf; e += 32) {
      const MscFix f = fix[warp][e];
      int y, z, k;
      msc_row_coords<Z>(g, f.w, y, z, k);
      uint32_t n[Z];
      msc_neighbours<Z>(other, g, c, y, z, k, n);
      MscWord w;
      rule.classify(own[f.w], n, w);
      w.D = f.D;
      w.U = f.U;
      for (int grp = 2; grp < 8 && w.U != 0; ++grp) msc_group<Z, RULE>(rule, w, k0, k1, f.w, sweep, (uint32_t)c, grp);
      const uint32_t s_new = (RULE == RULE_HB0) ? w.D : (w.s ^ w.D);
      msc_obs<Z>((w.s ^ s_new) & f.U, w.s, w.anti, idE, idM, inacc);
      own[f.w] = s_new;
    }
    __syncwarp();
    nf = 0;
  };
  constexpr uint32_t stride = (uint32_t)CL * ITEM_THREADS;
  const uint32_t t0 = Team<CL>::rank() * ITEM_THREADS + threadIdx.x;
  const uint32_t rounds = (g.words + stride - 1) / stride;  // the same for the whole team
  for (uint32_t it = 0; it < rounds; ++it) {
    const uint32_t widx = it * stride + t0;
    MscWord w;
    w.U = 0;
    if (widx < g.words) {
      int y, z, k;
      msc_row_coords<Z>(g, widx, y, z, k);
      uint32_t n[Z];
      msc_neighbours<Z>(other, g, c, y, z, k, n);
      rule.classify(own[widx], n, w);
      msc_group<Z, RULE>(rule, w, k0, k1, widx, sweep, (uint32_t)c, 0);
      msc_group<Z, RULE>(rule, w, k0, k1, widx, sweep, (uint32_t)c, 1);
      const uint32_t s_new = (RULE == RULE_HB0) ? w.D : (w.s ^ w.D);
      msc_obs<Z>((w.s ^ s_new) & ~w.U, w.s, w.anti, idE, idM, inacc);
      if (w.U == 0) own[widx] = s_new;
    }
    const uint32_t need = __ballot_sync(0xffffffffu, w.U != 0);
    if (need) {
      const int cnt = __popc(need);
      if (nf + cnt > 64) flush();
      if (w.U != 0) fix[warp][nf + __popc(need & lt_mask)] = MscFix{widx, w.U, w.D};
      nf += cnt;
    }
  }
  if (nf) flush();
  dE += idE;
  dM += idM;
  nacc += inacc;
  Team<CL>::sync();
}

// CL == 1: one block, the lattice copied into shared memory (`lat`).  CL > 1:
// a cluster of CL blocks updates the lattice in global memory, the cluster
// barrier separating the colours, and block 0 adds the blocks' sums from
// distributed shared memory; the same spins and series for every CL (a
// colour's words are independent, the sums are integers).  Block 0's thread 0
// alone polls the control and passes its answer to all blocks before the
// barrier that ends a measurement.
template <int Z, int CL>
__device__ void msci_chain(const critmc_item& it, uint32_t* lat, MscFix (*fix)[64], const RunCtl* ctl,
                           CtlPoll* poll) {
  using T = Team<CL>;
  __shared__ long long red[MSCI_WARPS];
  __shared__ int s_stop[2];
  __shared__ long long part[CL > 1 ? 2 : 1][CL][3];
  MscGeom g;
  msc_geom_device(it.dim, it.lx, it.ly, it.lz, g);
  uint32_t* gl = reinterpret_cast<uint32_t*>(it.spins);
  const int tid = threadIdx.x;
  const unsigned rank = T::rank();
  if constexpr (CL == 1) {
    for (uint32_t j = tid; j < 2 * g.words; j += ITEM_THREADS) lat[j] = gl[j];
  } else {
    lat = gl;
    if (tid == 0) s_stop[0] = 0;
  }
  T::sync();
  long long e_run = it.running[0], m_run = it.running[1];
  uint32_t sweep = it.sweep0;
  for (int meas = 0; meas < it.n_meas; ++meas) {
    if constexpr (CL == 1) {
      if (ctl) {  // stop between measurements when the budget or a cancel says so
        if (tid == 0) s_stop[0] = poll->check(*ctl);
        __syncthreads();
        if (s_stop[0]) break;
      }
    } else {
      if (s_stop[meas & 1]) break;  // block 0's answer, written before the last barrier
    }
    long long dE = 0, dM = 0, nacc = 0;
    for (int row = 0; row < it.n_rows; ++row) {
      const int slot = it.codes[row] == CRITMC_HEATBATH ? 1 : 0;
      const uint32_t* kd = it.kind_tab[slot];
      const uint32_t* th = it.thr_tab[slot];
      for (int rep = 0; rep < it.reps[row]; ++rep) {
        for (int c = 0; c < 2; ++c) {
          switch (it.rule[slot]) {
            case RULE_METRO0:
              msci_colour<Z, RULE_METRO0, CL>(MscRule<Z, RULE_METRO0>{kd, th}, g, lat, c, sweep, it.key[0], it.key[1], fix, dE, dM, nacc);
              break;
            case RULE_HB0:
              msci_colour<Z, RULE_HB0, CL>(MscRule<Z, RULE_HB0>{kd, th}, g, lat, c, sweep, it.key[0], it.key[1], fix, dE, dM, nacc);
              break;
            case RULE_GEN:
              msci_colour<Z, RULE_GEN, CL>(MscRule<Z, RULE_GEN>{kd, th}, g, lat, c, sweep, it.key[0], it.key[1], fix, dE, dM, nacc);
              break;
            default:
              msci_colour<Z, RULE_GENSPIN, CL>(MscRule<Z, RULE_GENSPIN>{kd, th}, g, lat, c, sweep, it.key[0], it.key[1], fix, dE, dM, nacc);
              break;
          }
        }
        ++sweep;
      }
    }
    dE = warp_sum(dE);
    dM = warp_sum(dM);
    nacc = warp_sum(nacc);
    long long tot[3] = {0, 0, 0};
    const long long vals[3] = {dE, dM, nacc};
    for (int q = 0; q < 3; ++q) {
      if ((tid & 31) == 0) red[tid >> 5] = vals[q];
      __syncthreads();
      for (int w = 0; w < MSCI_WARPS; ++w) tot[q] += red[w];
      __syncthreads();
    }
    if constexpr (CL > 1) {
      if (tid == 0) {
        long long* p = T::at(&part[meas & 1][rank][0], 0);
        p[0] = tot[0];
        p[1] = tot[1];
        p[2] = tot[2];
      }
      if (rank == 0 && tid == 0) {
        const int stop = ctl ? poll->check(*ctl) : 0;
        for (int r = 0; r < CL; ++r) *T::at(&s_stop[(meas + 1) & 1], (unsigned)r) = stop;
      }
      T::sync();
      // part of this parity is next written two measurements on, after
      // barriers that block 0 passes once it is done here
      tot[0] = tot[1] = tot[2] = 0;
      if (rank == 0 && tid == 0)
        for (int r = 0; r < CL; ++r)
          for (int q = 0; q < 3; ++q) tot[q] += part[meas & 1][r][q];
    }
    e_run += tot[0];
    m_run += tot[1];
    if (rank == 0 && tid == 0) {
      reinterpret_cast<long long*>(it.e_out)[meas] = e_run;
      reinterpret_cast<long long*>(it.vec_out)[meas] = m_run;
      it.aux_out[4 * meas + 0] = tot[2];
      it.aux_out[4 * meas + 1] = 0;
      it.aux_out[4 * meas + 2] = 0;
      it.aux_out[4 * meas + 3] = 0;
    }
  }
  if constexpr (CL == 1)
    for (uint32_t j = tid; j < 2 * g.words; j += ITEM_THREADS) gl[j] = lat[j];
  if (rank == 0 && tid == 0) {
    it.running[0] = e_run;
    it.running[1] = m_run;
  }
  T::sync();
}

// CL > 1: each item is advanced by a cluster of CL blocks (block 0 takes the
// item from the queue and hands its index to the others).
template <int CL>
__global__ void __launch_bounds__(ITEM_THREADS) msc_items_kernel(const critmc_item* items, int n,
                                                                 unsigned* queue, RunCtl ctl) {
  using T = Team<CL>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ MscFix fix[MSCI_WARPS][64];
  __shared__ int cur;
  uint32_t* lat = reinterpret_cast<uint32_t*>(smem_raw);
  CtlPoll poll;
  poll.start();
  const RunCtl* pc = ctl.status ? &ctl : nullptr;
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
    if (it.dim == 2) msci_chain<4, CL>(it, lat, fix, pc, &poll);
    else msci_chain<6, CL>(it, lat, fix, pc, &poll);
  }
}

int msc_items_team_clusters(int team) {
  switch (team) {
    case 2: return team_clusters(msc_items_kernel<2>, 2, ITEM_THREADS);
    case 4: return team_clusters(msc_items_kernel<4>, 4, ITEM_THREADS);
    case 8: return team_clusters(msc_items_kernel<8>, 8, ITEM_THREADS);
    case 16: return team_clusters(msc_items_kernel<16>, 16, ITEM_THREADS);
    default: return fail(CRITMC_ERR_INVALID, "team size must be 2, 4, 8 or 16");
  }
}

int msc_items_launch(const critmc_item* items, int n, unsigned* queue, size_t smem, int team, const RunCtl& ctl,
                     cudaStream_t s) {
  switch (team) {
    case 2: return launch_team(msc_items_kernel<2>, 2, ITEM_THREADS, n, s, items, n, queue, ctl);
    case 4: return launch_team(msc_items_kernel<4>, 4, ITEM_THREADS, n, s, items, n, queue, ctl);
    case 8: return launch_team(msc_items_kernel<8>, 8, ITEM_THREADS, n, s, items, n, queue, ctl);
    case 16: return launch_team(msc_items_kernel<16>, 16, ITEM_THREADS, n, s, items, n, queue, ctl);
    default: break;
  }
  auto kern = msc_items_kernel<1>;
  if (smem > 0 &&  // static + dynamic may pass 48 KiB
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return cuda_fail("shared memory attribute");
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ITEM_THREADS, smem);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, std::min(n, std::max(1, per_sm) * sms));
  kern<<<grid, ITEM_THREADS, smem, s>>>(items, n, queue, ctl);
  if (int e_ = cuda_check("launch")) return e_;
  return CRITMC_OK;
}

}  // namespace critmc
