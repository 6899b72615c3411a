// Multi-spin-coded Ising sweeps: per-word device logic shared by the
// half-sweep kernel (lattice in HBM) and the resident kernel (lattice in
// shared memory).
//
// Stream definition (what the CPU replay in oracle/ reproduces):
//   For word w (index inside its colour class: w = row*wc + k) of colour `col`
//   at sweep t, plane q (0..31) is word (q & 3) of
//       Philox4x32-10(c0 = w, c1 = t, c2 = TAG_PLANES | (q >> 2) << 8 | col << 16,
//                     c3 = 0; key = chain key).
//   Lane j of the word draws the 32-bit uniform u_j whose bit (31 - q) is bit j
//   of plane q.  The lane's decision is (u_j < thr[class]) for RANDOM classes.
// The kernels compare u_j with thr most-significant bit first and stop
// drawing planes once every lane of the word is decided; how many planes are
// evaluated inline is a tuning choice that does not change u_j.
//
// Per plane the comparison needs, for every undecided lane, the threshold bit
// of its class.  Rules below produce that bit plane from the lane's neighbour
// count with as few lop3 operations as the class structure allows; the
// thresholds are uniform per chain group (kernel parameters), so the
// broadcasts run on the uniform datapath.
#pragma once
#include "common.cuh"

namespace critmc {

struct MscGeom {
  int dim, lx, ly, lz;
  int wc, wc_log2;  // words per row per colour (power of two)
  int rows;         // ly * lz
  uint32_t words;   // rows * wc (words per colour per chain)
};

// geometry of a 2D/3D MSC lattice on the device (extents validated on the host)
__device__ __forceinline__ void msc_geom_device(int dim, int lx, int ly, int lz, MscGeom& g) {
  g.dim = dim;
  g.lx = lx;
  g.ly = ly;
  g.lz = dim == 3 ? lz : 1;
  g.wc = lx >> 6;
  g.wc_log2 = 31 - __clz(g.wc);
  g.rows = ly * g.lz;
  g.words = (uint32_t)g.rows * (uint32_t)g.wc;
}

enum MscRuleKind { RULE_METRO0 = 0, RULE_HB0 = 1, RULE_GEN = 2, RULE_GENSPIN = 3 };

constexpr int MSC_MAX_GROUPS = 16;

// Acceptance tables of up to MSC_MAX_GROUPS chain groups for one algorithm.
struct MscTables {
  uint32_t kind[MSC_MAX_GROUPS][CRITMC_NCLS];
  uint32_t thr[MSC_MAX_GROUPS][CRITMC_NCLS];
};

__device__ __forceinline__ uint32_t mux(uint32_t sel, uint32_t a, uint32_t b) {
  // sel ? a : b, lane by lane
  return lop3<(LA & LB) | (~LA & LC & 0xFF)>(sel, a, b);
}

// Neighbour words (other colour) of word k in row (y, z) of colour `col`.
template <int Z>
__device__ __forceinline__ void msc_neighbours(const uint32_t* __restrict__ other, const MscGeom& g,
                                               int col, int y, int z, int k, uint32_t* n) {
  const size_t r = (size_t)(y + g.ly * z) * g.wc;
  const uint32_t same = other[CRITMC_IDX(r + k, g.words)];
  const int p = (col + y + z) & 1;
  uint32_t sh;
  if (p == 0) {
    const int km = (k == 0) ? g.wc - 1 : k - 1;
    sh = __funnelshift_l(other[CRITMC_IDX(r + km, g.words)], same, 1);  // site index i-1 lives one bit lower
  } else {
    const int kp = (k == g.wc - 1) ? 0 : k + 1;
    sh = __funnelshift_r(same, other[CRITMC_IDX(r + kp, g.words)], 1);  // site index i+1 lives one bit higher
  }
  const int ym = (y == 0) ? g.ly - 1 : y - 1;
  const int yp = (y == g.ly - 1) ? 0 : y + 1;
  n[0] = same;
  n[1] = sh;
  n[2] = other[CRITMC_IDX((size_t)(ym + g.ly * z) * g.wc + k, g.words)];
  n[3] = other[CRITMC_IDX((size_t)(yp + g.ly * z) * g.wc + k, g.words)];
  if constexpr (Z == 6) {
    const int zm = (z == 0) ? g.lz - 1 : z - 1;
    const int zp = (z == g.lz - 1) ? 0 : z + 1;
    n[4] = other[CRITMC_IDX((size_t)(y + g.ly * zm) * g.wc + k, g.words)];
    n[5] = other[CRITMC_IDX((size_t)(y + g.ly * zp) * g.wc + k, g.words)];
  }
}

// Everything the plane loop needs about one word.
struct MscWord {
  uint32_t s;      // old spins
  Count3 anti;     // anti-aligned neighbour count (energy bookkeeping)
  Count3 cnt;      // class count (anti for Metropolis, up-neighbours for heat bath)
  uint32_t D, U;   // decided-1 lanes, undecided lanes
};

template <int Z, int RULE>
struct MscRule {
  const uint32_t* kind;  // uniform table of the chain's group
  const uint32_t* thr;

  __device__ __forceinline__ void classify(uint32_t s, const uint32_t* n, MscWord& w) const {
    uint32_t x[Z];
#pragma unroll
    for (int q = 0; q < Z; ++q) x[q] = s ^ n[q];
    w.s = s;
    w.anti = count_bits<Z>(x);
    if constexpr (RULE == RULE_HB0) {
      w.cnt = count_bits<Z>(n);
      w.D = 0;
      w.U = ~0u;
    } else if constexpr (RULE == RULE_METRO0) {
      w.cnt = w.anti;
      // always for count >= Z/2
      const uint32_t alw = (Z == 4) ? (w.cnt.b1 | w.cnt.b2)
                                    : (Z == 6) ? (w.cnt.b2 | (w.cnt.b1 & w.cnt.b0))
                                               : (w.cnt.b0 | w.cnt.b1);
      w.D = alw;
      w.U = ~alw;
    } else {
      w.cnt = w.anti;
      uint32_t D = 0, U = 0;
#pragma unroll
      for (int v = 0; v <= Z; ++v) {
        const uint32_t e = eq(w.cnt, v);
#pragma unroll
        for (int sb = 0; sb < 2; ++sb) {
          const int c = 2 * v + sb;
          const uint32_t m = (RULE == RULE_GENSPIN) ? (sb ? (e & s) : (e & ~s)) : e;
          if (RULE == RULE_GEN && sb) continue;
          if (kind[c] == CRITMC_KIND_ALWAYS) D |= m;
          else if (kind[c] == CRITMC_KIND_RANDOM) U |= m;
        }
      }
      w.D = D;
      w.U = U;
    }
  }

  __device__ __forceinline__ static uint32_t eq(const Count3& c, int v) {
    switch (v) {
      case 0: return count_eq<0>(c);
      case 1: return count_eq<1>(c);
      case 2: return count_eq<2>(c);
      case 3: return count_eq<3>(c);
      case 4: return count_eq<4>(c);
      case 5: return count_eq<5>(c);
      default: return count_eq<6>(c);
    }
  }

  // number of threshold classes the specialised rules read per plane
  static constexpr int NR = (RULE == RULE_METRO0) ? (Z / 2) : (RULE == RULE_HB0) ? (Z + 1) : 0;

  // broadcast threshold bits of the first 4*KG planes, computed once per thread
  template <int KG>
  __device__ __forceinline__ void prepare(uint32_t (&pre)[4 * KG][NR > 0 ? NR : 1]) const {
#pragma unroll
    for (int q = 0; q < 4 * KG; ++q)
#pragma unroll
      for (int v = 0; v < NR; ++v) pre[q][v] = bcast_bit(thr[2 * v], 31 - q);
  }

  // threshold bit plane from precomputed broadcasts (specialised rules)
  __device__ __forceinline__ uint32_t tbits_pre(const MscWord& w, const uint32_t* B) const {
    const Count3& c = w.cnt;
    if constexpr (RULE == RULE_METRO0) {
      const uint32_t lo = mux(c.b0, B[1], B[0]);
      if constexpr (Z == 6) return mux(c.b1, B[2], lo);
      return lo;
    } else {
      const uint32_t m10 = mux(c.b0, B[1], B[0]);
      if constexpr (Z == 2) return mux(c.b1, B[2], m10);
      const uint32_t m32 = mux(c.b0, B[3], B[2]);
      const uint32_t lo = mux(c.b1, m32, m10);
      if constexpr (Z == 4) return mux(c.b2, B[4], lo);
      const uint32_t m54 = mux(c.b0, B[5], B[4]);
      const uint32_t hi = mux(c.b1, B[6], m54);
      return mux(c.b2, hi, lo);
    }
  }

  // threshold bit plane of bit `bit` (31 = most significant) for the lanes of w
  __device__ __forceinline__ uint32_t tbits(const MscWord& w, int bit) const {
    const Count3& c = w.cnt;
    if constexpr (RULE == RULE_METRO0) {
      // only lanes with count < Z/2 are undecided
      const uint32_t lo = mux(c.b0, bcast_bit(thr[2], bit), bcast_bit(thr[0], bit));
      if constexpr (Z == 6) return mux(c.b1, bcast_bit(thr[4], bit), lo);
      return lo;
    } else if constexpr (RULE == RULE_HB0) {
      const uint32_t m10 = mux(c.b0, bcast_bit(thr[2], bit), bcast_bit(thr[0], bit));
      if constexpr (Z == 2) return mux(c.b1, bcast_bit(thr[4], bit), m10);
      const uint32_t m32 = mux(c.b0, bcast_bit(thr[6], bit), bcast_bit(thr[4], bit));
      const uint32_t lo = mux(c.b1, m32, m10);
      if constexpr (Z == 4) return mux(c.b2, bcast_bit(thr[8], bit), lo);
      const uint32_t m54 = mux(c.b0, bcast_bit(thr[10], bit), bcast_bit(thr[8], bit));
      const uint32_t hi = mux(c.b1, bcast_bit(thr[12], bit), m54);
      return mux(c.b2, hi, lo);
    } else {
      uint32_t t = 0;
#pragma unroll
      for (int v = 0; v <= Z; ++v) {
        const uint32_t e = eq(c, v);
#pragma unroll
        for (int sb = 0; sb < 2; ++sb) {
          const int cidx = 2 * v + sb;
          if (RULE == RULE_GEN && sb) continue;
          if (kind[cidx] != CRITMC_KIND_RANDOM) continue;
          const uint32_t m = (RULE == RULE_GENSPIN) ? (sb ? (e & w.s) : (e & ~w.s)) : e;
          t |= m & bcast_bit(thr[cidx], bit);
        }
      }
      return t;
    }
  }
};

// Compare planes 4 g .. 4 g + 3 (random bits r) for the undecided lanes of w.
template <int Z, int RULE>
__device__ __forceinline__ void msc_resolve(const MscRule<Z, RULE>& rule, MscWord& w, const critmc_u32x4& r,
                                            int grp, const uint32_t* pre) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t t;
    if constexpr (MscRule<Z, RULE>::NR > 0) {
      t = pre ? rule.tbits_pre(w, pre + q * MscRule<Z, RULE>::NR) : rule.tbits(w, 31 - (4 * grp + q));
    } else {
      t = rule.tbits(w, 31 - (4 * grp + q));
    }
    w.D |= w.U & t & ~r.v[q];
    w.U &= ~(r.v[q] ^ t);
  }
}

// Resolve plane group `grp` (planes 4 grp .. 4 grp + 3) for the undecided lanes.
// pre: broadcast threshold bits of these four planes (pre[q * NR + v]) or null.
// PR: Philox rounds of the planes (10; 7 only when a caller asks for it).
template <int Z, int RULE, int PR = CRITMC_PHILOX_ROUNDS>
__device__ __forceinline__ void msc_group(const MscRule<Z, RULE>& rule, MscWord& w, uint32_t k0,
                                          uint32_t k1, uint32_t widx, uint32_t sweep, uint32_t col,
                                          int grp, const uint32_t* pre = nullptr) {
  const critmc_u32x4 r = critmc_philox4x32_rounds(
      widx, sweep, CRITMC_TAG_PLANES | ((uint32_t)grp << 8) | (col << 16), 0u, k0, k1, PR);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t t;
    if constexpr (MscRule<Z, RULE>::NR > 0) {
      t = pre ? rule.tbits_pre(w, pre + q * MscRule<Z, RULE>::NR) : rule.tbits(w, 31 - (4 * grp + q));
    } else {
      t = rule.tbits(w, 31 - (4 * grp + q));
    }
    w.D |= w.U & t & ~r.v[q];
    w.U &= ~(r.v[q] ^ t);
  }
}

// Observable increments of the lanes in F (changed spins): the energy change
// of a flip is 2 z - 4 (anti-aligned neighbours before the flip).
template <int Z>
__device__ __forceinline__ void msc_obs(uint32_t F, uint32_t s_old, const Count3& anti, int& dE,
                                        int& dM, int& nacc) {
  const int f = __popc(F);
  const int na = __popc(F & anti.b0) + 2 * __popc(F & anti.b1) + 4 * __popc(F & anti.b2);
  dE += 2 * Z * f - 4 * na;
  dM -= 2 * (2 * __popc(F & s_old) - f);
  nacc += f;
}

}  // namespace critmc
