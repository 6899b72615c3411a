/*
 * A C restatement of critmc's CPU Ising sweeps -- TEST INFRASTRUCTURE and the
 * CPU baseline of the benchmark, never part of the GPU product.
 *
 * It follows critmc's numba kernels line by line, with critmc's own random
 * stream, so that the CPU baseline measures the reference's algorithm (a
 * typewriter sweep over an int64 neighbour table, float64 acceptance tables,
 * one uniform per site only when it is needed) rather than the GPU stream's
 * bit-plane replay:
 *   metropolis_table, metropolis_sweep   src/critmc/kernels/ising.py:48-57, :69-87
 *   heatbath_table, heatbath_sweep       src/critmc/kernels/ising.py:60-65, :91-107
 *   run (metropolis and heatbath rows)   src/critmc/kernels/ising.py:174-237
 * Random numbers: the PCG64DXSM generator (O'Neill's permuted congruential
 * generator, 128-bit state, cheap multiplier 0xda942042e4dd58b5, "double
 * xorshift multiply" output of the state before each advance), as numpy's
 * Generator(PCG64DXSM) draws them; random() = (next64 >> 11) * 2^-53.  Given
 * the Generator's state at the call, the spins and series equal critmc's bit
 * for bit (pinned in tests against fixtures that critmc itself wrote).
 */
#include <math.h>
#include <stdint.h>

typedef unsigned __int128 u128;

#define PCG_CHEAP_MUL 0xda942042e4dd58b5ULL

typedef struct {
  u128 state, inc;
} Pcg;

static inline uint64_t pcg_next(Pcg* g) {
  const u128 old = g->state;
  g->state = old * (u128)PCG_CHEAP_MUL + g->inc;
  uint64_t hi = (uint64_t)(old >> 64);
  const uint64_t lo = (uint64_t)old | 1u;
  hi ^= hi >> 32;
  hi *= PCG_CHEAP_MUL;
  hi ^= hi >> 48;
  hi *= lo;
  return hi;
}

static inline double pcg_random(Pcg* g) { return (double)(pcg_next(g) >> 11) * (1.0 / 9007199254740992.0); }

/* words: state hi, state lo, inc hi, inc lo */
static void pcg_load(Pcg* g, const uint64_t w[4]) {
  g->state = ((u128)w[0] << 64) | w[1];
  g->inc = ((u128)w[2] << 64) | w[3];
}

static void pcg_store(const Pcg* g, uint64_t w[4]) {
  w[0] = (uint64_t)(g->state >> 64);
  w[1] = (uint64_t)g->state;
  w[2] = (uint64_t)(g->inc >> 64);
  w[3] = (uint64_t)g->inc;
}

/* the first n raw 64-bit outputs from a state (for the generator's pin) */
void critmc_port_pcg_raw(uint64_t w[4], int64_t n, uint64_t* out) {
  Pcg g;
  pcg_load(&g, w);
  for (int64_t i = 0; i < n; ++i) out[i] = pcg_next(&g);
  pcg_store(&g, w);
}

int critmc_port_ising_run(int8_t* s, const int64_t* nbr, int64_t n, int z, double beta, double h, uint64_t pcg[4],
                          const int64_t* schedule, int n_rows, int n_meas, int64_t* running, int64_t* e_out,
                          int64_t* m_out, int64_t* aux_out) {
  if (z < 1 || z > 16) return -1;
  double table[33][2], p_up[33];
  for (int a = -z; a <= z; ++a) {
    for (int t = 0; t < 2; ++t) {
      const double spin = 2.0 * t - 1.0;
      const double d_e = 2.0 * a + 2.0 * h * spin;
      table[a + z][t] = d_e <= 0.0 ? 1.0 : exp(-beta * d_e);
    }
    p_up[a + z] = 1.0 / (1.0 + exp(-2.0 * beta * (a + h)));
  }
  Pcg g;
  pcg_load(&g, pcg);
  int64_t e_b = running[0], m = running[1];
  for (int meas = 0; meas < n_meas; ++meas) {
    int64_t accepted = 0;
    for (int row = 0; row < n_rows; ++row) {
      const int64_t code = schedule[2 * row];
      if (code != 0 && code != 2) return -2; /* metropolis and heatbath rows only */
      for (int64_t rep = 0; rep < schedule[2 * row + 1]; ++rep) {
        for (int64_t i = 0; i < n; ++i) {
          const int64_t* nb = nbr + i * z;
          int field = 0;
          for (int k = 0; k < z; ++k) field += s[nb[k]];
          const int si = s[i];
          if (code == 0) {
            const int a = si * field;
            const double p = table[a + z][(si + 1) >> 1];
            if (p >= 1.0 || pcg_random(&g) < p) {
              s[i] = (int8_t)(-si);
              e_b += 2 * a;
              m -= 2 * si;
              ++accepted;
            }
          } else {
            const int nw = pcg_random(&g) < p_up[field + z] ? 1 : -1;
            if (nw != si) {
              e_b += 2 * si * field;
              m += 2 * nw;
              s[i] = (int8_t)nw;
              ++accepted;
            }
          }
        }
      }
    }
    e_out[meas] = e_b;
    m_out[meas] = m;
    aux_out[4 * meas + 0] = accepted;
    aux_out[4 * meas + 1] = 0;
    aux_out[4 * meas + 2] = 0;
    aux_out[4 * meas + 3] = 0;
  }
  running[0] = e_b;
  running[1] = m;
  pcg_store(&g, pcg);
  return 0;
}
