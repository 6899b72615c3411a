/*
 * critmc_b200: C ABI of the B200 sampling kernels.
 *
 * Every entry point takes plain pointers and sizes, returns an int32 status
 * (0 = ok, < 0 = error; text via critmc_last_error) and runs asynchronously
 * on the caller's CUDA stream (passed as void*, NULL = legacy default stream).
 * Device buffers are allocated by the caller (the Python layer uses torch
 * tensors); the library allocates nothing except CUDA graph objects.
 *
 * The entry points replace the numba `run` kernels of critmc, which execute an
 * update schedule n_meas times and record the observables after each
 * application.  Update codes are critmc's (src/critmc/kernels/common.py:16-21).
 */
#ifndef CRITMC_B200_H
#define CRITMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define CRITMC_OK 0
#define CRITMC_ERR_INVALID (-1)     /* bad argument (checked before any launch) */
#define CRITMC_ERR_CUDA (-2)        /* CUDA runtime error */
#define CRITMC_ERR_UNSUPPORTED (-3) /* geometry/update not handled by this kernel */
#define CRITMC_ERR_TIMEOUT (-4)     /* a bounded device wait ran out */
#define CRITMC_ERR_CANCELLED (-5)   /* host cancel word was set */
#define CRITMC_ERR_DEVICE (-6)      /* a kernel flagged an internal inconsistency */

/* ---- update codes (critmc kernels/common.py:16-21) --------------------- */
#define CRITMC_METROPOLIS 0
#define CRITMC_METROPOLIS_RANDOM 1
#define CRITMC_HEATBATH 2
#define CRITMC_WOLFF 3
#define CRITMC_SWENDSEN_WANG 4
#define CRITMC_OVERRELAX 5

/* ---- aux columns (critmc kernels/common.py:36-40) ---------------------- */
#define CRITMC_N_AUX 4

/* ---- acceptance classes ---------------------------------------------------
 * Binary-spin kernels classify each site by a neighbour count v (0..z) and
 * its own spin bit sb (1 = spin +1).  Class index c = 2*v + sb.  A class is
 * NEVER (decision 0), ALWAYS (decision 1) or RANDOM: decision = (u < thr)
 * with u a uniform 32-bit integer.  For Metropolis v counts anti-aligned
 * neighbours and the decision flips the spin; for heat bath v counts
 * neighbours equal to +1 and the decision is the new spin (1 = +1).        */
#define CRITMC_NCLS 16
#define CRITMC_KIND_NEVER 0u
#define CRITMC_KIND_ALWAYS 1u
#define CRITMC_KIND_RANDOM 2u

/* library version (major*10000 + minor*100 + patch) */
int32_t critmc_version(void);

/* Bounds-checked builds (compiled with -DCRITMC_CHECK, e.g. python -m
 * critmc_b200._build --check): the hot kernels compare their lattice indices
 * with the array extents, record the first bad index of every source file and
 * access element 0 instead, without trapping.  Returns the number of bad
 * indices seen since the last call (and clears the records), with one
 * "file:line index i of n" entry per file in buf; -1 in a release build.
 * No counterpart in critmc (numba's boundscheck option plays this role).   */
int64_t critmc_check_report(char* buf, int32_t size);

/* copy the last error message of the calling thread (always NUL-terminated) */
int32_t critmc_last_error(char* buf, int32_t size);

/* Acceptance table of a binary-spin kernel: kind[16], thr[16].
 * Metropolis: p = min(1, exp(-beta*(2a + 2h s))), a = s*sum_j s_j
 *   (critmc kernels/ising.py:48-57 metropolis_table).
 * Heat bath: p_up = 1/(1 + exp(-2 beta (sum_j s_j + h)))
 *   (critmc kernels/ising.py:60-65 heatbath_table).
 * thr = round(p * 2^32); p >= 1 or thr == 2^32 gives ALWAYS, thr == 0 NEVER.
 * Returns 1 in *spin_dependent when the classes depend on the own spin.   */
int32_t critmc_ising_class_table(int32_t algo, int32_t z, double beta, double h, uint32_t* kind,
                                 uint32_t* thr, int32_t* spin_dependent);

/* ---- multi-spin-coded Ising (2D square / 3D cubic, periodic) -------------
 * Layout of one chain: spins[colour][row][word], colour = (x+y+z)&1,
 * row = y + ly*z, word k bit j holds the colour's site x = 2*(32k+j) + p with
 * p = (colour + y + z) & 1; bit value 1 = spin +1.  lx must be a multiple of
 * 64 with lx/64 a power of two; ly, lz even.  Chains are contiguous:
 * chain c starts at spins + c * 2 * rows * (lx/64).
 *
 * Replaces critmc kernels/ising.py:174-237 `run` (Metropolis and heat-bath
 * rows of the schedule) with checkerboard sweeps.  Chains come in n_groups
 * equal groups of consecutive chains (n_groups <= 16) sharing one acceptance
 * table (one beta, h): tables is a HOST array [n_groups][2][2][16]
 * (metropolis kind, thr, then heat-bath kind, thr; see
 * critmc_ising_class_table).  keys is a HOST array [n_chains][2] of Philox
 * keys.  Device inputs: running[n_chains][2] (E_b, M, updated in place).  Device outputs:
 * e_out/m_out[n_chains][n_meas], aux_out[n_chains][n_meas][4].  scratch must
 * hold critmc_ising_msc_scratch_bytes(n_chains, n_meas) bytes of device
 * memory.  schedule is a HOST array of n_rows (code, reps) pairs; sweep k of
 * the call uses sweep index sweep0 + k of every chain.
 * mode: 0 auto, 1 one launch per half-sweep, 3 = 1 replayed as CUDA graphs;
 * plus, in bits 8..11, v = 1..6 for 2^(v-1) rows walked per thread (0 =
 * automatic).  Both are tuning knobs (critmc_b200.autotune picks them).
 * Bit 12 (CRITMC_MSC_PHILOX7) is not a tuning knob: it draws the acceptance
 * planes from Philox4x32-7 instead of Philox4x32-10 (same counters), a
 * different random stream that the CPU oracle replays with rounds = 7.  Off by
 * default; 7 rounds is the smallest count Salmon et al. (SC'11) report as
 * passing BigCrush.
 * k_inline: 4 or 8 acceptance planes resolved inline (tuning only; the
 * results do not depend on it).                                            */
#define CRITMC_MSC_PHILOX7 0x1000
#define CRITMC_MSC_BATCH_MAX 16
int64_t critmc_ising_msc_scratch_bytes(int32_t n_chains, int32_t n_meas);
int32_t critmc_ising_msc_run(uint32_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                             int32_t n_chains, const uint32_t* keys, const uint32_t* tables,
                             int32_t n_groups, uint32_t sweep0, const int64_t* schedule,
                             int32_t n_rows, int32_t n_meas, int64_t* running, int64_t* e_out,
                             int64_t* m_out, int64_t* aux_out, void* scratch, int32_t mode,
                             int32_t k_inline, void* stream);

/* critmc_ising_msc_run for up to CRITMC_MSC_BATCH_MAX separately allocated
 * chains of one lattice shape in one call (one launch per half-sweep covers
 * them all): each chain brings its own lattice, running sums, series outputs
 * (all DEVICE), Philox key, first sweep and acceptance table (an index into
 * the HOST tables [n_tables][2][2][16] of critmc_ising_msc_run).  The results
 * of a chain equal critmc_ising_msc_run's for it alone.  scratch: DEVICE,
 * critmc_ising_msc_batch_scratch_bytes(n_chains, n_meas) bytes; the call
 * copies the sweep bases into it.  mode as critmc_ising_msc_run's (no Philox
 * option; 8 inline planes).  No counterpart in critmc (one chain per
 * process); the serving loop batches its large lattices with it.          */
typedef struct {
  uint32_t* spins;
  int64_t* running;  /* [2]: E_b, M */
  int64_t* e_out;    /* [n_meas] */
  int64_t* m_out;    /* [n_meas] */
  int64_t* aux_out;  /* [n_meas][4] */
  uint32_t key[2];
  uint32_t sweep0;
  int32_t table;
} critmc_msc_chain;
int64_t critmc_ising_msc_batch_scratch_bytes(int32_t n_chains, int32_t n_meas);
int32_t critmc_ising_msc_run_batch(const critmc_msc_chain* chains, int32_t n_chains, int32_t dim, int32_t lx,
                                   int32_t ly, int32_t lz, const uint32_t* tables, int32_t n_tables,
                                   const int64_t* schedule, int32_t n_rows, int32_t n_meas, void* scratch,
                                   int32_t mode, void* stream);

/* Initial configurations of MSC chains, drawn on the device: start 0 = random
 * (word w of colour c is word 0 of Philox(w, 0, 0x05 | c << 16, 0) with the
 * chain's key), 1 = all up, -1 = all down.  keys: DEVICE [n_chains][2].
 * critmc models.py:113-121 draws the same hot/cold starts on the host.    */
int32_t critmc_ising_msc_init(uint32_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                              int32_t n_chains, const uint32_t* keys, int32_t start, void* stream);

/* ---- byte lattices (int8 Ising, q-state Potts) -----------------------------
 * Layout of one chain: elem[colour][row][i] (int8), row = y + ly*z, slot i
 * of the colour's row holds site x = 2i + p, p = (colour + y + z) & 1.  All
 * extents must be even (dim 1..3).  One thread block advances one chain
 * through the whole schedule; the lattice is staged in shared memory when it
 * fits (lx*ly*lz bytes <= 160 KiB) and updated in HBM otherwise.
 * keys: HOST [n_chains][2].  Chains form n_groups equal groups of
 * consecutive chains sharing one acceptance table / beta.
 * Each site draws Philox4x32-10(c0 = slot (row*lx/2 + i), c1 = sweep,
 * c2 = 0x02 | colour << 16, c3 = 0) once per sweep.                        */

/* Ising with int8 spins (+1/-1), same class tables and outputs as
 * critmc_ising_msc_run; replaces critmc kernels/ising.py:174-237.         */
int32_t critmc_ising_byte_run(int8_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                              int32_t n_chains, const uint32_t* keys, const uint32_t* tables,
                              int32_t n_groups, uint32_t sweep0, const int64_t* schedule,
                              int32_t n_rows, int32_t n_meas, int64_t* running, int64_t* e_out,
                              int64_t* m_out, int64_t* aux_out, void* stream);

/* q-state Potts (2 <= q <= 127), states 0..q-1 in int8.  betas: HOST
 * [n_groups].  Device in/out: energy[n_chains] (E = -#satisfied bonds),
 * counts[n_chains][q].  Device outputs: e_out[n_chains][n_meas],
 * counts_out[n_chains][n_meas][q], aux_out[n_chains][n_meas][4].
 * Replaces critmc kernels/potts.py:171-235 (`run`), :45-71 (Metropolis with
 * a uniformly proposed different state, boltz[d] = exp(-beta d)) and :75-103
 * (heat bath, weight[n] = exp(beta n)).                                    */
int32_t critmc_potts_run(int8_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz, int32_t q,
                         int32_t n_chains, const uint32_t* keys, const double* betas,
                         int32_t n_groups, uint32_t sweep0, const int64_t* schedule,
                         int32_t n_rows, int32_t n_meas, int64_t* energy, int64_t* counts,
                         int64_t* e_out, int64_t* counts_out, int64_t* aux_out, void* stream);

/* Potts acceptance tables for one beta: boltz_thr[8] (accept iff u < thr for
 * a uniform 32-bit u; thr = round(2^32 exp(-beta d)), 2^32 = always, for
 * d = 0..7) and hb_weight[8] (uint64 weights round(2^52 exp(beta n - max)),
 * n = 0..7; the heat bath picks state k with probability proportional to
 * hb_weight[#neighbours in state k]).                                       */
int32_t critmc_potts_tables(int32_t z, double beta, uint64_t* boltz_thr, uint64_t* hb_weight);

/* ---- O(n) vector models (n = 2 XY, n = 3 Heisenberg), FP32 spins ------------
 * Layout of one chain: comp[n][colour][row][i] (float32, structure of
 * arrays, same colour-major site order as the byte lattices).  Even extents,
 * dim 1..3.  One block per chain; the lattice is staged in shared memory when
 * n * lx*ly*lz * 4 bytes <= 200 KiB.  betas, steps: HOST [n_groups]
 * (inverse temperature and Metropolis step size of each group).
 * Random words of a site per sweep: Philox(slot, sweep, 0x02 | colour << 16, 0)
 * and, for rejection steps and extra Gaussians, Philox(slot, sweep,
 * 0x03 | colour << 16, k).
 * Schedule rows: metropolis (0), heatbath (2), overrelax (5).
 * After each schedule application every spin is renormalised and the
 * observables are summed exactly: each site's FP64 term is rounded to a
 * multiple of 2^-36 and the terms are added as int64 (independent of the
 * thread layout), then returned as doubles:
 * e_out[n_chains][n_meas] = -sum_<ij> S_i.S_j, m_out[..][n],
 * stiff_c_out / stiff_s_out[..][dim] (per-axis sums of S_i^0 S_j^0 + S_i^1 S_j^1
 * and S_i^0 S_j^1 - S_i^1 S_j^0 over bonds i -> i + e_a), aux_out[..][4]
 * (accepted Metropolis moves in column 0).
 * Replaces critmc kernels/on.py:349-418 (`run`), :113-137 (metropolis_sweep),
 * :141-183 (overrelax_sweep), :187-261 (von Mises / heat bath),
 * :36-87 (energy, magnetization, stiffness_sums, normalize).             */
int32_t critmc_on_run(float* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz, int32_t n,
                      int32_t n_chains, const uint32_t* keys, const double* betas,
                      const double* steps, int32_t n_groups, uint32_t sweep0,
                      const int64_t* schedule, int32_t n_rows, int32_t n_meas, double* e_out,
                      double* m_out, double* stiff_c_out, double* stiff_s_out, int64_t* aux_out,
                      void* stream);

/* The same run with many thread blocks per chain (one launch per colour of a
 * sweep, a normalisation and a measurement launch per measurement, replayed
 * as CUDA graphs): lower latency for large lattices, results identical to
 * critmc_on_run (spins and sums bit for bit).  scratch: device memory of
 * critmc_on_grid_scratch_bytes(n_chains, n_meas, n, dim) bytes.
 * blocks_per_chain: blocks of 256 threads per chain and colour, 0 = auto.
 * No counterpart in critmc (one process per chain).                        */
int64_t critmc_on_grid_scratch_bytes(int32_t n_chains, int32_t n_meas, int32_t n, int32_t dim);
int32_t critmc_on_run_grid(float* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz, int32_t n,
                           int32_t n_chains, const uint32_t* keys, const double* betas,
                           const double* steps, int32_t n_groups, uint32_t sweep0,
                           const int64_t* schedule, int32_t n_rows, int32_t n_meas, double* e_out,
                           double* m_out, double* stiff_c_out, double* stiff_s_out, int64_t* aux_out,
                           void* scratch, int32_t blocks_per_chain, void* stream);

/* ---- Edwards-Anderson +-J spin glass with parallel tempering ---------------
 * A sample holds two independent replica sets of m <= 32 configurations on a
 * periodic lattice (dim 2 or 3, even extents, at most 4096 sites).  Device
 * layout (replica multi-spin coding): words[sample][set][colour][slot]
 * (uint32, colour-major slots as for the byte lattices), bit k = spin (1 = +1)
 * of the configuration currently at temperature index k; temperatures are
 * ordered hot -> cold (critmc glass.py:140).  conf_at[sample][set][m] (uint8)
 * names the configuration at each temperature (critmc's perm), labels
 * [sample][set][m] (uint8) the last visited end (0, 1 hot, 2 cold).
 * jneg[sample][colour][slot] (uint8): bit q set if the coupling of the bond to
 * neighbour q is -1, neighbours in the order (x-side, other x-side, y-1, y+1,
 * z-1, z+1) of the colour-major layout (critmc_ea_coupling_bits builds it).
 *
 * One call runs n_steps PT steps (critmc kernels/glass.py:81-163 `pt_run`):
 * sweeps_per_step checkerboard Metropolis sweeps of every configuration at
 * its temperature, then for each set swaps of neighbouring temperatures
 * k = 0..m-2 in order (accept x >= 0 or u < exp(x), x = (b_k - b_k+1)
 * (E_k - E_k+1)), round-trip labels, and the measurement of e, q_l, |q|, q^2,
 * q^4, |q(k_min)|^2 per temperature into acc[sample][bin][m][7] (double;
 * step t0+t goes to bin floor(log2(t+1)) of this call).  Counters (device,
 * accumulated): swap_acc/swap_try[sample][m-1], label_hist[sample][m][2],
 * trips[sample][2] (int64).  betas: HOST [m].  keys: HOST [n_samples][2][2]
 * (one Philox key per replica set).  swap_thr: DEVICE table from
 * critmc_pt_swap_table.  Site draws use the MSC plane stream of
 * critmc_ising_msc_run with counter word c0 = slot and sweep index
 * (t0 + t) * sweeps_per_step + s; swap k of set r at step t draws word 0 of
 * Philox(k, t0 + t, 0x04 | r << 16, 0).                                      */
int32_t critmc_pt_swap_table(int32_t m, const double* betas, int32_t width, uint32_t* out);
int32_t critmc_ea_coupling_bits(int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                                const double* couplings, uint8_t* jneg);
int32_t critmc_ea_pt_run(uint32_t* words, const uint8_t* jneg, int32_t dim, int32_t lx, int32_t ly,
                         int32_t lz, int32_t m, int32_t n_samples, const uint32_t* keys,
                         const double* betas, const uint32_t* swap_thr, int32_t swap_width,
                         uint8_t* conf_at, uint8_t* labels, uint32_t t0, int32_t n_steps,
                         int32_t n_bins, int32_t sweeps_per_step, double* acc, int64_t* swap_acc,
                         int64_t* swap_try, int64_t* label_hist, int64_t* trips, void* stream);

/* A campaign of several lattice sizes (same dim and temperatures) in ONE
 * persistent launch: thread blocks take (size, sample) items from a queue,
 * largest lattices first, and run critmc_ea_pt_run's steps on each; results
 * equal critmc_ea_pt_run per size.  sizes: HOST array; their keys are DEVICE
 * arrays [n_samples][2][2].  buffer: device memory of
 * critmc_ea_campaign_buffer_bytes(n_sizes, total samples) bytes; staging:
 * NULL or pinned host memory of the same size (the call fills it and copies
 * from it asynchronously).  No counterpart in critmc (one process per
 * sample, src/critmc/runner.py:154-223).                                     */
typedef struct {
  uint32_t* words;
  const uint8_t* jneg;
  const uint32_t* keys;
  uint8_t* conf_at;
  uint8_t* labels;
  double* acc;
  int64_t* swap_acc;
  int64_t* swap_try;
  int64_t* label_hist;
  int64_t* trips;
  int32_t lx, ly, lz, n_samples;
} critmc_ea_size;
int64_t critmc_ea_campaign_buffer_bytes(int32_t n_sizes, int64_t total_samples);
int32_t critmc_ea_campaign_run(const critmc_ea_size* sizes, int32_t n_sizes, int32_t dim, int32_t m,
                               const double* betas, const uint32_t* swap_thr, int32_t swap_width,
                               uint32_t t0, int32_t n_steps, int32_t n_bins, int32_t sweeps_per_step,
                               void* buffer, int64_t buffer_bytes, void* staging, void* stream);

/* ---- bounded runs of the persistent kernels ----------------------------------
 * A critmc_control is a page of pinned host memory mapped into the device: a
 * cancel word the host sets and a status word the kernels set.  The _ctl
 * variants of the persistent entry points take one (NULL = unbounded, the
 * plain entry points).  One thread of every block polls between steps (EA) or
 * measurements (items): its block's elapsed time (globaltimer) against the
 * budget at every poll, the host-mapped words at most every 100 us.  A block
 * over budget writes CRITMC_ERR_TIMEOUT, a block that sees the cancel word
 * writes CRITMC_ERR_CANCELLED (the first reason stays); every block then
 * leaves its work at its next poll, so the kernel returns on its own and the
 * device stays usable.  The outputs and device state of a run that stopped
 * are incomplete (samples or items part-way): restore the state saved before
 * the call.  No counterpart in critmc (its kernels run to completion).
 * create/destroy: allocate / free the page (not while a run uses it).
 * arm: clear both words and set the budget in ns (0 = none) for the next
 *   runs; only while no run using it is in flight.
 * cancel: set the cancel word (any host thread, while runs are in flight).
 * status: the status word now (0 while nothing stopped).
 * wait: synchronise `stream`, then return the status word as the status
 *   (CRITMC_OK, CRITMC_ERR_TIMEOUT or CRITMC_ERR_CANCELLED).               */
typedef struct critmc_control critmc_control;
int32_t critmc_control_create(critmc_control** ctl);
int32_t critmc_control_destroy(critmc_control* ctl);
int32_t critmc_control_arm(critmc_control* ctl, int64_t budget_ns);
int32_t critmc_control_cancel(critmc_control* ctl);
int32_t critmc_control_status(const critmc_control* ctl);
int32_t critmc_control_wait(const critmc_control* ctl, void* stream);

/* critmc_ea_campaign_run under a control (the step loop of every sample polls it). */
int32_t critmc_ea_campaign_run_ctl(const critmc_ea_size* sizes, int32_t n_sizes, int32_t dim, int32_t m,
                                   const double* betas, const uint32_t* swap_thr, int32_t swap_width,
                                   uint32_t t0, int32_t n_steps, int32_t n_bins, int32_t sweeps_per_step,
                                   void* buffer, int64_t buffer_bytes, void* staging, critmc_control* ctl,
                                   void* stream);

/* ---- heterogeneous work items (continuous batching, serving) --------------
 * One item advances one chain by n_meas schedule applications: any model and
 * lattice size, its own beta, key and sweep counter.  critmc_run_items runs
 * a persistent kernel per model family (multi-spin-coded Ising resident in
 * shared memory, byte lattices, O(n)) whose thread blocks pull items from a
 * queue until it is empty, so chains of different sizes and lengths share the
 * GPU.  Random streams are those of the per-model entry points (an item gives
 * the same results as critmc_ising_msc_run / critmc_ising_byte_run /
 * critmc_potts_run / critmc_on_run for the same chain), so a chain's result
 * does not depend on what it is batched with.  No counterpart in critmc, which
 * runs one chain per process (src/critmc/runner.py:154-223).                 */
#define CRITMC_ITEM_MSC_ISING 0 /* spins: uint32 MSC words (2D/3D, lx/64 power of two, <= 1024^2) */
#define CRITMC_ITEM_BYTE_ISING 1 /* spins: int8 colour-major */
#define CRITMC_ITEM_POTTS 2     /* spins: int8 colour-major, q_or_n = q */
#define CRITMC_ITEM_ON 3        /* spins: float32 [n][colour][slot], q_or_n = n */

typedef struct {
  void* spins;       /* device: the chain's lattice, advanced in place */
  int64_t* running;  /* device: Ising (E_b, M); Potts E; unused for O(n) */
  int64_t* counts;   /* device: Potts counts[q] in/out */
  void* e_out;       /* device: [n_meas], int64 (Ising, Potts) or double (O(n)) */
  void* vec_out;     /* device: Ising M [n_meas] int64; Potts counts [n_meas][q] int64;
                        O(n) M [n_meas][n] double */
  double* sc_out;    /* device: O(n) stiffness sums [n_meas][dim] */
  double* ss_out;
  int64_t* aux_out;  /* device: [n_meas][4] */
  int32_t kind;      /* CRITMC_ITEM_* */
  int32_t dim, lx, ly, lz, q_or_n;
  uint32_t key[2];
  uint32_t sweep0;
  int32_t n_meas;
  int32_t n_rows;
  int32_t codes[4], reps[4];
  int32_t rule[2];   /* filled by critmc_item_prepare */
  float beta, step;  /* O(n) */
  uint32_t kind_tab[2][16], thr_tab[2][16]; /* Ising acceptance classes (metropolis, heat bath) */
  uint64_t boltz[8], weight[8];             /* Potts tables */
  int32_t team;      /* thread blocks per item: 0 or 1 = one block (lattice in shared
                        memory when it fits); 2, 4, 8 or 16 = a thread-block cluster of
                        that many blocks on one GPC, the lattice in global memory (large
                        lattices: about team times less time per sweep) */
  int32_t reserved;  /* 0 */
} critmc_item;

/* Fill the acceptance tables of an item for inverse temperature beta (and
 * field h for Ising) and check its geometry and schedule.                   */
int32_t critmc_item_prepare(critmc_item* item, double beta, double h, double step);

/* Teams of `team` blocks (2, 4, 8 or 16) of the item kernel for items of
 * `kind` (and q_or_n, dim for O(n)) that the current GPU runs at once: 0 if it
 * cannot schedule clusters of that size (critmc_run_items would then refuse
 * such items with CRITMC_ERR_UNSUPPORTED), a negative status on error.      */
int32_t critmc_items_team_clusters(int32_t kind, int32_t q_or_n, int32_t dim, int32_t team);

/* Device bytes needed to run n_items items (descriptors + queue counters).  */
int64_t critmc_items_buffer_bytes(int32_t n_items);

/* Copy the HOST items to the DEVICE buffer (grouped by family and team size)
 * and run them; the kernels of the groups run side by side on library-owned
 * streams forked from and joined into `stream` (CUDA-graph capturable).  A
 * team size the GPU cannot schedule fails with CRITMC_ERR_UNSUPPORTED.
 * staging: NULL, or PINNED host memory of n_items * sizeof(critmc_item)
 *   bytes that the call fills and copies from asynchronously (do not reuse it
 *   before `stream` has passed this call).  With NULL the copy comes from
 *   pageable memory and may wait for `stream`.
 * smem_limit: dynamic shared memory per block allowed for byte/O(n) lattices
 * (larger lattices are updated in HBM); 0 picks 200 KiB.                    */
int32_t critmc_run_items(const critmc_item* items, int32_t n_items, void* buffer,
                         int64_t buffer_bytes, void* staging, int32_t smem_limit, void* stream);

/* critmc_run_items under a control (see critmc_control): every block polls it
 * before it takes an item and between the measurements of its item.        */
int32_t critmc_run_items_ctl(const critmc_item* items, int32_t n_items, void* buffer,
                             int64_t buffer_bytes, void* staging, int32_t smem_limit, critmc_control* ctl,
                             void* stream);

/* ---- cluster updates (Swendsen-Wang, Wolff) ----------------------------------
 * One cluster update of n_chains Ising or Potts chains.  bits: 1 for the
 * multi-spin-coded Ising words, 0 for int8 spins (Ising +-1, Potts 0..q-1).
 * q: 0 for Ising, else the Potts q.  keys: HOST [n_chains][2].  algo:
 * CRITMC_WOLFF or CRITMC_SWENDSEN_WANG.  Sites are numbered by their
 * colour-major layout index u; bond (colour-0 site s, direction q) is active
 * when both ends agree and word q%4 of Philox(s, sweep, 0x07 | (q/4)<<8, 0)
 * < round(p 2^32), p = 1 - e^{-2 beta} (Ising), 1 - e^{-beta} (Potts).  The
 * root of a cluster is its smallest u.  SW: root r draws word 0 of
 * Philox(r, sweep, 0x08, 0) (Ising: flip if >= 2^31; Potts: state
 * (w q) >> 32).  Wolff: seed (w0 N) >> 32 from Philox(0, sweep, 0x09, 0),
 * Potts new state (old + 1 + ((w1 (q-1)) >> 32)) mod q.
 * Device in/out: running (Ising [n][2] E_b, M; Potts energy [n]), counts
 * (Potts [n][q]), stats [n][3] (+= Wolff cluster size; SW sum |C|^2 and
 * cluster count of this decomposition).  scratch:
 * critmc_cluster_scratch_bytes(n_chains, sites per chain) bytes.
 * Replaces critmc kernels/ising.py:111-171, kernels/potts.py:107-168.       */
int64_t critmc_cluster_scratch_bytes(int32_t n_chains, int64_t n_sites);
int32_t critmc_cluster_update(int32_t bits, void* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz,
                              int32_t q, int32_t n_chains, const uint32_t* keys, double beta,
                              int32_t algo, uint32_t sweep, int64_t* running, int64_t* counts,
                              int64_t* stats, void* scratch, void* stream);

/* One Wolff (algo 3) or Swendsen-Wang (4) update of n_chains O(n) chains
 * (n = 2, 3) on the embedded Ising model of a random axis r: spins DEVICE
 * float [n_chains][n][N] in the colour-major layout of critmc_on_run.  r from
 * Philox(0, sweep, 0x0B, 0) (XY: angle 2 pi u0; n = 3: z = 2 u0 - 1, angle
 * 2 pi u1), p_i = S_i . r, bond (as in critmc_cluster_update) active when
 * p_i p_j > 0 and its 24-bit uniform < 1 - exp(-2 beta p_i p_j); flipped
 * clusters are reflected, S <- S - 2 p r.  Spins are not renormalised (the
 * next critmc_on_run measurement does it).  stats and scratch as above.
 * Replaces critmc kernels/on.py:265-345 (wolff_update, sw_update).          */
int32_t critmc_on_cluster_update(float* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz, int32_t n,
                                 int32_t n_chains, const uint32_t* keys, double beta, int32_t algo,
                                 uint32_t sweep, int64_t* stats, void* scratch, void* stream);

/* ---- streaming Gamma-method sums ---------------------------------------------
 * Append n values per chain (values: DEVICE [n_chains][ld], int64 or double)
 * to the per-chain state (DEVICE, critmc_stream_state_bytes(n_chains,
 * max_lag) bytes, zeroed before the first update): count, shift (first value),
 * sum and sum of squares of value - shift, lag sums S_t (t = 1..max_lag), first
 * and last max_lag values.  Gamma(t) for t <= max_lag follows exactly, as
 * critmc's gamma_method gets it from the full series
 * (src/critmc/stats/autocorr.py:381).                                         */
int64_t critmc_stream_state_bytes(int32_t n_chains, int32_t max_lag);
int32_t critmc_stream_update(const void* values, int32_t is_double, int32_t n_chains, int32_t n, int64_t ld,
                             double* state, int32_t max_lag, void* stream);

/* ---- flat-histogram walks (Wang-Landau, multicanonical) ----------------------
 * n_walkers independent walkers of one zero-field Ising (q = 0) or Potts
 * (q = 2..127) lattice, one thread each.  Levels: Ising idx = (E_b + B)/4,
 * Potts idx = E + B (B bonds), `levels` of them.  Move t of a walker uses
 * Philox(t mod 2^32, t / 2^32, 0x0A, 0) under its key: word 0 the site
 * ((w0 N) >> 32), word 1 the Potts proposal ((w1 (q-1)) >> 32, skipping the old
 * state), words 2, 3 the 53-bit uniform u; accepted if ln w(new) >= ln w(old) or
 * ln u < ln w(new) - ln w(old) (critmc's u < exp(ln w(new) - ln w(old))); a
 * move leaving [window[0], window[1]] is rejected.  All arrays are DEVICE arrays, per walker: spins [N] (critmc site
 * order), keys [2], idx (level), order (Ising M; Potts counts [q]), lng
 * [levels] (mode 0 Wang-Landau: ln g, incremented by ln f each move; mode 1
 * multicanonical: the weights ln w, read only), hist [levels] (+1 per move),
 * window [2], trials (move counter, advanced).  Mode 0: ln_f [w] constant,
 * or, where one_over_t [w] is set, ln f = n_levels [w] / (trials - t_base [w]
 * + 1); `moves` per walker.  Mode 1: n_meas measurements of `moves` moves each,
 * idx_out / order_out [w][n_meas] (Ising M, Potts sum_k n_k^2).  Walkers
 * run in shared memory when all can be resident that way or >= 256 fit an SM
 * (and a call makes fewer than 2^31 moves per walker), else in global memory;
 * mode | 0x10 forces global memory, mode | 0x20 shared memory (same results).
 * At most 2^24 sites per walker.
 * Replaces critmc kernels/flathist.py:28-132.                                */
int32_t critmc_fh_run(int32_t mode, int8_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz, int32_t q,
                      int32_t n_walkers, const uint32_t* keys, int32_t levels, int64_t* idx, int64_t* order,
                      double* lng, int64_t* hist, const int32_t* window, uint64_t* trials, const double* ln_f,
                      const double* n_levels, const int32_t* one_over_t, const uint64_t* t_base, int64_t moves,
                      int32_t n_meas, int64_t* idx_out, int64_t* order_out, void* stream);

/* Greedy descent of each walker into its window before a flat-histogram run:
 * step j draws Philox(j mod 2^32, j / 2^32, 0x0C, 0) with the walker's key
 * (site and Potts proposal as in critmc_fh_run) and keeps the move when the
 * level does not move away from [window[0], window[1]].  spins, idx (the
 * starting level of each configuration), order (Ising M; Potts counts [q])
 * are updated; steps_out [w] gets the steps taken, -1 when max_steps did not
 * reach the window.  All arrays are DEVICE arrays as for critmc_fh_run.
 * Replaces critmc flathist.py:96-130 (_walk_into_window).                    */
int32_t critmc_fh_descend(int8_t* spins, int32_t dim, int32_t lx, int32_t ly, int32_t lz, int32_t q,
                          int32_t n_walkers, const uint32_t* keys, int32_t levels, int64_t* idx, int64_t* order,
                          const int32_t* window, int64_t max_steps, int64_t* steps_out, void* stream);

/* ---- chains owned by the library (handles) ----------------------------------
 * The library allocates and keeps a chain's lattice, running sums, Philox key
 * and sweep counter; the caller passes states in critmc's site order (first
 * coordinate fastest) and gets per-measurement series.  Replaces critmc's
 * Model.advance with the state held by Simulation (src/critmc/models.py:58-68,
 * sim.py:174, :188-191).
 * model_kind: CRITMC_MODEL_*.  dims: extents {lx, ly, lz}, 0 for absent
 * axes (1D: {L, 0, 0}); every extent even.  q_or_n: Potts q, O(n) n (2, 3);
 * h: Ising field.  The chain's Philox key is words 0, 1 of
 * Philox(chain_id, 0, 0x205, chain_id >> 32) under the key (seed_lo, seed_hi).
 * start: CRITMC_START_RANDOM (from the chain's key), _ORDERED (all +1 / state
 * 0 / (1, 0, ..)), or _STATE from init_state (HOST: int8 [N] Ising +-1 or
 * Potts 0..q-1, double [N][n] O(n)).  Multi-spin-coded Ising (2D/3D, lx/64 a
 * power of two) and 1-byte lattices are chosen by shape.                     */
typedef struct critmc_chain critmc_chain;
#define CRITMC_MODEL_ISING 0
#define CRITMC_MODEL_POTTS 1
#define CRITMC_MODEL_ON 2
#define CRITMC_START_RANDOM 0
#define CRITMC_START_ORDERED 1
#define CRITMC_START_STATE 2
int32_t critmc_chain_create(int32_t model_kind, const int32_t dims[3], int32_t q_or_n, double h,
                            uint32_t seed_lo, uint32_t seed_hi, uint64_t chain_id, int32_t start,
                            const void* init_state, critmc_chain** handle);
int32_t critmc_chain_destroy(critmc_chain* chain);
/* layout: 0 multi-spin-coded, 1 byte, 2 float; sweep: the chain's counter */
int32_t critmc_chain_info(const critmc_chain* chain, int32_t* layout, uint32_t* sweep, uint32_t key[2]);
/* O(n) Metropolis step size (critmc's running["step"], sim.py:226-229) */
int32_t critmc_chain_set_step(critmc_chain* chain, double step);
/* n_meas applications of schedule (HOST (code, reps) rows) at inverse
 * temperature beta, on `stream`.  Outputs (device-accessible):
 * Ising e_out = E_b, m_out = M [n_meas] int64; Potts e_out = E, m_out =
 * counts [n_meas][q]; O(n) f64_out = E [n_meas] | M [n_meas][n] | stiffness
 * cos [n_meas][dim] | sin [n_meas][dim]; aux_out [n_meas][4] for all.
 * Results equal the per-model entry points for the same key and sweep.     */
int32_t critmc_advance(critmc_chain* chain, double beta, const int64_t* schedule, int32_t n_rows,
                       int32_t n_meas, int64_t* e_out, int64_t* m_out, int64_t* aux_out,
                       double* f64_out, void* stream);
/* State in critmc's site order into / from HOST memory (synchronous);
 * running_out (HOST, may be null): Ising (E_b, M), Potts (E, counts[q]).  */
int32_t critmc_get_state(critmc_chain* chain, void* host_out, int64_t* running_out, void* stream);
int32_t critmc_set_state(critmc_chain* chain, const void* host_in, void* stream);

/* Batch queue over handles: submissions of many chains run together as work
 * items (critmc_run_items), one submission per chain per round, in
 * submission order per chain.  poll runs rounds until nothing is pending or
 * max_done tickets are finished, then waits for `stream`; cancel drops a
 * pending submission.  No counterpart in critmc (process pool,
 * src/critmc/runner.py:154-223).                                            */
typedef struct critmc_batch critmc_batch;
int32_t critmc_batch_create(critmc_batch** batch);
int32_t critmc_batch_destroy(critmc_batch* batch);
int32_t critmc_batch_submit(critmc_batch* batch, critmc_chain* chain, double beta,
                            const int64_t* schedule, int32_t n_rows, int32_t n_meas, int64_t* e_out,
                            int64_t* m_out, int64_t* aux_out, double* f64_out, int64_t* ticket);
int32_t critmc_batch_poll(critmc_batch* batch, void* stream, int64_t* done, int32_t max_done,
                          int32_t* n_done);
int32_t critmc_batch_cancel(critmc_batch* batch, int64_t ticket);
int32_t critmc_batch_pending(const critmc_batch* batch);

/* Instantiated CUDA graphs are cached across calls with identical parameters
 * (the same chains advanced slice after slice): capacity in entries (default
 * 64, 0 disables caching and frees every entry) and current size.  No
 * counterpart in critmc.                                                     */
int32_t critmc_graph_cache_set_capacity(int32_t entries);
int32_t critmc_graph_cache_size(void);

/* critmc_ising_msc_run for callers that cannot allocate device memory.
 * No counterpart in the reference (critmc has no device memory at all).
 * Some callers cannot call cudaMalloc where they run the sampler: a plugin
 * whose host framework owns the device allocator, code that must not stall
 * the device with an allocation, an embedded host that forbids allocation
 * after start-up.  This variant takes the same arguments minus `scratch`,
 * `mode` (always one launch per half-sweep, no CUDA graph) and keeps its
 * accumulators in a 1 MiB array built into the library, which every GPU that
 * loads the library holds until the process exits.  Limit:
 * critmc_ising_msc_scratch_bytes(n_chains, n_meas) <= 1 MiB, i.e.
 * n_chains * n_meas <= 43690; larger calls fail with CRITMC_ERR_INVALID
 * before any launch.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  A lookup that fails is not cached (the next call tries again), and
 * the address is looked up again after cudaDeviceReset, which gives the device
 * a new context in which the array may sit elsewhere.  All calls share the array: calls that overlap on the GPU (other
 * streams, other host threads) race and must be serialised by the caller.
 * It calls no cudaMalloc/cudaFree and creates no streams, events or graphs.  */
int64_t critmc_ising_msc_noalloc_max_scratch_bytes(void);
int32_t critmc_ising_msc_run_noalloc(uint32_t* spins, int32_t dim, int32_t lx, int32_t ly,
                                     int32_t lz, int32_t n_chains, const uint32_t* keys,
                                     const uint32_t* tables, int32_t n_groups, uint32_t sweep0,
                                     const int64_t* schedule, int32_t n_rows, int32_t n_meas,
                                     int64_t* running, int64_t* e_out, int64_t* m_out,
                                     int64_t* aux_out, int32_t k_inline, void* stream);

/* Energy E_b = -sum_<ij> s_i s_j and magnetisation M of MSC chains, written
 * to out[n_chains][2] (device).  critmc kernels/ising.py:32-45.           */
int32_t critmc_ising_msc_measure(const uint32_t* spins, int32_t dim, int32_t lx, int32_t ly,
                                 int32_t lz, int32_t n_chains, int64_t* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CRITMC_B200_H */
