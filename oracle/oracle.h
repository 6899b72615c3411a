/* CPU oracle of the critmc_b200 kernels -- test infrastructure only. */
#ifndef CRITMC_ORACLE_H
#define CRITMC_ORACLE_H
#include <stdint.h>

void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void oracle_philox_rounds(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4], int rounds);
int oracle_ising_table(int algo, int z, double beta, double h, uint32_t* kind, uint32_t* thr);
int64_t oracle_ising_bond_energy(const int8_t* s, int dim, int lx, int ly, int lz);
int oracle_ising_msc_run(int8_t* s, int dim, int lx, int ly, int lz, const uint32_t key[2],
                         const uint32_t* tables, uint32_t sweep0, const int64_t* schedule,
                         int n_rows, int n_meas, int64_t* running, int64_t* e_out, int64_t* m_out,
                         int64_t* aux_out);
int oracle_ising_msc_run_rounds(int8_t* s, int dim, int lx, int ly, int lz, const uint32_t key[2],
                                const uint32_t* tables, uint32_t sweep0, const int64_t* schedule,
                                int n_rows, int n_meas, int64_t* running, int64_t* e_out, int64_t* m_out,
                                int64_t* aux_out, int rounds);
int oracle_ising_byte_run(int8_t* s, int dim, int lx, int ly, int lz, const uint32_t key[2],
                          const uint32_t* tables, uint32_t sweep0, const int64_t* schedule,
                          int n_rows, int n_meas, int64_t* running, int64_t* e_out,
                          int64_t* m_out, int64_t* aux_out);
int oracle_potts_tables(int z, double beta, uint64_t* boltz, uint64_t* weight);
int oracle_potts_run(int8_t* s, int dim, int lx, int ly, int lz, int q, const uint32_t key[2],
                     double beta, uint32_t sweep0, const int64_t* schedule, int n_rows, int n_meas,
                     int64_t* energy, int64_t* counts, int64_t* e_out, int64_t* counts_out,
                     int64_t* aux_out);
int oracle_on_run(float* s, int dim, int lx, int ly, int lz, int n, const uint32_t key[2],
                  double beta, double step, uint32_t sweep0, const int64_t* schedule, int n_rows,
                  int n_meas, double* e_out, double* m_out, double* sc_out, double* ss_out,
                  int64_t* aux_out);
int oracle_cluster_update(int8_t* lay, int dim, int lx, int ly, int lz, int q, const uint32_t key[2],
                          double beta, int algo, uint32_t sweep, int64_t* d_energy, int64_t* d_mag,
                          int64_t* counts_delta, int64_t stats[3]);
int oracle_on_cluster_update(float* s, int dim, int lx, int ly, int lz, int ncomp, const uint32_t key[2],
                             double beta, int algo, uint32_t sweep, int64_t stats[3]);
int oracle_fh_run(int mode, int8_t* s, int dim, int lx, int ly, int lz, int q, const uint32_t key[2],
                  int64_t* idx_io, int64_t* order, double* lng, int64_t* hist, int lo, int hi,
                  uint64_t* trials, double ln_f, double n_levels, int one_over_t, uint64_t t_base,
                  int64_t moves, int n_meas, int64_t* idx_out, int64_t* order_out);
int64_t oracle_fh_descend(int8_t* s, int dim, int lx, int ly, int lz, int q, const uint32_t key[2], int64_t* idx_io,
                          int64_t* order, int lo, int hi, int64_t max_steps);
int oracle_ea_pt_run(int8_t* spins, const double* J, int dim, int lx, int ly, int lz, int m,
                     const uint32_t* keys, const double* betas, const uint32_t* swap_thr, int width,
                     int* perm, int* labels, uint32_t t0, int n_steps, int n_bins,
                     int sweeps_per_step, double* acc, int64_t* swap_acc, int64_t* swap_try,
                     int64_t* label_hist, int64_t* trips);
void critmc_port_pcg_raw(uint64_t w[4], int64_t n, uint64_t* out);
int critmc_port_ising_run(int8_t* s, const int64_t* nbr, int64_t n, int z, double beta, double h, uint64_t pcg[4],
                          const int64_t* schedule, int n_rows, int n_meas, int64_t* running, int64_t* e_out,
                          int64_t* m_out, int64_t* aux_out);
#endif
