// Per-family launchers of the work-item kernels (implemented next to each
// family's sweep code) used by critmc_run_items.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "critmc_b200.h"

namespace critmc {

constexpr int ITEM_THREADS = 512;

// Each launcher starts a persistent kernel over `n` items at `items` (device)
// whose blocks pull item indices from *queue (zeroed by the caller).  team 1:
// one block per item (`smem` bytes of dynamic shared memory for resident
// lattices); team 2, 4, 8 or 16: a thread-block cluster of that many blocks
// per item, the lattice in global memory.  `ctl` bounds the run (all null:
// unbounded).
int msc_items_launch(const critmc_item* items, int n, unsigned* queue, size_t smem, int team, const RunCtl& ctl,
                     cudaStream_t s);
int byte_items_launch(const critmc_item* items, int n, unsigned* queue, size_t smem, int team, const RunCtl& ctl,
                      cudaStream_t s);
// O(n): all n items share n_comp and dim (one kernel per variant)
int on_items_launch(const critmc_item* items, int n, int n_comp, int dim, unsigned* queue, size_t smem, int team,
                    const RunCtl& ctl, cudaStream_t s);

// Clusters of `team` blocks (2, 4, 8, 16) of each family's item kernel that the
// current GPU runs at once (0: it cannot schedule that size), or an error.
int msc_items_team_clusters(int team);
int byte_items_team_clusters(int team);
int on_items_team_clusters(int n_comp, int dim, int team);

}  // namespace critmc
