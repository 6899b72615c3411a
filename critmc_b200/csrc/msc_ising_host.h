// Host-side helpers of the MSC Ising kernels shared between translation units.
#pragma once
#include "msc_ising.cuh"

namespace critmc {

int msc_geom(int dim, int lx, int ly, int lz, MscGeom& g);
int msc_pick_rule(const uint32_t* kind, const uint32_t* thr, int z, int algo, int n_groups);

}  // namespace critmc
