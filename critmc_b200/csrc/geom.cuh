// Site geometry of the colour-major lattices (byte and float layouts) and
// small block-level helpers shared by the one-block-per-chain kernels.
#pragma once
#include "common.cuh"
#include "host_common.h"

namespace critmc {

struct ByteGeom {
  int dim, lx, ly, lz, hx, rows;
  uint32_t slots;  // sites per colour
};

__device__ __forceinline__ void byte_row_index(const ByteGeom& g, uint32_t slot, int& r, int& i) {
  r = (int)(slot / (uint32_t)g.hx);
  i = (int)slot - r * g.hx;
}

// slots (in the other colour's plane) of the Z neighbours of slot (r, i) of colour c
template <int Z>
__device__ __forceinline__ void byte_neighbours(const ByteGeom& g, int c, int r, int i, uint32_t* nb) {
  int y = r, z = 0;
  if constexpr (Z == 6) {
    y = r % g.ly;
    z = r / g.ly;
  }
  const int p = (c + y + z) & 1;
  const int ia = p ? ((i == g.hx - 1) ? 0 : i + 1) : ((i == 0) ? g.hx - 1 : i - 1);
  nb[0] = (uint32_t)(r * g.hx + i);
  nb[1] = (uint32_t)(r * g.hx + ia);
  if constexpr (Z >= 4) {
    const int ym = (y == 0) ? g.ly - 1 : y - 1, yp = (y == g.ly - 1) ? 0 : y + 1;
    nb[2] = (uint32_t)((ym + g.ly * z) * g.hx + i);
    nb[3] = (uint32_t)((yp + g.ly * z) * g.hx + i);
  }
  if constexpr (Z == 6) {
    const int zm = (z == 0) ? g.lz - 1 : z - 1, zp = (z == g.lz - 1) ? 0 : z + 1;
    nb[4] = (uint32_t)((y + g.ly * zm) * g.hx + i);
    nb[5] = (uint32_t)((y + g.ly * zp) * g.hx + i);
  }
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  T out = 0;
  const int nw = (blockDim.x + 31) >> 5;
  for (int q = 0; q < nw; ++q) out += red[q];
  return out;
}

inline int byte_geom(int dim, int lx, int ly, int lz, ByteGeom& g) {
  if (dim < 1 || dim > 3) return fail(CRITMC_ERR_UNSUPPORTED, "dimension must be 1, 2 or 3");
  if (dim < 2) ly = 1;
  if (dim < 3) lz = 1;
  if (lx < 2 || lx % 2 || (dim >= 2 && (ly < 2 || ly % 2)) || (dim == 3 && (lz < 2 || lz % 2)))
    return fail(CRITMC_ERR_UNSUPPORTED, "checkerboard sweeps need every extent even and >= 2");
  const long long n = (long long)lx * ly * lz;
  if (n >= (1LL << 30)) return fail(CRITMC_ERR_UNSUPPORTED, "lattice too large");
  g.dim = dim;
  g.lx = lx;
  g.ly = ly;
  g.lz = lz;
  g.hx = lx / 2;
  g.rows = ly * lz;
  g.slots = (uint32_t)(n / 2);
  return CRITMC_OK;
}

}  // namespace critmc
