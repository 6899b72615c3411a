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

// slots (in the other colour's plane) of the Z neighbours of slot (r, i) of
// colour c, with the row's y and z given (r = y + ly z)
template <int Z>
__device__ __forceinline__ void byte_neighbours_at(const ByteGeom& g, int c, int r, int i, int y, int z,
                                                   uint32_t* nb) {
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

template <int Z>
__device__ __forceinline__ void byte_neighbours(const ByteGeom& g, int c, int r, int i, uint32_t* nb) {
  int y = r, z = 0;
  if constexpr (Z == 6) {
    y = r % g.ly;
    z = r / g.ly;
  }
  byte_neighbours_at<Z>(g, c, r, i, y, z, nb);
}

// Slot s of a colour plane and its coordinates (r = s / hx, i = s % hx,
// y = r % ly, z = r / ly), advanced by a fixed stride without a division per
// step: a thread that walks s, s + stride, ... divides once, at init.
struct SiteCursor {
  uint32_t s, stride;
  int r, i, y, z;
  int dr, di, dy, dz;
  __device__ __forceinline__ void init(const ByteGeom& g, uint32_t s0, uint32_t step) {
    s = s0;
    stride = step;
    r = (int)(s0 / (uint32_t)g.hx);
    i = (int)s0 - r * g.hx;
    y = r % g.ly;
    z = r / g.ly;
    dr = (int)(step / (uint32_t)g.hx);
    di = (int)step - dr * g.hx;
    dy = dr % g.ly;
    dz = dr / g.ly;
  }
  __device__ __forceinline__ void next(const ByteGeom& g) {
    s += stride;
    i += di;
    r += dr;
    y += dy;
    z += dz;
    if (i >= g.hx) {  // di < hx: one carry at most
      i -= g.hx;
      ++r;
      ++y;
    }
    if (y >= g.ly) {  // y + dy + 1 <= 2 ly - 1: one wrap at most
      y -= g.ly;
      ++z;
    }
  }
};

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
