// Streaming sums for the Gamma-method (U. Wolff, Comput. Phys. Commun. 156
// (2004) 143) of many chains' measurement series, accumulated on the device
// slice after slice so a series never has to leave the GPU.
//
// Per chain the state holds (all double): count n, shift x_0 (the first value;
// sums use y = x - x_0, which keeps the products small), sum y, sum y^2, the
// lag sums S_t = sum_i y_i y_{i+t} for t = 1..W, the first W values (head)
// and the last W values (tail).  From these the autocorrelation function
// Gamma(t) = [S_t - m (A_t + B_t) + (n - t) m^2] / (n - t) for t <= W follows
// exactly (A_t: all but the last t values, B_t: all but the first t), which is
// what critmc's gamma_method computes from the full series
// (src/critmc/stats/autocorr.py:381).
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "host_common.h"

namespace critmc {

constexpr int SS_TILE = 1024;

// state layout per chain, in doubles
__host__ __device__ inline size_t ss_stride(int W) { return 4 + 3 * (size_t)W; }

template <typename T>
__global__ void ss_update_kernel(const T* __restrict__ values, int n, int64_t ld, double* state, int W) {
  extern __shared__ double buf[];  // [W previous values | SS_TILE new values]
  const int chain = blockIdx.x;
  const T* x = values + (size_t)chain * ld;
  double* st = state + (size_t)chain * ss_stride(W);
  double* lag = st + 4;
  double* head = lag + W;
  double* tail = head + W;
  const int tid = threadIdx.x;
  double count = st[0];
  double shift = st[1];
  if (count == 0.0 && n > 0) shift = (double)x[0];
  // previous W values (valid ones: min(count, W)), oldest first
  const int have = (int)(count < W ? count : W);
  for (int k = tid; k < W; k += blockDim.x) buf[k] = (k >= W - have) ? tail[k] : 0.0;
  double lsum = 0.0, lsum2 = 0.0;
  double my_lag = 0.0;  // thread t handles lag t + 1 (blockDim >= W)
  __syncthreads();
  for (int base = 0; base < n; base += SS_TILE) {
    const int m = min(SS_TILE, n - base);
    for (int j = tid; j < m; j += blockDim.x) {
      const double y = (double)x[base + j] - shift;
      buf[W + j] = y;
      lsum += y;
      lsum2 += y * y;
      const double idx = count + base + j;
      if (idx < W) head[(int)idx] = y;
    }
    __syncthreads();
    if (tid < W) {
      const int t = tid + 1;
      const double valid_prev = count + base;  // values before this tile
      for (int j = 0; j < m; ++j) {
        // pair (i, i + t) with i + t = count + base + j, i >= 0
        if (valid_prev + j - t >= 0.0) my_lag += buf[W + j] * buf[W + j - t];
      }
    }
    __syncthreads();
    // keep the last W values in front of the next tile
    for (int k = tid; k < W; k += blockDim.x) {
      const int src = m + k;  // position in [prev | tile] of the new k-th of the last W
      buf[SS_TILE + W + k] = buf[src];  // stage in the spare area
    }
    __syncthreads();
    for (int k = tid; k < W; k += blockDim.x) buf[k] = buf[SS_TILE + W + k];
    __syncthreads();
  }
  // block sums of y and y^2
  __shared__ double red[2][32];
  lsum = warp_sum(lsum);
  lsum2 = warp_sum(lsum2);
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = lsum;
    red[1][tid >> 5] = lsum2;
  }
  __syncthreads();
  if (tid == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    st[0] = count + n;
    st[1] = shift;
    st[2] += a;
    st[3] += b;
  }
  if (tid < W) lag[tid] += my_lag;
  for (int k = tid; k < W; k += blockDim.x) tail[k] = buf[k];
}

}  // namespace critmc

using namespace critmc;

extern "C" int64_t critmc_stream_state_bytes(int32_t n_chains, int32_t max_lag) {
  if (n_chains < 1 || max_lag < 1 || max_lag > 1024) return -1;
  return (int64_t)n_chains * (int64_t)ss_stride(max_lag) * 8;
}

extern "C" int32_t critmc_stream_update(const void* values, int32_t is_double, int32_t n_chains, int32_t n,
                                        int64_t ld, double* state, int32_t max_lag, void* stream) {
  clear_error();
  if (!values || !state) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_chains < 1 || n < 0 || ld < n || max_lag < 1 || max_lag > 1024)
    return fail(CRITMC_ERR_INVALID, "need n_chains >= 1, 0 <= n <= ld, 1 <= max_lag <= 1024");
  if (n == 0) return CRITMC_OK;
  const int threads = std::max(64, ((max_lag + 31) / 32) * 32);
  const size_t smem = (size_t)(2 * max_lag + SS_TILE) * 8;
  cudaStream_t s = (cudaStream_t)stream;
  auto launch = [&](auto kern, auto* v) -> int {
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return cuda_fail("shared memory attribute");
    kern<<<n_chains, threads, smem, s>>>(v, n, ld, state, max_lag);
    return cuda_check("launch");
  };
  if (is_double) return launch(ss_update_kernel<double>, static_cast<const double*>(values));
  return launch(ss_update_kernel<long long>, static_cast<const long long*>(values));
}
