// Host-side helpers of the C ABI: per-thread error text and status codes.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

#include "critmc_b200.h"

namespace critmc {

void set_error(const char* msg);
void clear_error();

inline int fail(int code, const char* msg) {
  set_error(msg);
  return code;
}

// record the pending CUDA error (clearing it) and return CRITMC_ERR_CUDA
int cuda_fail(const char* what);
// CRITMC_OK if no CUDA error is pending, else record and clear it (CRITMC_ERR_CUDA)
int cuda_check(const char* what);

// Clusters of `cl` blocks (2..16) of `threads` threads of a team kernel that
// the current GPU can run at once (0: it cannot schedule that cluster size);
// clusters of more than 8 blocks need the non-portable size attribute.
// The answer is kept per device, kernel and size (a server asks before every
// tick's launch).
int team_clusters_cached(const void* kern, int cl, int* out);
void team_clusters_store(const void* kern, int cl, int clusters);
template <typename... KArgs>
int team_clusters(void (*kern)(KArgs...), int cl, int threads) {
  if (cl < 2 || cl > 16) return fail(CRITMC_ERR_INVALID, "team size must be 2..16");
  int known = 0;
  if (team_clusters_cached(reinterpret_cast<const void*>(kern), cl, &known)) return known;
  if (cl > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return cuda_fail("cluster size attribute");
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cl);
  cfg.blockDim = dim3((unsigned)threads);
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess) return cuda_fail("cluster occupancy");
  team_clusters_store(reinterpret_cast<const void*>(kern), cl, clusters);
  return clusters;
}

// Persistent launch of a team kernel: as many clusters of `cl` blocks as fit
// on the GPU at once and no more than `n_items`.  A size the GPU cannot
// schedule is refused rather than launched.
template <typename... KArgs, typename... Args>
int launch_team(void (*kern)(KArgs...), int cl, int threads, int n_items, cudaStream_t s, Args&&... args) {
  const int clusters = team_clusters(kern, cl, threads);
  if (clusters < 0) return clusters;
  if (clusters < 1) return fail(CRITMC_ERR_UNSUPPORTED, "this GPU cannot schedule a cluster of that many blocks");
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(std::min(n_items, clusters) * cl));
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...) != cudaSuccess) return cuda_fail("team launch");
  return CRITMC_OK;
}

// Makes `dev` the calling thread's current device for the guard's lifetime
// and restores the previous one.  Handle-based entry points (chains, batches)
// remember the device they were created on and must launch there whatever
// device the caller's thread has current.
struct DeviceScope {
  int prev = -1;
  int status = CRITMC_OK;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      status = cuda_fail("cudaGetDevice");
    } else if (prev != dev && cudaSetDevice(dev) != cudaSuccess) {
      status = cuda_fail("cudaSetDevice");
    }
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

// A stream the library may capture into a CUDA graph: the caller's stream, or,
// when the caller passed the legacy default stream, a per-thread private
// stream ordered after it (and `finish` orders the legacy stream after it).
// The private stream is kept per thread and per device, so a thread that
// switches devices never enqueues work on another device's stream.
struct CaptureStream {
  cudaStream_t user = nullptr;
  cudaStream_t work = nullptr;
  bool private_stream = false;
  int begin(void* stream);
  int finish();
};

// Instantiated CUDA graphs of repeated calls, keyed by the exact bytes of
// everything their capture depends on (kernel parameters, launch shapes,
// schedule).  A caller that advances the same chains slice after slice (a
// server's ticks, Simulation.run chunks) replays its graph instead of
// capturing and instantiating it again.  Least recently used entries are
// destroyed beyond the capacity (a graph still in flight is freed by CUDA
// when it completes).
class GraphKey {
 public:
  template <typename T>
  GraphKey& add(const T& v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    bytes.insert(bytes.end(), p, p + sizeof(T));
    return *this;
  }
  GraphKey& add_bytes(const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    bytes.insert(bytes.end(), c, c + n);
    return *this;
  }
  std::vector<unsigned char> bytes;
};

cudaGraphExec_t graph_cache_find(const GraphKey& key);
// takes ownership of exec
void graph_cache_insert(const GraphKey& key, cudaGraphExec_t exec);

}  // namespace critmc
