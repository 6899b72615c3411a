// Host-side helpers of the C ABI: per-thread error text and status codes.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
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

// A stream the library may capture into a CUDA graph: the caller's stream, or,
// when the caller passed the legacy default stream, a per-thread private
// stream ordered after it (and `finish` orders the legacy stream after it).
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
