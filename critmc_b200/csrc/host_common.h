// Host-side helpers of the C ABI: per-thread error text and status codes.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

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

}  // namespace critmc
