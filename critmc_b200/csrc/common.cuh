// Device helpers shared by every sampler kernel of the library.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

#include "philox.h"
#include "critmc_b200.h"

namespace critmc {

// ---------------------------------------------------------------------------
// Bit-sliced arithmetic on 32 independent lanes (one lane per bit).
// ---------------------------------------------------------------------------

// three-input boolean function with a compile-time truth table
template <unsigned LUT>
__device__ __forceinline__ uint32_t lop3(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(LUT));
  return d;
}
// truth-table constants for lop3: a = 0xF0, b = 0xCC, c = 0xAA
constexpr unsigned LA = 0xF0, LB = 0xCC, LC = 0xAA;
constexpr unsigned lut_xor3 = LA ^ LB ^ LC;
constexpr unsigned lut_maj = (LA & LB) | (LA & LC) | (LB & LC);

// Per-lane count (0..Z) of the set bits of Z masks, as three bit planes.
struct Count3 {
  uint32_t b0, b1, b2;
};

template <int Z>
__device__ __forceinline__ Count3 count_bits(const uint32_t* x);

template <>
__device__ __forceinline__ Count3 count_bits<2>(const uint32_t* x) {
  return Count3{x[0] ^ x[1], x[0] & x[1], 0u};
}

template <>
__device__ __forceinline__ Count3 count_bits<4>(const uint32_t* x) {
  const uint32_t s1 = x[0] ^ x[1], c1 = x[0] & x[1];
  const uint32_t s2 = x[2] ^ x[3], c2 = x[2] & x[3];
  const uint32_t c3 = s1 & s2;
  return Count3{s1 ^ s2, lop3<lut_xor3>(c1, c2, c3), lop3<lut_maj>(c1, c2, c3)};
}

template <>
__device__ __forceinline__ Count3 count_bits<6>(const uint32_t* x) {
  const uint32_t sa = lop3<lut_xor3>(x[0], x[1], x[2]), ca = lop3<lut_maj>(x[0], x[1], x[2]);
  const uint32_t sb = lop3<lut_xor3>(x[3], x[4], x[5]), cb = lop3<lut_maj>(x[3], x[4], x[5]);
  const uint32_t cab = sa & sb;
  return Count3{sa ^ sb, lop3<lut_xor3>(ca, cb, cab), lop3<lut_maj>(ca, cb, cab)};
}

// mask of the lanes whose count equals V (compile-time V)
template <int V>
__device__ __forceinline__ uint32_t count_eq(const Count3& c) {
  constexpr unsigned m0 = (V & 1) ? LC : (0xFFu & ~LC);
  constexpr unsigned m1 = (V & 2) ? LB : (0xFFu & ~LB);
  constexpr unsigned m2 = (V & 4) ? LA : (0xFFu & ~LA);
  return lop3<(m0 & m1 & m2)>(c.b2, c.b1, c.b0);
}

// broadcast bit `bit` of a uniform word to a full lane mask
__device__ __forceinline__ uint32_t bcast_bit(uint32_t t, int bit) {
  return 0u - ((t >> bit) & 1u);
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ unsigned long long as_ull(long long v) {
  return static_cast<unsigned long long>(v);
}

// ---------------------------------------------------------------------------
// Bounds-checked builds (-DCRITMC_CHECK).  CRITMC_IDX(i, n) compares an index
// with the extent of its array.  An index out of range is recorded (the first
// one per translation unit: source line, index and extent, plus a count of
// every bad index) and replaced by 0, so the access stays inside the array and
// the kernel runs on: a check never traps.  critmc_check_report() reads and
// clears the records of every translation unit.  Release builds compile the
// checks away.
// ---------------------------------------------------------------------------
struct CheckRecord {
  int line;
  unsigned int hits;
  unsigned long long index, extent;
};
// host: adds a translation unit's reader to the report (returns 0)
int check_register(const char* file, int (*read_and_clear)(CheckRecord*));

#ifdef CRITMC_CHECK
static __device__ CheckRecord g_check_record;
__device__ __forceinline__ size_t check_index(size_t i, size_t n, int line) {
  if (i < n) return i;
  if (atomicAdd(&g_check_record.hits, 1u) == 0) {
    g_check_record.line = line;
    g_check_record.index = i;
    g_check_record.extent = n;
  }
  return 0;
}
static int check_read_and_clear(CheckRecord* out) {
  if (cudaMemcpyFromSymbol(out, g_check_record, sizeof(CheckRecord)) != cudaSuccess) return -1;
  const CheckRecord zero{0, 0u, 0ull, 0ull};
  if (cudaMemcpyToSymbol(g_check_record, &zero, sizeof(CheckRecord)) != cudaSuccess) return -1;
  return 0;
}
static const int g_check_registered = check_register(__FILE__, &check_read_and_clear);
#define CRITMC_IDX(i, n) ::critmc::check_index((size_t)(i), (size_t)(n), __LINE__)
#else
#define CRITMC_IDX(i, n) (i)
#endif

// ---------------------------------------------------------------------------
// Bounded runs of the persistent kernels (critmc_control).  One thread per
// block polls: the block's elapsed time against the budget every time, and the
// host-mapped cancel and status words at most every CTL_POLL_NS (each read
// crosses the bus).  A block that must stop records why in the status word
// (first reason wins) and leaves its work; the others see the status word on
// their next poll.  No wait in here: a poll never blocks.
// ---------------------------------------------------------------------------
struct RunCtl {
  const volatile unsigned* cancel;  // host-mapped; nonzero = cancel (null: unbounded run)
  int* status;                      // host-mapped; 0, CRITMC_ERR_TIMEOUT or CRITMC_ERR_CANCELLED
  unsigned long long budget_ns;     // per-block run time budget, 0 = none
};

constexpr unsigned long long CTL_POLL_NS = 100000ull;

// device view of a critmc_control (all null for an unbounded run); host code
RunCtl control_device(const critmc_control* ctl);

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct CtlPoll {
  unsigned long long t0, last;
  __device__ __forceinline__ void start() { t0 = last = global_ns(); }
  // 0 to go on, else the status that stops the block
  __device__ __forceinline__ int check(const RunCtl& c) {
    if (!c.status) return 0;
    const unsigned long long now = global_ns();
    if (c.budget_ns && now - t0 > c.budget_ns) {
      atomicCAS_system(c.status, 0, CRITMC_ERR_TIMEOUT);
      return CRITMC_ERR_TIMEOUT;
    }
    if (now - last >= CTL_POLL_NS) {
      last = now;
      if (*c.cancel) {
        atomicCAS_system(c.status, 0, CRITMC_ERR_CANCELLED);
        return CRITMC_ERR_CANCELLED;
      }
      const int st = *(volatile int*)c.status;
      if (st) return st;
    }
    return 0;
  }
};

// ---------------------------------------------------------------------------
// Teams: the thread blocks that advance one work item together.  CL == 1 is
// one block; CL > 1 a thread-block cluster of CL blocks on CL SMs of one GPC
// (the hardware schedules a cluster's blocks together).  sync() is the block
// barrier, or the cluster barrier (barrier.cluster.arrive has release and
// barrier.cluster.wait acquire semantics at cluster scope): what any thread of
// the team wrote before it, to shared or global memory, every thread of the
// team sees after it.  Every thread of every block of a team must reach the
// same sequence of sync() calls, so all control flow around them depends only
// on values that are the same in the whole team.  at(p, r) is block r's copy
// of the shared variable p (distributed shared memory).
// ---------------------------------------------------------------------------
template <int CL>
struct Team {
  static_assert(CL == 1 || CL == 2 || CL == 4 || CL == 8 || CL == 16, "team sizes: 1, 2, 4, 8 or 16 blocks");
  __device__ static __forceinline__ unsigned rank() {
    if constexpr (CL == 1) return 0;
    else return cooperative_groups::this_cluster().block_rank();
  }
  __device__ static __forceinline__ void sync() {
    if constexpr (CL == 1) __syncthreads();
    else cooperative_groups::this_cluster().sync();
  }
  template <typename T>
  __device__ static __forceinline__ T* at(T* p, unsigned r) {
    if constexpr (CL == 1) return p;
    else return cooperative_groups::this_cluster().map_shared_rank(p, r);
  }
};

// ---------------------------------------------------------------------------
// Error reporting from kernels: the first failing kernel writes its code.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void report_error(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

}  // namespace critmc
