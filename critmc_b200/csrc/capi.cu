// C ABI plumbing shared by all kernels: version, error text, class tables.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "host_common.h"

// A bounded-run control: one page of pinned host memory mapped into the
// device, [0] the cancel word (host writes), [1] the status word (kernels
// write), plus the per-block time budget of the runs it is passed to.
struct critmc_control {
  unsigned* host = nullptr;
  unsigned* dev = nullptr;
  unsigned long long budget_ns = 0;
};

namespace critmc {

static thread_local char g_error[512] = {0};

void set_error(const char* msg) {
  std::snprintf(g_error, sizeof(g_error), "%s", msg ? msg : "");
}

void clear_error() { g_error[0] = 0; }

int cuda_fail(const char* what) {
  const cudaError_t e = cudaGetLastError();
  std::snprintf(g_error, sizeof(g_error), "%s: %s", what, cudaGetErrorString(e));
  return CRITMC_ERR_CUDA;
}

int cuda_check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return CRITMC_OK;
  std::snprintf(g_error, sizeof(g_error), "%s: %s", what, cudaGetErrorString(e));
  return CRITMC_ERR_CUDA;
}

namespace {
struct TeamCapacity {
  int dev, cl, clusters;
  const void* kern;
};
std::mutex g_team_mutex;
std::vector<TeamCapacity> g_team_capacity;  // a few entries: kernels x sizes x devices
}  // namespace

int team_clusters_cached(const void* kern, int cl, int* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  std::lock_guard<std::mutex> lock(g_team_mutex);
  for (const TeamCapacity& t : g_team_capacity)
    if (t.dev == dev && t.cl == cl && t.kern == kern) {
      *out = t.clusters;
      return 1;
    }
  return 0;
}

void team_clusters_store(const void* kern, int cl, int clusters) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  std::lock_guard<std::mutex> lock(g_team_mutex);
  g_team_capacity.push_back(TeamCapacity{dev, cl, clusters, kern});
}

namespace {

struct GraphEntry {
  std::vector<unsigned char> key;
  cudaGraphExec_t exec;
  uint64_t used;
};
std::mutex g_graph_mu;
std::vector<GraphEntry> g_graphs;
uint64_t g_graph_clock = 0;
size_t g_graph_capacity = 64;

}  // namespace

cudaGraphExec_t graph_cache_find(const GraphKey& key) {
  std::lock_guard<std::mutex> lock(g_graph_mu);
  for (GraphEntry& e : g_graphs)
    if (e.key == key.bytes) {
      e.used = ++g_graph_clock;
      return e.exec;
    }
  return nullptr;
}

void graph_cache_insert(const GraphKey& key, cudaGraphExec_t exec) {
  std::lock_guard<std::mutex> lock(g_graph_mu);
  while (!g_graphs.empty() && g_graphs.size() >= g_graph_capacity) {
    auto old = std::min_element(g_graphs.begin(), g_graphs.end(),
                                [](const GraphEntry& a, const GraphEntry& b) { return a.used < b.used; });
    cudaGraphExecDestroy(old->exec);
    g_graphs.erase(old);
  }
  if (g_graph_capacity == 0) {
    cudaGraphExecDestroy(exec);
    return;
  }
  g_graphs.push_back(GraphEntry{key.bytes, exec, ++g_graph_clock});
}

int CaptureStream::begin(void* stream) {
  user = (cudaStream_t)stream;
  if (user != nullptr && user != cudaStreamLegacy && user != cudaStreamPerThread) {
    work = user;
    private_stream = false;
    return CRITMC_OK;
  }
  constexpr int MAX_DEVICES = 64;
  static thread_local cudaStream_t priv[MAX_DEVICES] = {};
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return cuda_fail("cudaGetDevice");
  if (dev < 0 || dev >= MAX_DEVICES) return fail(CRITMC_ERR_UNSUPPORTED, "device ordinal out of range");
  if (!priv[dev] && cudaStreamCreateWithFlags(&priv[dev], cudaStreamNonBlocking) != cudaSuccess)
    return cuda_fail("stream create");
  work = priv[dev];
  private_stream = true;
  cudaEvent_t ev;
  if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return cuda_fail("event");
  cudaEventRecord(ev, user);
  cudaStreamWaitEvent(work, ev, 0);
  cudaEventDestroy(ev);
  return CRITMC_OK;
}

int CaptureStream::finish() {
  if (!private_stream) return CRITMC_OK;
  cudaEvent_t ev;
  if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return cuda_fail("event");
  cudaEventRecord(ev, work);
  cudaStreamWaitEvent(user, ev, 0);
  cudaEventDestroy(ev);
  return CRITMC_OK;
}

}  // namespace critmc

namespace {

struct CheckReader {
  const char* file;
  int (*read)(critmc::CheckRecord*);
};
std::vector<CheckReader>& check_readers() {
  static std::vector<CheckReader> r;
  return r;
}

}  // namespace

int critmc::check_register(const char* file, int (*read_and_clear)(CheckRecord*)) {
  check_readers().push_back(CheckReader{file, read_and_clear});
  return 0;
}

extern "C" int64_t critmc_check_report(char* buf, int32_t size) {
  critmc::clear_error();
  if (buf && size > 0) buf[0] = 0;
#ifndef CRITMC_CHECK
  return -1;  // not a bounds-checked build
#else
  int64_t hits = 0;
  size_t used = 0;
  for (const CheckReader& r : check_readers()) {
    critmc::CheckRecord rec;
    if (r.read(&rec) != 0) return critmc::cuda_fail("read check record");
    if (!rec.hits) continue;
    hits += rec.hits;
    if (buf && size > 0 && used + 1 < (size_t)size) {
      const char* base = std::strrchr(r.file, '/');
      used += (size_t)std::snprintf(buf + used, (size_t)size - used, "%s:%d index %llu of %llu (%u bad); ",
                                    base ? base + 1 : r.file, rec.line, rec.index, rec.extent, rec.hits);
      if (used >= (size_t)size) used = (size_t)size - 1;
    }
  }
  return hits;
#endif
}

critmc::RunCtl critmc::control_device(const critmc_control* ctl) {
  RunCtl r{nullptr, nullptr, 0ull};
  if (ctl && ctl->dev) {
    r.cancel = ctl->dev;
    r.status = reinterpret_cast<int*>(ctl->dev + 1);
    r.budget_ns = ctl->budget_ns;
  }
  return r;
}

using namespace critmc;

extern "C" int32_t critmc_version(void) { return 100; }

extern "C" int32_t critmc_control_create(critmc_control** ctl) {
  clear_error();
  if (!ctl) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  *ctl = nullptr;
  critmc_control* c = new critmc_control();
  void* h = nullptr;
  if (cudaHostAlloc(&h, 64, cudaHostAllocMapped) != cudaSuccess) {
    delete c;
    return cuda_fail("pinned control page");
  }
  void* d = nullptr;
  if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
    cudaFreeHost(h);
    delete c;
    return cuda_fail("device view of the control page");
  }
  c->host = static_cast<unsigned*>(h);
  c->dev = static_cast<unsigned*>(d);
  std::memset(c->host, 0, 64);
  *ctl = c;
  return CRITMC_OK;
}

extern "C" int32_t critmc_control_destroy(critmc_control* ctl) {
  if (!ctl) return CRITMC_OK;
  if (ctl->host) cudaFreeHost(ctl->host);
  delete ctl;
  return CRITMC_OK;
}

extern "C" int32_t critmc_control_arm(critmc_control* ctl, int64_t budget_ns) {
  clear_error();
  if (!ctl || !ctl->host) return fail(CRITMC_ERR_INVALID, "null control");
  if (budget_ns < 0) return fail(CRITMC_ERR_INVALID, "budget_ns must not be negative");
  volatile unsigned* w = ctl->host;
  w[0] = 0;
  w[1] = 0;
  ctl->budget_ns = (unsigned long long)budget_ns;
  return CRITMC_OK;
}

extern "C" int32_t critmc_control_cancel(critmc_control* ctl) {
  clear_error();
  if (!ctl || !ctl->host) return fail(CRITMC_ERR_INVALID, "null control");
  volatile unsigned* w = ctl->host;
  w[0] = 1;
  return CRITMC_OK;
}

extern "C" int32_t critmc_control_status(const critmc_control* ctl) {
  if (!ctl || !ctl->host) return CRITMC_ERR_INVALID;
  const volatile int* w = reinterpret_cast<const volatile int*>(ctl->host + 1);
  return *w;
}

extern "C" int32_t critmc_control_wait(const critmc_control* ctl, void* stream) {
  clear_error();
  if (!ctl || !ctl->host) return fail(CRITMC_ERR_INVALID, "null control");
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return cuda_fail("synchronize");
  const int st = critmc_control_status(ctl);
  if (st == CRITMC_ERR_TIMEOUT) set_error("a bounded run ran out of its time budget; its outputs are incomplete");
  if (st == CRITMC_ERR_CANCELLED) set_error("a bounded run was cancelled; its outputs are incomplete");
  return st;
}

extern "C" int32_t critmc_graph_cache_set_capacity(int32_t entries) {
  if (entries < 0) return CRITMC_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_graph_mu);
  g_graph_capacity = (size_t)entries;
  while (g_graphs.size() > g_graph_capacity) {
    cudaGraphExecDestroy(g_graphs.front().exec);
    g_graphs.erase(g_graphs.begin());
  }
  return CRITMC_OK;
}

extern "C" int32_t critmc_graph_cache_size(void) {
  std::lock_guard<std::mutex> lock(g_graph_mu);
  return (int32_t)g_graphs.size();
}

extern "C" int32_t critmc_last_error(char* buf, int32_t size) {
  if (!buf || size <= 0) return CRITMC_ERR_INVALID;
  std::snprintf(buf, (size_t)size, "%s", g_error);
  return CRITMC_OK;
}

// p -> (kind, thr) with thr = round(p 2^32)
static void classify_p(double p, uint32_t& kind, uint32_t& thr) {
  if (!(p > 0.0)) {  // also NaN
    kind = CRITMC_KIND_NEVER;
    thr = 0;
    return;
  }
  if (p >= 1.0) {
    kind = CRITMC_KIND_ALWAYS;
    thr = 0;
    return;
  }
  const double t = std::nearbyint(std::ldexp(p, 32));
  if (t >= 4294967296.0) {
    kind = CRITMC_KIND_ALWAYS;
    thr = 0;
  } else if (t <= 0.0) {
    kind = CRITMC_KIND_NEVER;
    thr = 0;
  } else {
    kind = CRITMC_KIND_RANDOM;
    thr = (uint32_t)t;
  }
}

extern "C" int32_t critmc_ising_class_table(int32_t algo, int32_t z, double beta, double h,
                                            uint32_t* kind, uint32_t* thr,
                                            int32_t* spin_dependent) {
  clear_error();
  if (!kind || !thr) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (z < 1 || z > 7) return fail(CRITMC_ERR_INVALID, "coordination number must be in [1, 7]");
  if (!std::isfinite(beta) || !std::isfinite(h)) return fail(CRITMC_ERR_INVALID, "beta and h must be finite");
  for (int c = 0; c < CRITMC_NCLS; ++c) {
    kind[c] = CRITMC_KIND_NEVER;
    thr[c] = 0;
  }
  int dep = 0;
  for (int v = 0; v <= z; ++v) {
    for (int sb = 0; sb < 2; ++sb) {
      const double spin = sb ? 1.0 : -1.0;
      double p;
      if (algo == CRITMC_METROPOLIS) {
        // v anti-aligned neighbours: a = s * sum_j s_j = z - 2v; dE = 2a + 2 h s
        // (critmc kernels/ising.py:48-57)
        const double a = (double)(z - 2 * v);
        const double d_e = 2.0 * a + 2.0 * h * spin;
        p = d_e <= 0.0 ? 1.0 : std::exp(-beta * d_e);
      } else if (algo == CRITMC_HEATBATH) {
        // v neighbours up: sum_j s_j = 2v - z (critmc kernels/ising.py:60-65)
        const double field = (double)(2 * v - z);
        p = 1.0 / (1.0 + std::exp(-2.0 * beta * (field + h)));
      } else {
        return fail(CRITMC_ERR_UNSUPPORTED, "class tables exist for metropolis and heatbath");
      }
      classify_p(p, kind[2 * v + sb], thr[2 * v + sb]);
    }
    if (kind[2 * v] != kind[2 * v + 1] || thr[2 * v] != thr[2 * v + 1]) dep = 1;
  }
  if (spin_dependent) *spin_dependent = dep;
  return CRITMC_OK;
}
