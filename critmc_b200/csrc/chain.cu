// Chains owned by the library (handles) and a batch queue over them.
//
// A handle holds one chain's device lattice, running sums, Philox key and
// sweep counter; critmc_advance applies a schedule n_meas times through the
// per-model entry points, critmc_get_state / critmc_set_state convert between
// critmc's site order (first coordinate fastest) and the device layouts.  The
// batch queue collects critmc_advance requests of many handles and runs them
// together as work items (critmc_run_items), one round per poll.
//
// Stands in for critmc's Model.advance with the state and running sums kept
// by the caller (src/critmc/models.py:58-68, :113-135, :176-196, :248-272).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "host_common.h"
#include "philox.h"

using namespace critmc;

namespace {

enum Layout { LAYOUT_MSC = 0, LAYOUT_BYTE = 1, LAYOUT_ON = 2 };

}  // namespace

struct critmc_chain {
  int kind;    // CRITMC_MODEL_*
  int layout;  // Layout
  int dim, lx, ly, lz, q_or_n;
  double h;
  float step;
  uint32_t key[2];
  uint32_t sweep;
  int device;
  void* lattice;
  size_t lattice_bytes;
  int64_t* running;  // Ising (E_b, M); Potts (E, counts[q])
  void* scratch;
  size_t scratch_bytes;
};

struct critmc_batch {
  struct Sub {
    int64_t ticket;
    critmc_chain* c;
    double beta;
    std::vector<int64_t> sched;
    int n_meas;
    int64_t *e_out, *m_out, *aux_out;
    double* f64_out;
  };
  std::vector<Sub> pending;
  int64_t next_ticket = 1;
  int device = -1;  // device of the first submitted chain; every chain of a batch lives there
  void* buffer = nullptr;
  size_t buffer_bytes = 0;
};

namespace {

long long n_sites(const critmc_chain& c) { return (long long)c.lx * c.ly * c.lz; }
int rows(const critmc_chain& c) { return c.ly * c.lz; }

long long site(const critmc_chain& c, int x, int y, int z) { return x + (long long)c.lx * (y + (long long)c.ly * z); }

// ---- layout conversion (host) --------------------------------------------
void pack(const critmc_chain& c, const void* state, std::vector<unsigned char>& out) {
  out.assign(c.lattice_bytes, 0);
  const int hx = c.lx / 2, R = rows(c);
  for (int col = 0; col < 2; ++col)
    for (int r = 0; r < R; ++r) {
      const int y = r % c.ly, z = r / c.ly, p = (col + y + z) & 1;
      for (int i = 0; i < hx; ++i) {
        const long long s = site(c, 2 * i + p, y, z);
        const size_t slot = ((size_t)col * R + r) * hx + i;
        if (c.layout == LAYOUT_MSC) {
          if (static_cast<const int8_t*>(state)[s] > 0) {
            uint32_t* w = reinterpret_cast<uint32_t*>(out.data());
            w[((size_t)col * R + r) * (hx / 32) + i / 32] |= 1u << (i % 32);
          }
        } else if (c.layout == LAYOUT_BYTE) {
          reinterpret_cast<int8_t*>(out.data())[slot] = static_cast<const int8_t*>(state)[s];
        } else {
          float* f = reinterpret_cast<float*>(out.data());
          const size_t per = 2 * (size_t)R * hx;
          for (int k = 0; k < c.q_or_n; ++k)
            f[k * per + slot] = (float)static_cast<const double*>(state)[s * c.q_or_n + k];
        }
      }
    }
}

void unpack(const critmc_chain& c, const std::vector<unsigned char>& in, void* state) {
  const int hx = c.lx / 2, R = rows(c);
  for (int col = 0; col < 2; ++col)
    for (int r = 0; r < R; ++r) {
      const int y = r % c.ly, z = r / c.ly, p = (col + y + z) & 1;
      for (int i = 0; i < hx; ++i) {
        const long long s = site(c, 2 * i + p, y, z);
        const size_t slot = ((size_t)col * R + r) * hx + i;
        if (c.layout == LAYOUT_MSC) {
          const uint32_t* w = reinterpret_cast<const uint32_t*>(in.data());
          const uint32_t bit = (w[((size_t)col * R + r) * (hx / 32) + i / 32] >> (i % 32)) & 1u;
          static_cast<int8_t*>(state)[s] = bit ? 1 : -1;
        } else if (c.layout == LAYOUT_BYTE) {
          static_cast<int8_t*>(state)[s] = reinterpret_cast<const int8_t*>(in.data())[slot];
        } else {
          const float* f = reinterpret_cast<const float*>(in.data());
          const size_t per = 2 * (size_t)R * hx;
          for (int k = 0; k < c.q_or_n; ++k)
            static_cast<double*>(state)[s * c.q_or_n + k] = f[k * per + slot];
        }
      }
    }
}

// running sums of a host state: Ising (E_b, M), Potts (E, counts[q])
void host_sums(const critmc_chain& c, const void* state, std::vector<int64_t>& out) {
  const int8_t* s = static_cast<const int8_t*>(state);
  int64_t e = 0, m = 0;
  std::vector<int64_t> counts(c.kind == CRITMC_MODEL_POTTS ? c.q_or_n : 0, 0);
  for (int z = 0; z < c.lz; ++z)
    for (int y = 0; y < c.ly; ++y)
      for (int x = 0; x < c.lx; ++x) {
        const int8_t v = s[site(c, x, y, z)];
        int8_t nb[3];
        nb[0] = s[site(c, (x + 1) % c.lx, y, z)];
        nb[1] = s[site(c, x, (y + 1) % c.ly, z)];
        nb[2] = s[site(c, x, y, (z + 1) % c.lz)];
        for (int a = 0; a < c.dim; ++a) e -= (c.kind == CRITMC_MODEL_ISING) ? (int64_t)v * nb[a] : (v == nb[a]);
        if (c.kind == CRITMC_MODEL_ISING) m += v;
        else ++counts[v];
      }
  out.clear();
  out.push_back(e);
  if (c.kind == CRITMC_MODEL_ISING) out.push_back(m);
  else out.insert(out.end(), counts.begin(), counts.end());
}

int check_state(const critmc_chain& c, const void* state) {
  if (!state) return fail(CRITMC_ERR_INVALID, "null state");
  const long long n = n_sites(c);
  if (c.kind == CRITMC_MODEL_ISING) {
    for (long long i = 0; i < n; ++i) {
      const int8_t v = static_cast<const int8_t*>(state)[i];
      if (v != 1 && v != -1) return fail(CRITMC_ERR_INVALID, "Ising spins must be +1 or -1");
    }
  } else if (c.kind == CRITMC_MODEL_POTTS) {
    for (long long i = 0; i < n; ++i) {
      const int8_t v = static_cast<const int8_t*>(state)[i];
      if (v < 0 || v >= c.q_or_n) return fail(CRITMC_ERR_INVALID, "Potts states must be in [0, q)");
    }
  } else {
    for (long long i = 0; i < n * c.q_or_n; ++i)
      if (!std::isfinite(static_cast<const double*>(state)[i])) return fail(CRITMC_ERR_INVALID, "O(n) spins must be finite");
  }
  return CRITMC_OK;
}

// Upload a host state (critmc order) and reset the running sums.
int upload(critmc_chain& c, const void* state, void* stream) {
  std::vector<unsigned char> img;
  pack(c, state, img);
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(c.lattice, img.data(), img.size(), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return cuda_fail("copy state");
  if (c.running) {
    std::vector<int64_t> sums;
    host_sums(c, state, sums);
    if (cudaMemcpyAsync(c.running, sums.data(), sums.size() * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return cuda_fail("copy sums");
  }
  // the pageable sources must stay alive until the copies have read them
  if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_fail("synchronize");
  return CRITMC_OK;
}

// Random start from the chain's key: site i (critmc order) takes
// Philox(i, 1, TAG_INIT | 0x100, 0); the multi-spin-coded layout draws on the device.
void random_state(const critmc_chain& c, std::vector<unsigned char>& state) {
  const long long n = n_sites(c);
  state.assign(c.kind == CRITMC_MODEL_ON ? n * c.q_or_n * 8 : n, 0);
  for (long long i = 0; i < n; ++i) {
    const critmc_u32x4 r = critmc_philox4x32((uint32_t)i, 1u, CRITMC_TAG_INIT | 0x100u, (uint32_t)(i >> 32),
                                             c.key[0], c.key[1]);
    if (c.kind == CRITMC_MODEL_ISING) {
      reinterpret_cast<int8_t*>(state.data())[i] = (r.v[0] >> 31) ? 1 : -1;
    } else if (c.kind == CRITMC_MODEL_POTTS) {
      reinterpret_cast<int8_t*>(state.data())[i] = (int8_t)(((uint64_t)r.v[0] * (uint64_t)c.q_or_n) >> 32);
    } else {
      double g[4];
      for (int k = 0; k < 2; ++k) {  // Box-Muller pairs from words (2k, 2k+1)
        const double u1 = ((double)r.v[2 * k] + 1.0) * 0x1p-32, u2 = (double)r.v[2 * k + 1] * 0x1p-32;
        const double rad = std::sqrt(-2.0 * std::log(u1));
        g[2 * k] = rad * std::cos(2.0 * M_PI * u2);
        g[2 * k + 1] = rad * std::sin(2.0 * M_PI * u2);
      }
      double nrm = 0.0;
      for (int k = 0; k < c.q_or_n; ++k) nrm += g[k] * g[k];
      nrm = std::sqrt(nrm);
      for (int k = 0; k < c.q_or_n; ++k) reinterpret_cast<double*>(state.data())[i * c.q_or_n + k] = g[k] / nrm;
    }
  }
}

int ising_tables(const critmc_chain& c, double beta, uint32_t* tables) {
  for (int slot = 0; slot < 2; ++slot) {
    int st = critmc_ising_class_table(slot ? CRITMC_HEATBATH : CRITMC_METROPOLIS, 2 * c.dim, beta, c.h,
                                      tables + slot * 32, tables + slot * 32 + 16, nullptr);
    if (st) return st;
  }
  return CRITMC_OK;
}

int grow(void** p, size_t* have, size_t need, cudaStream_t s) {
  if (*have >= need) return CRITMC_OK;
  if (*p && cudaFreeAsync(*p, s) != cudaSuccess) return cuda_fail("free");
  *p = nullptr;
  *have = 0;
  if (cudaMallocAsync(p, need, s) != cudaSuccess) return cuda_fail("allocate");
  *have = need;
  return CRITMC_OK;
}

long long sweeps_of(const int64_t* sched, int n_rows) {
  long long t = 0;
  for (int r = 0; r < n_rows; ++r) t += sched[2 * r + 1];
  return t;
}

}  // namespace

extern "C" int32_t critmc_chain_create(int32_t model_kind, const int32_t dims[3], int32_t q_or_n, double h,
                                       uint32_t seed_lo, uint32_t seed_hi, uint64_t chain_id, int32_t start,
                                       const void* init_state, critmc_chain** handle) {
  clear_error();
  if (!dims || !handle) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  *handle = nullptr;
  if (model_kind < CRITMC_MODEL_ISING || model_kind > CRITMC_MODEL_ON) return fail(CRITMC_ERR_INVALID, "unknown model kind");
  if (start < CRITMC_START_RANDOM || start > CRITMC_START_STATE) return fail(CRITMC_ERR_INVALID, "unknown start");
  if (!std::isfinite(h)) return fail(CRITMC_ERR_INVALID, "h must be finite");
  critmc_chain c{};
  c.kind = model_kind;
  c.dim = dims[1] > 0 ? (dims[2] > 0 ? 3 : 2) : 1;
  c.lx = dims[0];
  c.ly = c.dim >= 2 ? dims[1] : 1;
  c.lz = c.dim >= 3 ? dims[2] : 1;
  c.q_or_n = model_kind == CRITMC_MODEL_ISING ? 2 : q_or_n;
  c.h = model_kind == CRITMC_MODEL_ISING ? h : 0.0;
  c.step = 1.0f;
  if (c.lx < 2 || c.lx % 2 || (c.dim >= 2 && (c.ly < 2 || c.ly % 2)) || (c.dim == 3 && (c.lz < 2 || c.lz % 2)))
    return fail(CRITMC_ERR_UNSUPPORTED, "checkerboard sweeps need every extent even and >= 2");
  if (n_sites(c) >= (1LL << 30)) return fail(CRITMC_ERR_UNSUPPORTED, "lattice too large");
  if (model_kind == CRITMC_MODEL_POTTS && (q_or_n < 2 || q_or_n > 127)) return fail(CRITMC_ERR_INVALID, "need 2 <= q <= 127");
  if (model_kind == CRITMC_MODEL_ON && q_or_n != 2 && q_or_n != 3) return fail(CRITMC_ERR_UNSUPPORTED, "O(n) handles n = 2 and n = 3");
  const int wc = c.lx / 64;
  const bool msc = model_kind == CRITMC_MODEL_ISING && c.dim >= 2 && c.lx % 64 == 0 && (wc & (wc - 1)) == 0;
  c.layout = model_kind == CRITMC_MODEL_ON ? LAYOUT_ON : (msc ? LAYOUT_MSC : LAYOUT_BYTE);
  c.lattice_bytes = c.layout == LAYOUT_MSC ? (size_t)n_sites(c) / 8
                    : c.layout == LAYOUT_BYTE ? (size_t)n_sites(c)
                                              : (size_t)n_sites(c) * c.q_or_n * 4;
  // Philox key of the chain: words 0, 1 of Philox(chain_id, 0, TAG_INIT | 0x200, chain_id >> 32) under the seed
  const critmc_u32x4 k = critmc_philox4x32((uint32_t)chain_id, 0u, CRITMC_TAG_INIT | 0x200u,
                                           (uint32_t)(chain_id >> 32), seed_lo, seed_hi);
  c.key[0] = k.v[0];
  c.key[1] = k.v[1];
  if (start == CRITMC_START_STATE) {
    int st = check_state(c, init_state);
    if (st) return st;
  }
  if (cudaGetDevice(&c.device) != cudaSuccess) return cuda_fail("device");
  if (cudaMalloc(&c.lattice, c.lattice_bytes) != cudaSuccess) return cuda_fail("allocate lattice");
  if (model_kind != CRITMC_MODEL_ON) {
    const size_t rb = 8 * (size_t)(model_kind == CRITMC_MODEL_ISING ? 2 : 1 + c.q_or_n);
    if (cudaMalloc(&c.running, rb) != cudaSuccess) {
      cudaFree(c.lattice);
      return cuda_fail("allocate running sums");
    }
  }
  critmc_chain* out = new critmc_chain(c);
  int st = CRITMC_OK;
  if (start == CRITMC_START_STATE) {
    st = upload(*out, init_state, nullptr);
  } else if (c.layout == LAYOUT_MSC) {
    uint32_t* dkey = nullptr;
    if (cudaMalloc(&dkey, 8) != cudaSuccess || cudaMemcpy(dkey, c.key, 8, cudaMemcpyHostToDevice) != cudaSuccess) {
      st = cuda_fail("key");
    } else {
      st = critmc_ising_msc_init((uint32_t*)c.lattice, c.dim, c.lx, c.ly, c.lz, 1, dkey,
                                 start == CRITMC_START_RANDOM ? 0 : 1, nullptr);
      if (!st) st = critmc_ising_msc_measure((uint32_t*)c.lattice, c.dim, c.lx, c.ly, c.lz, 1, c.running, nullptr);
      if (!st && cudaDeviceSynchronize() != cudaSuccess) st = cuda_fail("synchronize");
    }
    if (dkey) cudaFree(dkey);
  } else {
    std::vector<unsigned char> state;
    if (start == CRITMC_START_RANDOM) {
      random_state(c, state);
    } else {
      state.assign(c.kind == CRITMC_MODEL_ON ? n_sites(c) * c.q_or_n * 8 : n_sites(c), 0);
      for (long long i = 0; i < n_sites(c); ++i) {
        if (c.kind == CRITMC_MODEL_ISING) state[i] = 1;
        else if (c.kind == CRITMC_MODEL_ON) reinterpret_cast<double*>(state.data())[i * c.q_or_n] = 1.0;
      }
    }
    st = upload(*out, state.data(), nullptr);
  }
  if (st) {
    critmc_chain_destroy(out);
    return st;
  }
  *handle = out;
  return CRITMC_OK;
}

extern "C" int32_t critmc_chain_destroy(critmc_chain* c) {
  if (!c) return CRITMC_OK;
  DeviceScope ds(c->device);
  cudaDeviceSynchronize();  // no work of this chain may still be in flight
  if (c->lattice) cudaFree(c->lattice);
  if (c->running) cudaFree(c->running);
  if (c->scratch) cudaFree(c->scratch);
  delete c;
  return CRITMC_OK;
}

extern "C" int32_t critmc_chain_info(const critmc_chain* c, int32_t* layout, uint32_t* sweep, uint32_t key[2]) {
  clear_error();
  if (!c) return fail(CRITMC_ERR_INVALID, "null chain");
  if (layout) *layout = c->layout;
  if (sweep) *sweep = c->sweep;
  if (key) {
    key[0] = c->key[0];
    key[1] = c->key[1];
  }
  return CRITMC_OK;
}

extern "C" int32_t critmc_chain_set_step(critmc_chain* c, double step) {
  clear_error();
  if (!c || !std::isfinite(step) || step <= 0.0) return fail(CRITMC_ERR_INVALID, "need a chain and step > 0");
  c->step = (float)step;
  return CRITMC_OK;
}

extern "C" int32_t critmc_get_state(critmc_chain* c, void* host_out, int64_t* running_out, void* stream) {
  clear_error();
  if (!c || !host_out) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  DeviceScope ds(c->device);
  if (ds.status) return ds.status;
  std::vector<unsigned char> img(c->lattice_bytes);
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(img.data(), c->lattice, img.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return cuda_fail("copy state");
  if (running_out && c->running) {
    const size_t rb = 8 * (size_t)(c->kind == CRITMC_MODEL_ISING ? 2 : 1 + c->q_or_n);
    if (cudaMemcpyAsync(running_out, c->running, rb, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return cuda_fail("copy sums");
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_fail("synchronize");
  unpack(*c, img, host_out);
  return CRITMC_OK;
}

extern "C" int32_t critmc_set_state(critmc_chain* c, const void* host_in, void* stream) {
  clear_error();
  if (!c) return fail(CRITMC_ERR_INVALID, "null chain");
  int st = check_state(*c, host_in);
  if (st) return st;
  DeviceScope ds(c->device);
  if (ds.status) return ds.status;
  return upload(*c, host_in, stream);
}

extern "C" int32_t critmc_advance(critmc_chain* c, double beta, const int64_t* schedule, int32_t n_rows,
                                  int32_t n_meas, int64_t* e_out, int64_t* m_out, int64_t* aux_out,
                                  double* f64_out, void* stream) {
  clear_error();
  if (!c || !schedule || !aux_out) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_meas < 0) return fail(CRITMC_ERR_INVALID, "n_meas must not be negative");
  DeviceScope ds(c->device);
  if (ds.status) return ds.status;
  const long long per = sweeps_of(schedule, n_rows);
  int st = CRITMC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (c->kind == CRITMC_MODEL_ISING) {
    if (!e_out || !m_out) return fail(CRITMC_ERR_INVALID, "Ising chains need e_out and m_out");
    uint32_t tables[64];
    if ((st = ising_tables(*c, beta, tables))) return st;
    if (c->layout == LAYOUT_MSC) {
      const int64_t need = critmc_ising_msc_scratch_bytes(1, std::max(n_meas, 1));
      if ((st = grow(&c->scratch, &c->scratch_bytes, (size_t)need, s))) return st;
      st = critmc_ising_msc_run((uint32_t*)c->lattice, c->dim, c->lx, c->ly, c->lz, 1, c->key, tables, 1, c->sweep,
                                schedule, n_rows, n_meas, c->running, e_out, m_out, aux_out, c->scratch, 0, 8, stream);
    } else {
      st = critmc_ising_byte_run((int8_t*)c->lattice, c->dim, c->lx, c->ly, c->lz, 1, c->key, tables, 1, c->sweep,
                                 schedule, n_rows, n_meas, c->running, e_out, m_out, aux_out, stream);
    }
  } else if (c->kind == CRITMC_MODEL_POTTS) {
    if (!e_out || !m_out) return fail(CRITMC_ERR_INVALID, "Potts chains need e_out and m_out (counts)");
    st = critmc_potts_run((int8_t*)c->lattice, c->dim, c->lx, c->ly, c->lz, c->q_or_n, 1, c->key, &beta, 1, c->sweep,
                          schedule, n_rows, n_meas, c->running, c->running + 1, e_out, m_out, aux_out, stream);
  } else {
    if (!f64_out) return fail(CRITMC_ERR_INVALID, "O(n) chains need f64_out");
    const double step = c->step;
    double* e = f64_out;
    double* m = e + n_meas;
    double* sc = m + (size_t)n_meas * c->q_or_n;
    double* ss = sc + (size_t)n_meas * c->dim;
    st = critmc_on_run((float*)c->lattice, c->dim, c->lx, c->ly, c->lz, c->q_or_n, 1, c->key, &beta, &step, 1,
                       c->sweep, schedule, n_rows, n_meas, e, m, sc, ss, aux_out, stream);
  }
  if (st) return st;
  c->sweep += (uint32_t)(per * n_meas);
  return CRITMC_OK;
}

// ---- batch queue -----------------------------------------------------------

extern "C" int32_t critmc_batch_create(critmc_batch** b) {
  clear_error();
  if (!b) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  *b = new critmc_batch();
  return CRITMC_OK;
}

extern "C" int32_t critmc_batch_destroy(critmc_batch* b) {
  if (!b) return CRITMC_OK;
  if (b->buffer) {
    DeviceScope ds(b->device);
    cudaDeviceSynchronize();
    cudaFree(b->buffer);
  }
  delete b;
  return CRITMC_OK;
}

extern "C" int32_t critmc_batch_submit(critmc_batch* b, critmc_chain* c, double beta, const int64_t* schedule,
                                       int32_t n_rows, int32_t n_meas, int64_t* e_out, int64_t* m_out,
                                       int64_t* aux_out, double* f64_out, int64_t* ticket) {
  clear_error();
  if (!b || !c || !schedule || !ticket || !aux_out) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (n_rows < 1 || n_rows > 8 || n_meas < 0) return fail(CRITMC_ERR_INVALID, "need 1..8 schedule rows and n_meas >= 0");
  if (!std::isfinite(beta)) return fail(CRITMC_ERR_INVALID, "beta must be finite");
  if (c->kind != CRITMC_MODEL_ON && (!e_out || !m_out)) return fail(CRITMC_ERR_INVALID, "missing e_out or m_out");
  if (c->kind == CRITMC_MODEL_ON && !f64_out) return fail(CRITMC_ERR_INVALID, "O(n) chains need f64_out");
  if (b->device >= 0 && c->device != b->device)
    return fail(CRITMC_ERR_INVALID, "every chain of a batch must live on the device of its first chain");
  b->device = c->device;
  critmc_batch::Sub sub;
  sub.ticket = b->next_ticket++;
  sub.c = c;
  sub.beta = beta;
  sub.sched.assign(schedule, schedule + 2 * n_rows);
  sub.n_meas = n_meas;
  sub.e_out = e_out;
  sub.m_out = m_out;
  sub.aux_out = aux_out;
  sub.f64_out = f64_out;
  b->pending.push_back(std::move(sub));
  *ticket = b->pending.back().ticket;
  return CRITMC_OK;
}

extern "C" int32_t critmc_batch_cancel(critmc_batch* b, int64_t ticket) {
  clear_error();
  if (!b) return fail(CRITMC_ERR_INVALID, "null batch");
  for (size_t i = 0; i < b->pending.size(); ++i)
    if (b->pending[i].ticket == ticket) {
      b->pending.erase(b->pending.begin() + (long)i);
      return CRITMC_OK;
    }
  return fail(CRITMC_ERR_INVALID, "ticket is not pending");
}

namespace {

// one chain's submission as a work item, or false if it needs the per-model path
bool as_item(const critmc_batch::Sub& u, critmc_item& it, int& st) {
  const critmc_chain& c = *u.c;
  st = CRITMC_OK;
  if (u.sched.size() / 2 > 4) return false;
  if (c.layout == LAYOUT_MSC && c.lattice_bytes > 128 * 1024) return false;  // items hold <= 2^20 MSC sites
  std::memset(&it, 0, sizeof(it));
  it.spins = c.lattice;
  it.kind = c.layout == LAYOUT_MSC ? CRITMC_ITEM_MSC_ISING
            : c.kind == CRITMC_MODEL_ISING ? CRITMC_ITEM_BYTE_ISING
            : c.kind == CRITMC_MODEL_POTTS ? CRITMC_ITEM_POTTS
                                           : CRITMC_ITEM_ON;
  it.dim = c.dim;
  it.lx = c.lx;
  it.ly = c.ly;
  it.lz = c.lz;
  it.q_or_n = c.kind == CRITMC_MODEL_ISING ? 0 : c.q_or_n;
  it.key[0] = c.key[0];
  it.key[1] = c.key[1];
  it.sweep0 = c.sweep;
  it.n_meas = u.n_meas;
  it.n_rows = (int)(u.sched.size() / 2);
  for (int r = 0; r < it.n_rows; ++r) {
    it.codes[r] = (int)u.sched[2 * r];
    it.reps[r] = (int)u.sched[2 * r + 1];
  }
  it.aux_out = u.aux_out;
  if (c.kind == CRITMC_MODEL_ON) {
    double* e = u.f64_out;
    it.e_out = e;
    it.vec_out = e + u.n_meas;
    it.sc_out = e + u.n_meas + (size_t)u.n_meas * c.q_or_n;
    it.ss_out = it.sc_out + (size_t)u.n_meas * c.dim;
  } else {
    it.e_out = u.e_out;
    it.vec_out = u.m_out;
    it.running = c.running;
    if (c.kind == CRITMC_MODEL_POTTS) it.counts = c.running + 1;
  }
  st = critmc_item_prepare(&it, u.beta, c.h, c.step);
  return st == CRITMC_OK;
}

}  // namespace

extern "C" int32_t critmc_batch_poll(critmc_batch* b, void* stream, int64_t* done, int32_t max_done,
                                     int32_t* n_done) {
  clear_error();
  if (!b || !n_done || (max_done > 0 && !done)) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  *n_done = 0;
  cudaStream_t s = (cudaStream_t)stream;
  if (b->pending.empty()) {
    if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_fail("synchronize");
    return CRITMC_OK;
  }
  DeviceScope ds(b->device);
  if (ds.status) return ds.status;
  // rounds: each takes the first pending submission of every chain (FIFO per chain)
  while (!b->pending.empty() && *n_done < max_done) {
    std::vector<size_t> take;
    std::vector<const critmc_chain*> seen;
    for (size_t i = 0; i < b->pending.size() && (int)(*n_done + take.size()) < max_done; ++i) {
      const critmc_chain* c = b->pending[i].c;
      if (std::find(seen.begin(), seen.end(), c) != seen.end()) {
        seen.push_back(c);  // later submissions of a chain wait for a later round
        continue;
      }
      seen.push_back(c);
      take.push_back(i);
    }
    std::vector<critmc_item> items;
    for (size_t i : take) {
      critmc_batch::Sub& u = b->pending[i];
      critmc_item it;
      int st;
      if (as_item(u, it, st)) {
        items.push_back(it);
      } else {
        if (st) return st;
        if ((st = critmc_advance(u.c, u.beta, u.sched.data(), (int)(u.sched.size() / 2), u.n_meas, u.e_out, u.m_out,
                                 u.aux_out, u.f64_out, stream)))
          return st;
        u.c = nullptr;  // advanced: its sweep counter already moved
      }
    }
    if (!items.empty()) {
      const int64_t need = critmc_items_buffer_bytes((int32_t)items.size());
      int st = grow(&b->buffer, &b->buffer_bytes, (size_t)need, s);
      if (st) return st;
      if ((st = critmc_run_items(items.data(), (int32_t)items.size(), b->buffer, (int64_t)b->buffer_bytes, nullptr, 0,
                                 stream)))
        return st;
    }
    std::vector<critmc_batch::Sub> rest;
    for (size_t i = 0, t = 0; i < b->pending.size(); ++i) {
      if (t < take.size() && take[t] == i) {
        critmc_batch::Sub& u = b->pending[i];
        if (u.c) u.c->sweep += (uint32_t)(sweeps_of(u.sched.data(), (int)(u.sched.size() / 2)) * u.n_meas);
        done[(*n_done)++] = u.ticket;
        ++t;
      } else {
        rest.push_back(std::move(b->pending[i]));
      }
    }
    b->pending.swap(rest);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_fail("synchronize");
  return CRITMC_OK;
}

extern "C" int32_t critmc_batch_pending(const critmc_batch* b) { return b ? (int32_t)b->pending.size() : 0; }
