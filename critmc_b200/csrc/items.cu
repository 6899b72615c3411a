// Host side of the work-item ABI: table preparation, validation, grouping by
// model family and the per-family persistent launches.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "geom.cuh"
#include "host_common.h"
#include "items_host.h"
#include "msc_ising_host.h"

using namespace critmc;

namespace {

constexpr size_t ITEMS_HEADER = 256;  // queue counters of the launch groups
constexpr int ITEMS_SMEM_DEFAULT = 200 * 1024;

int family_of(int kind) {
  switch (kind) {
    case CRITMC_ITEM_MSC_ISING: return 0;
    case CRITMC_ITEM_BYTE_ISING:
    case CRITMC_ITEM_POTTS: return 1;
    case CRITMC_ITEM_ON: return 2;
    default: return -1;
  }
}

// Kernel groups: 0 multi-spin-coded Ising, 1 byte lattices, 2..7 O(n) by
// (n, dim) (a kernel per variant).  Launch groups: kernel group x team size,
// one persistent kernel each.
constexpr int N_KGROUPS = 8;
constexpr int N_TEAMS = 5;  // 1, 2, 4, 8, 16 blocks per item
constexpr int N_GROUPS = N_KGROUPS * N_TEAMS;
static_assert(N_GROUPS * sizeof(unsigned) <= ITEMS_HEADER, "queue counters");
int team_slot(int team) {
  switch (team) {
    case 0:
    case 1: return 0;
    case 2: return 1;
    case 4: return 2;
    case 8: return 3;
    case 16: return 4;
    default: return -1;
  }
}
int group_of(const critmc_item& it) {
  const int fam = family_of(it.kind);
  const int kg = fam < 2 ? fam : 2 + (it.q_or_n - 2) * 3 + (it.dim - 1);
  return kg * N_TEAMS + team_slot(it.team);
}

int check_schedule(const critmc_item& it) {
  if (it.n_rows < 1 || it.n_rows > 4) return fail(CRITMC_ERR_INVALID, "items take 1..4 schedule rows");
  for (int r = 0; r < it.n_rows; ++r) {
    const int c = it.codes[r];
    const bool ok = c == CRITMC_METROPOLIS || c == CRITMC_HEATBATH ||
                    (c == CRITMC_OVERRELAX && it.kind == CRITMC_ITEM_ON);
    if (!ok) return fail(CRITMC_ERR_UNSUPPORTED, "unsupported update code in an item schedule");
    if (it.reps[r] < 1 || it.reps[r] > (1 << 20)) return fail(CRITMC_ERR_INVALID, "item repetitions must be in [1, 2^20]");
  }
  return CRITMC_OK;
}

int check_item(const critmc_item& it) {
  const int fam = family_of(it.kind);
  if (fam < 0) return fail(CRITMC_ERR_INVALID, "unknown item kind");
  if (team_slot(it.team) < 0) return fail(CRITMC_ERR_INVALID, "item team must be 0, 1, 2, 4, 8 or 16 blocks");
  if (!it.spins || !it.e_out || !it.vec_out || !it.aux_out) return fail(CRITMC_ERR_INVALID, "item with a null pointer");
  if (it.n_meas < 0) return fail(CRITMC_ERR_INVALID, "item n_meas must not be negative");
  int st = check_schedule(it);
  if (st) return st;
  long long per = 0;
  for (int r = 0; r < it.n_rows; ++r) per += it.reps[r];
  if ((long long)it.sweep0 + per * it.n_meas > 0xFFFFFFFFLL) return fail(CRITMC_ERR_INVALID, "item sweep counter would pass 2^32");
  if (fam == 0) {
    MscGeom g;
    if ((st = msc_geom(it.dim, it.lx, it.ly, it.lz, g))) return st;
    if (it.team <= 1 && 2 * (size_t)g.words * 4 > 128 * 1024)
      return fail(CRITMC_ERR_UNSUPPORTED, "one-block MSC items hold at most 2^20 sites (128 KiB)");
    if (!it.running) return fail(CRITMC_ERR_INVALID, "item with a null pointer");
  } else {
    ByteGeom g;
    if ((st = byte_geom(it.dim, it.lx, it.ly, it.lz, g))) return st;
    if (fam == 1 && !it.running) return fail(CRITMC_ERR_INVALID, "item with a null pointer");
    if (it.kind == CRITMC_ITEM_POTTS && (it.q_or_n < 2 || it.q_or_n > 127 || !it.counts))
      return fail(CRITMC_ERR_INVALID, "Potts items need 2 <= q <= 127 and counts");
    if (fam == 2 && ((it.q_or_n != 2 && it.q_or_n != 3) || !it.sc_out || !it.ss_out))
      return fail(CRITMC_ERR_INVALID, "O(n) items need n = 2 or 3 and stiffness outputs");
  }
  return CRITMC_OK;
}

size_t item_smem(const critmc_item& it, int fam, size_t limit) {
  if (it.team > 1) return 0;  // teams update the lattice in global memory
  if (fam == 0) {
    MscGeom g;
    msc_geom(it.dim, it.lx, it.ly, it.lz, g);
    return 2 * (size_t)g.words * 4;
  }
  if (fam >= 2) fam = 2;
  ByteGeom g;
  byte_geom(it.dim, it.lx, it.ly, it.lz, g);
  const size_t need = fam == 1 ? 2 * (size_t)g.slots : (size_t)it.q_or_n * 2 * g.slots * 4;
  return need <= limit ? need : 0;  // larger lattices are updated in HBM
}

}  // namespace

extern "C" int32_t critmc_item_prepare(critmc_item* it, double beta, double h, double step) {
  clear_error();
  if (!it) return fail(CRITMC_ERR_INVALID, "null item");
  const int fam = family_of(it->kind);
  if (fam < 0) return fail(CRITMC_ERR_INVALID, "unknown item kind");
  int st = check_schedule(*it);
  if (st) return st;
  const int z = 2 * it->dim;
  if (it->kind == CRITMC_ITEM_MSC_ISING || it->kind == CRITMC_ITEM_BYTE_ISING) {
    for (int slot = 0; slot < 2; ++slot) {
      const int algo = slot ? CRITMC_HEATBATH : CRITMC_METROPOLIS;
      if ((st = critmc_ising_class_table(algo, z, beta, h, it->kind_tab[slot], it->thr_tab[slot], nullptr))) return st;
      it->rule[slot] = msc_pick_rule(it->kind_tab[slot], it->thr_tab[slot], z, algo, 1);
    }
  } else if (it->kind == CRITMC_ITEM_POTTS) {
    if ((st = critmc_potts_tables(z, beta, it->boltz, it->weight))) return st;
  } else {
    if (!std::isfinite(beta) || !std::isfinite(step)) return fail(CRITMC_ERR_INVALID, "beta and step must be finite");
    it->beta = (float)beta;
    it->step = (float)step;
  }
  return CRITMC_OK;
}

extern "C" int32_t critmc_items_team_clusters(int32_t kind, int32_t q_or_n, int32_t dim, int32_t team) {
  clear_error();
  const int fam = family_of(kind);
  if (fam < 0) return fail(CRITMC_ERR_INVALID, "unknown item kind");
  if (team != 2 && team != 4 && team != 8 && team != 16) return fail(CRITMC_ERR_INVALID, "team size must be 2, 4, 8 or 16");
  if (fam == 0) return msc_items_team_clusters(team);
  if (fam == 1) return byte_items_team_clusters(team);
  return on_items_team_clusters(q_or_n, dim, team);
}

extern "C" int64_t critmc_items_buffer_bytes(int32_t n_items) {
  return (int64_t)ITEMS_HEADER + (int64_t)n_items * (int64_t)sizeof(critmc_item);
}

namespace {

// Library-owned streams on which the three family kernels of one call run
// side by side (fork from and join into the caller's stream).  The enqueue
// sequence is serialised per process so the fork/join events are never
// re-recorded while a wait on them is being enqueued.
struct FamilyStreams {
  cudaStream_t aux[N_GROUPS] = {};
  cudaEvent_t fork = nullptr, join[N_GROUPS] = {};
};
std::mutex g_family_mutex;
FamilyStreams g_family[64];

// the fork event and, made on first use, the streams of the launch groups in `used`
int family_streams(int dev, const int (&used)[N_GROUPS], FamilyStreams*& out) {
  if (dev < 0 || dev >= 64) return fail(CRITMC_ERR_UNSUPPORTED, "device ordinal above 63");
  FamilyStreams& f = g_family[dev];
  if (!f.fork && cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming) != cudaSuccess) return cuda_fail("event");
  for (int k = 0; k < N_GROUPS; ++k) {
    if (!used[k] || f.aux[k]) continue;
    if (cudaStreamCreateWithFlags(&f.aux[k], cudaStreamNonBlocking) != cudaSuccess) return cuda_fail("stream");
    if (cudaEventCreateWithFlags(&f.join[k], cudaEventDisableTiming) != cudaSuccess) return cuda_fail("event");
  }
  out = &f;
  return CRITMC_OK;
}

}  // namespace

extern "C" int32_t critmc_run_items(const critmc_item* items, int32_t n_items, void* buffer,
                                    int64_t buffer_bytes, void* staging, int32_t smem_limit,
                                    void* stream) {
  return critmc_run_items_ctl(items, n_items, buffer, buffer_bytes, staging, smem_limit, nullptr, stream);
}

extern "C" int32_t critmc_run_items_ctl(const critmc_item* items, int32_t n_items, void* buffer,
                                        int64_t buffer_bytes, void* staging, int32_t smem_limit,
                                        critmc_control* ctl, void* stream) {
  clear_error();
  const RunCtl rc = control_device(ctl);
  if (n_items < 0) return fail(CRITMC_ERR_INVALID, "n_items must not be negative");
  if (n_items == 0) return CRITMC_OK;
  if (!items || !buffer) return fail(CRITMC_ERR_INVALID, "null pointer argument");
  if (buffer_bytes < critmc_items_buffer_bytes(n_items)) return fail(CRITMC_ERR_INVALID, "item buffer too small");
  const size_t limit = smem_limit > 0 ? (size_t)smem_limit : (size_t)ITEMS_SMEM_DEFAULT;
  if (limit > 220 * 1024) return fail(CRITMC_ERR_INVALID, "smem_limit above 220 KiB");
  std::vector<critmc_item> own;
  critmc_item* sorted = static_cast<critmc_item*>(staging);
  if (!sorted) {
    own.resize(n_items);
    sorted = own.data();
  }
  int count[N_GROUPS] = {};
  size_t smem[N_GROUPS] = {};
  int fill = 0;
  for (int i = 0; i < n_items; ++i) {
    int st = check_item(items[i]);
    if (st) return st;
  }
  for (int f = 0; f < N_GROUPS; ++f)
    for (int i = 0; i < n_items; ++i) {
      if (group_of(items[i]) != f) continue;
      sorted[fill++] = items[i];
      ++count[f];
      smem[f] = std::max(smem[f], item_smem(items[i], family_of(items[i].kind), limit));  // per launch group
    }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return cuda_fail("device");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned* queues = (unsigned*)buffer;
  critmc_item* dev_items = (critmc_item*)((char*)buffer + ITEMS_HEADER);
  if (cudaMemsetAsync(queues, 0, ITEMS_HEADER, s) != cudaSuccess) return cuda_fail("memset");
  if (cudaMemcpyAsync(dev_items, sorted, (size_t)n_items * sizeof(critmc_item), cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return cuda_fail("copy items");
  int groups = 0;
  for (int f = 0; f < N_GROUPS; ++f) groups += count[f] > 0;
  std::unique_lock<std::mutex> lock(g_family_mutex, std::defer_lock);
  FamilyStreams* fs = nullptr;
  if (groups > 1) {
    lock.lock();
    int st = family_streams(dev, count, fs);
    if (st) return st;
    if (cudaEventRecord(fs->fork, s) != cudaSuccess) return cuda_fail("event record");
  }
  int offset = 0;
  for (int f = 0; f < N_GROUPS; ++f) {
    if (!count[f]) continue;
    cudaStream_t fstream = s;
    if (fs) {
      fstream = fs->aux[f];
      if (cudaStreamWaitEvent(fstream, fs->fork, 0) != cudaSuccess) return cuda_fail("stream wait");
    }
    int st = CRITMC_OK;
    const critmc_item* first = sorted + offset;
    const int kg = f / N_TEAMS, team = 1 << (f % N_TEAMS);
    if (kg == 0) st = msc_items_launch(dev_items + offset, count[f], queues + f, smem[f], team, rc, fstream);
    else if (kg == 1) st = byte_items_launch(dev_items + offset, count[f], queues + f, smem[f], team, rc, fstream);
    else st = on_items_launch(dev_items + offset, count[f], first->q_or_n, first->dim, queues + f, smem[f], team, rc,
                              fstream);
    if (st) return st;
    if (fs) {
      if (cudaEventRecord(fs->join[f], fstream) != cudaSuccess) return cuda_fail("event record");
      if (cudaStreamWaitEvent(s, fs->join[f], 0) != cudaSuccess) return cuda_fail("stream wait");
    }
    offset += count[f];
  }
  return CRITMC_OK;
}
