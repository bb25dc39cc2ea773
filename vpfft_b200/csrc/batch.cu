// batch.cu -- the batch engine: many RVEs (grids of different sizes) advanced
// together, one kernel launch per phase over every RVE in that phase, with
// continuous admission of new requests between ticks.
//
// A request is one increment (RunSingleStrainStep, MaterialGrid.cpp:897-1084)
// on a caller-owned grid.  Its life in the batch:
//   queued  -> admitted when a slot is free and its two spectrum buffers fit
//              the HBM budget (first-fit in one arena allocated at creation);
//   INIT    -> batched initialisation + reference medium; after the tick the
//              host forms L0, inverse(-L0) and the Newton constants exactly as
//              the single-grid path does;
//   ITER    -> the tick's fixed-point iterations (five FFT passes with the
//              Green operator, NR sweep, per-slot reductions), each kernel one
//              launch over all iterating slots; a slot whose loop has finished
//              lets its blocks return at once;
//   done    -> batched texture/hardening update, result recorded, slot and
//              arena space released.
// The per-slot block counts of the persistent kernels equal the single-grid
// launches', so every slot's sums are formed in the same order as when it is
// solved alone.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "grid.h"

using namespace vpfft;
using namespace vpfft::grid_ops;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

thread_local std::string g_batch_err;

// First-fit allocator over [0, size) with 256-byte granules (host bookkeeping
// of the device arena).
class Arena {
 public:
  explicit Arena(size_t size = 0) : size_(size) {}
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) & ~size_t(255);
    size_t pos = 0;
    for (auto it = used_.begin(); it != used_.end(); ++it) {
      if (it->first - pos >= bytes) break;
      pos = it->first + it->second;
    }
    if (pos + bytes > size_) return false;
    used_[pos] = bytes;
    in_use_ += bytes;
    *off = pos;
    return true;
  }
  void release(size_t off) {
    auto it = used_.find(off);
    if (it == used_.end()) return;
    in_use_ -= it->second;
    used_.erase(it);
  }
  size_t in_use() const { return in_use_; }
  size_t size() const { return size_; }

 private:
  size_t size_;
  size_t in_use_ = 0;
  std::map<size_t, size_t> used_;  // offset -> bytes
};

enum Phase { kInit = 0, kIter = 1, kDone = 2 };

struct Request {
  int64_t id = 0;
  vpfft_grid* g = nullptr;
  double edot[5] = {0};
  int max_iter = 100;
  double dt = 0;
  double eps = 0;
  double t_submit = 0;
  double t_admit = 0;
  bool cancelled = false;
};

struct Active {
  Request r;
  int slot = -1;
  size_t off = 0;  // arena offset of X (X2 follows)
  Phase phase = kInit;
  bool tau = false;  // per-voxel CRSS
  int fam = -1;      // tile family of the batched FFT passes
};

// Host mirror of one device block list: slots and cumulative block counts.
struct HostList {
  std::vector<int> slot, prefix{0};
  void clear() {
    slot.clear();
    prefix.assign(1, 0);
  }
  void add(int s, int blocks) {
    slot.push_back(s);
    prefix.push_back(prefix.back() + blocks);
  }
  int m() const { return (int)slot.size(); }
  int blocks() const { return prefix.back(); }
  // the common block count when every slot has the same, else 0
  int per() const {
    for (size_t i = 2; i < prefix.size(); ++i)
      if (prefix[i] - prefix[i - 1] != prefix[1]) return 0;
    return prefix.size() > 1 ? prefix[1] : 0;
  }
};

// Device copy of a set of lists, packed into one buffer, staged through a
// pinned host buffer (so the upload does not wait for the stream).
struct DeviceLists {
  int* d = nullptr;
  int* h = nullptr;
  int cap = 0;  // ints
};

}  // namespace

struct vpfft_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  vpfft_precision prec = VPFFT_PREC_MIXED;
  vpfft_material mat{};
  vpfft_solver_options opt{};
  vpfft_batch_options bopt{};
  int nexp = 0;
  // device memory
  void* arena_base = nullptr;
  Arena arena;
  void* d_desc = nullptr;     // SlotDesc<S>[max_slots]
  IterCtrl* d_ctrl = nullptr; // IterCtrl[max_slots]
  double* d_sum25 = nullptr;  // 25 per slot
  DeviceLists setup_lists, iter_lists;
  // pinned host copies
  IterCtrl* h_ctrl = nullptr;
  double* h_sum25 = nullptr;
  // bookkeeping
  unsigned char* h_desc = nullptr;  // SlotDesc<S>[max_slots] host images (pinned)
  std::vector<int> free_slots;
  std::deque<Request> queue;
  std::vector<Active> active;
  std::deque<vpfft_batch_result> results;
  int64_t next_id = 1;
  int64_t ticks = 0, graph_replays = 0, launches = 0, completed = 0, deferred = 0;
  // captured iteration chunk
  uint64_t iter_generation = 1, graph_generation = 0, eager_generation = 0;
  cudaGraphExec_t graph = nullptr;
  // the FFT pass chains of different size classes run concurrently: forked
  // from `stream` onto these streams and joined back before the NR sweep
  static constexpr int kAux = 8;
  cudaStream_t aux[kAux] = {};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kAux] = {};
  // FFT tile families: per RVE size, in order of first admission
  std::map<std::tuple<int, int, int>, int> fam_of;
  std::vector<vpfft_tile_tuning> tunings;
  cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;  // autotuner timing
  std::string err;
};

namespace {

vpfft_status bfail(vpfft_batch* b, vpfft_status s, const std::string& msg) {
  if (b)
    b->err = msg;
  else
    g_batch_err = msg;
  return s;
}

#define BCK(b, call)                                                                       \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return bfail((b), e_ == cudaErrorMemoryAllocation ? VPFFT_ERR_OUT_OF_MEMORY          \
                                                        : VPFFT_ERR_CUDA,                  \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

template <typename S>
SlotDesc<S>* host_desc(vpfft_batch* b, int slot) {
  return reinterpret_cast<SlotDesc<S>*>(b->h_desc) + slot;
}
template <typename S>
SlotDesc<S>* dev_desc(vpfft_batch* b) {
  return reinterpret_cast<SlotDesc<S>*>(b->d_desc);
}

// Uploads host lists into a device buffer; returns BatchLaunch views.
vpfft_status upload_lists(vpfft_batch* b, DeviceLists& dl, const std::vector<HostList*>& lists,
                          std::vector<BatchLaunch>& out) {
  size_t need = 0;
  for (const HostList* l : lists) need += l->slot.size() + l->prefix.size();
  if ((int)need > dl.cap) {
    BCK(b, cudaStreamSynchronize(b->stream));
    if (dl.d) cudaFree(dl.d);
    if (dl.h) cudaFreeHost(dl.h);
    dl.d = nullptr;
    dl.h = nullptr;
    dl.cap = 0;
    const int cap = (int)std::max<size_t>(need, 64) * 2;
    BCK(b, cudaMalloc(&dl.d, sizeof(int) * cap));
    BCK(b, cudaMallocHost(&dl.h, sizeof(int) * cap));
    dl.cap = cap;
  }
  size_t pos = 0;
  out.clear();
  for (const HostList* l : lists) {
    BatchLaunch bl;
    bl.slot = dl.d + pos;
    std::copy(l->slot.begin(), l->slot.end(), dl.h + pos);
    pos += l->slot.size();
    bl.prefix = dl.d + pos;
    std::copy(l->prefix.begin(), l->prefix.end(), dl.h + pos);
    pos += l->prefix.size();
    bl.m = l->m();
    bl.blocks = l->blocks();
    bl.per = l->per();
    out.push_back(bl);
  }
  if (pos)
    BCK(b, cudaMemcpyAsync(dl.d, dl.h, sizeof(int) * pos, cudaMemcpyHostToDevice, b->stream));
  return VPFFT_OK;
}

template <typename S>
vpfft_status upload_desc(vpfft_batch* b, int slot) {
  BCK(b, cudaMemcpyAsync(dev_desc<S>(b) + slot, host_desc<S>(b, slot), sizeof(SlotDesc<S>),
                         cudaMemcpyHostToDevice, b->stream));
  return VPFFT_OK;
}

vpfft_status upload_ctrl(vpfft_batch* b, int slot) {
  BCK(b, cudaMemcpyAsync(b->d_ctrl + slot, b->h_ctrl + slot, sizeof(IterCtrl),
                         cudaMemcpyHostToDevice, b->stream));
  return VPFFT_OK;
}

void release(vpfft_batch* b, Active& a) {
  b->arena.release(a.off);
  b->free_slots.push_back(a.slot);
  a.r.g->in_batch = false;
}

void record(vpfft_batch* b, const Active& a, vpfft_status st, double t_end) {
  vpfft_batch_result r{};
  r.request_id = a.r.id;
  r.status = st;
  const IterCtrl& c = b->h_ctrl[a.slot];
  if (a.phase != kInit) {
    r.iterations = c.iter;
    r.converged = (c.last[10] <= a.r.eps && c.last[11] <= a.r.eps) ? 1 : 0;
    for (int k = 0; k < 5; ++k) r.avg_stress[k] = c.last[k];
    r.stress_error = c.last[10];
    r.strain_rate_error = c.last[11];
    r.nr_not_converged = (int64_t)c.nr_capped;
    r.status_bits = c.status | (r.converged ? 0 : VPFFT_STATUS_LOOP_NOT_CONVERGED) |
                    (c.nr_capped ? VPFFT_STATUS_NR_CAPPED : 0);
  }
  r.seconds_queued = a.r.t_admit - a.r.t_submit;
  r.seconds_total = t_end - a.r.t_submit;
  b->results.push_back(r);
  b->completed++;
}

// Admission: FIFO over the queue; a request whose grid is busy waits without
// blocking the others; the first request that does not fit the budget stops
// admission for this tick.
template <typename S>
vpfft_status admit(vpfft_batch* b, std::vector<int>& admitted) {
  for (auto it = b->queue.begin(); it != b->queue.end();) {
    if (b->free_slots.empty()) break;
    vpfft_grid* g = it->g;
    if (g->in_batch) {
      ++it;
      continue;
    }
    const size_t spec = spectrum_bytes(g);
    const size_t spec_al = (spec + 255) & ~size_t(255);
    size_t off = 0;
    if (!b->arena.alloc(2 * spec_al, &off)) {
      b->deferred++;
      break;
    }
    Active a;
    a.r = *it;
    a.r.t_admit = now_s();
    a.off = off;
    a.slot = b->free_slots.back();
    b->free_slots.pop_back();
    a.phase = kInit;
    g->in_batch = true;
    if (vpfft_status s = ensure_hist(g, a.r.max_iter)) {
      release(b, a);
      return bfail(b, s, g->err);
    }
    if (vpfft_status s = ensure_crss_array(g)) {
      release(b, a);
      return bfail(b, s, g->err);
    }
    a.tau = g->crss_per_voxel;
    char* base = static_cast<char*>(b->arena_base) + off;
    SlotDesc<S>& d = *host_desc<S>(b, a.slot);
    d = SlotDesc<S>{};
    d.nr_init = nr_params(g, a.r.edot, true);
    d.vox = voxel_params(g, a.r.edot);
    d.f = fields<S>(g);
    d.sp = spectral<S>(g, base, base + spec_al);
    d.fs = FftSlot<S>{d.sp.nx,  d.sp.ny,  d.sp.nz,  d.sp.nh, d.sp.px.by_n, d.sp.py.by_n,
                      d.sp.twx, d.sp.twy, d.sp.twz, d.sp.X,  d.sp.X2,      d.f.work};
    d.crss_out = (S*)g->crss;
    d.partials = g->partials;
    d.sum25 = b->d_sum25 + 25 * (size_t)a.slot;
    d.ctrl = b->d_ctrl + a.slot;
    d.hist = g->hist;
    d.init_blocks = nr_launch_blocks<S>(d.nr_init, a.tau, true);
    IterCtrl& c = b->h_ctrl[a.slot];
    c = IterCtrl{};
    c.n_voxels = (double)g->n;
    if (vpfft_status s = upload_ctrl(b, a.slot)) return s;
    if (vpfft_status s = upload_desc<S>(b, a.slot)) return s;
    for (int k = 0; k < 5; ++k) g->last_edot[k] = a.r.edot[k];
    admitted.push_back((int)b->active.size());
    b->active.push_back(a);
    it = b->queue.erase(it);
  }
  return VPFFT_OK;
}

// ---- autotuner of the batched FFT passes' tile family (vpfft_batch_options
// fft_tiles = -1, the default).  A family only regroups lines into blocks and
// performs the same operations (the line transforms spell out their fused
// multiply-adds and are built without contraction): results are the same bit
// for bit in every family.
struct TileChoice {
  int fam;
  double ms[3];
};
std::mutex g_tile_mu;
std::map<std::tuple<int, int, int, int, int>, TileChoice> g_tiles;  // (device, bytes, nx, ny, nz)

// Mean time of the five passes in family fam over the slots of active[idxs]
// (all of one size): one warm-up chain, then three timed.
template <typename S>
vpfft_status time_chain(vpfft_batch* b, const std::vector<int>& idxs, int fam, double* ms) {
  HostList z, y, x;
  SpectralShape sh{};
  size_t s_zr = 0, s_zc = 0, s_y = 0, s_x = 0;
  for (int idx : idxs) {
    const Active& a = b->active[idx];
    sh = spectral_shape<S>(host_desc<S>(b, a.slot)->sp, 5, fam);
    z.add(a.slot, sh.blocks_z);
    y.add(a.slot, sh.blocks_y);
    x.add(a.slot, sh.blocks_x);
    s_zr = std::max(s_zr, sh.smem_z_r2c);
    s_zc = std::max(s_zc, sh.smem_z_c2r);
    s_y = std::max(s_y, sh.smem_y);
    s_x = std::max(s_x, sh.smem_x);
  }
  std::vector<BatchLaunch> bl;
  if (vpfft_status s = upload_lists(b, b->setup_lists, {&z, &y, &x}, bl)) return s;
  const PassChain c{sh.set_z, sh.set_y, sh.set_x, bl[0], bl[1], bl[2], s_zr, s_zc, s_y, s_x,
                    sh.fam_z, sh.fam_y, sh.fam_x};
  constexpr int kReps = 3;
  b->launches += launch_spectral_chain<S>(dev_desc<S>(b), c, b->stream);
  BCK(b, cudaEventRecord(b->ev_t0, b->stream));
  for (int r = 0; r < kReps; ++r) b->launches += launch_spectral_chain<S>(dev_desc<S>(b), c, b->stream);
  BCK(b, cudaEventRecord(b->ev_t1, b->stream));
  BCK(b, cudaGetLastError());
  // the timed chains also finish before the host stages the next lists
  BCK(b, cudaEventSynchronize(b->ev_t1));
  float t = 0.f;
  BCK(b, cudaEventElapsedTime(&t, b->ev_t0, b->ev_t1));
  *ms = (double)t / kReps;
  return VPFFT_OK;
}

// Tile family of every newly admitted slot.  Runs before the slots'
// initialisation, which rewrites the real field (work) the chain's last pass
// writes; the chain's other outputs are the slots' spectrum buffers.
template <typename S>
vpfft_status assign_tiles(vpfft_batch* b, const std::vector<int>& admitted) {
  // sizes in order of admission, each with its slots
  std::vector<std::pair<std::tuple<int, int, int>, std::vector<int>>> groups;
  for (int idx : admitted) {
    const vpfft_grid* g = b->active[idx].r.g;
    const auto key = std::make_tuple(g->nx, g->ny, g->nz);
    auto it = std::find_if(groups.begin(), groups.end(),
                           [&](const auto& e) { return e.first == key; });
    if (it == groups.end()) it = groups.insert(groups.end(), {key, {}});
    it->second.push_back(idx);
  }
  for (auto& kv : groups) {
    auto it = b->fam_of.find(kv.first);
    if (it == b->fam_of.end()) {
      vpfft_tile_tuning t{};
      std::tie(t.nx, t.ny, t.nz) = kv.first;
      const int nf = spectral_shape<S>(host_desc<S>(b, b->active[kv.second[0]].slot)->sp, 5)
                         .families;
      t.families = nf;
      int fam = nf - 1;
      if (b->bopt.fft_tiles >= 0) {
        fam = std::min(b->bopt.fft_tiles, nf - 1);
        t.source = 0;
      } else if (nf == 1) {
        t.source = 1;
      } else {
        const auto key = std::make_tuple(b->device, (int)sizeof(S), t.nx, t.ny, t.nz);
        bool cached = false;
        {
          std::lock_guard<std::mutex> lk(g_tile_mu);
          auto c = g_tiles.find(key);
          if (c != g_tiles.end()) {
            fam = c->second.fam;
            for (int f = 0; f < 3; ++f) t.ms_per_chain[f] = c->second.ms[f];
            cached = true;
          }
        }
        if (cached) {
          t.source = 2;
        } else {
          for (int f = 0; f < nf; ++f)
            if (vpfft_status s = time_chain<S>(b, kv.second, f, &t.ms_per_chain[f])) return s;
          fam = 0;
          for (int f = 1; f < nf; ++f)
            if (t.ms_per_chain[f] < t.ms_per_chain[fam]) fam = f;
          TileChoice ch{fam, {t.ms_per_chain[0], t.ms_per_chain[1], t.ms_per_chain[2]}};
          std::lock_guard<std::mutex> lk(g_tile_mu);
          g_tiles.emplace(key, ch);
          t.source = 3;
        }
      }
      t.fft_tiles = fam;
      b->tunings.push_back(t);
      it = b->fam_of.emplace(kv.first, fam).first;
    }
    for (int idx : kv.second) b->active[idx].fam = it->second;
  }
  return VPFFT_OK;
}

// After the INIT tick: L0 and the loop constants of an admitted slot.
template <typename S>
vpfft_status start_loop(vpfft_batch* b, Active& a) {
  vpfft_grid* g = a.r.g;
  SlotDesc<S>& d = *host_desc<S>(b, a.slot);
  if (vpfft_status s = finish_ref_medium(g, b->h_sum25 + 25 * (size_t)a.slot)) return s;
  d.nr = nr_params(g, a.r.edot, false);
  d.gp = green_params<S>(g->nx, g->ny, g->nz, g->h, g->L0, g->Linv);
  d.post = post_params(g, a.r.dt);
  d.nr_blocks = nr_launch_blocks<S>(d.nr, a.tau, false);
  b->h_ctrl[a.slot] = loop_ctrl(g, a.r.edot, a.r.max_iter, a.r.eps);
  if (vpfft_status s = upload_ctrl(b, a.slot)) return s;
  if (vpfft_status s = upload_desc<S>(b, a.slot)) return s;
  a.phase = kIter;
  b->iter_generation++;
  return VPFFT_OK;
}

// The iteration lists of the slots in ITER phase.
// The iterating RVEs of one size class (the same line engines on all axes).
struct ClassList {
  const void* set_z;
  const void* set_y;
  const void* set_x;
  int fam_z, fam_y, fam_x;
  HostList z, y, x;
  size_t smem_z_r2c = 0, smem_z_c2r = 0, smem_y = 0, smem_x = 0;
};
struct IterLists {
  std::vector<ClassList> cls;
  HostList nr[2], fin[2];
};

template <typename S>
void build_iter_lists(vpfft_batch* b, IterLists& L) {
  for (const Active& a : b->active) {
    if (a.phase != kIter) continue;
    const SlotDesc<S>& d = *host_desc<S>(b, a.slot);
    const SpectralShape sh = spectral_shape<S>(d.sp, 5, a.fam);
    ClassList* c = nullptr;
    for (ClassList& e : L.cls)
      if (e.set_z == sh.set_z && e.set_y == sh.set_y && e.set_x == sh.set_x &&
          e.fam_z == sh.fam_z && e.fam_y == sh.fam_y && e.fam_x == sh.fam_x)
        c = &e;
    if (!c) {
      L.cls.push_back(ClassList{sh.set_z, sh.set_y, sh.set_x, sh.fam_z, sh.fam_y, sh.fam_x,
                                {}, {}, {}});
      c = &L.cls.back();
    }
    c->z.add(a.slot, sh.blocks_z);
    c->y.add(a.slot, sh.blocks_y);
    c->x.add(a.slot, sh.blocks_x);
    c->smem_z_r2c = std::max(c->smem_z_r2c, sh.smem_z_r2c);
    c->smem_z_c2r = std::max(c->smem_z_c2r, sh.smem_z_c2r);
    c->smem_y = std::max(c->smem_y, sh.smem_y);
    c->smem_x = std::max(c->smem_x, sh.smem_x);
    L.nr[a.tau].add(a.slot, d.nr_blocks);
    L.fin[a.tau].add(a.slot, 1);
  }
}

// lists: z, y, x of every class in order, then nr[0], nr[1], fin[0], fin[1]
template <typename S>
int enqueue_iterations(vpfft_batch* b, const std::vector<BatchLaunch>& bl, const IterLists& L,
                       int iters) {
  std::vector<PassChain> chains;
  size_t k = 0;
  for (const ClassList& c : L.cls) {
    chains.push_back(PassChain{c.set_z, c.set_y, c.set_x, bl[k], bl[k + 1], bl[k + 2],
                               c.smem_z_r2c, c.smem_z_c2r, c.smem_y, c.smem_x, c.fam_z, c.fam_y,
                               c.fam_x});
    k += 3;
  }
  // material and solver constants: those of any iterating slot (a batch admits
  // only grids with its own material and options)
  const int any = !L.nr[0].slot.empty() ? L.nr[0].slot[0] : L.nr[1].slot[0];
  const NRParams& material = host_desc<S>(b, any)->nr;
  const int nch = (int)chains.size();
  const int naux = std::min(nch, vpfft_batch::kAux);
  int n = 0;
  for (int it = 0; it < iters; ++it) {
    if (nch == 1) {
      n += launch_spectral_chain<S>(dev_desc<S>(b), chains[0], b->stream);
    } else {
      cudaEventRecord(b->ev_fork, b->stream);
      for (int a = 0; a < naux; ++a) cudaStreamWaitEvent(b->aux[a], b->ev_fork, 0);
      for (int c = 0; c < nch; ++c)
        n += launch_spectral_chain<S>(dev_desc<S>(b), chains[c], b->aux[c % naux]);
      for (int a = 0; a < naux; ++a) {
        cudaEventRecord(b->ev_join[a], b->aux[a]);
        cudaStreamWaitEvent(b->stream, b->ev_join[a], 0);
      }
    }
    for (int t = 0; t < 2; ++t)
      n += launch_nr_update_batch<S>(dev_desc<S>(b), bl[k + t], bl[k + 2 + t], material, b->nexp,
                                     t == 1, b->stream);
  }
  return n;
}

// The tick's iterations.  While the set of iterating slots stays the same the
// launches are replayed from a CUDA graph: the first chunk of a new set runs
// eagerly (it also sets the kernels' shared-memory attributes), the second is
// captured and launched, later ones replay it.
template <typename S>
vpfft_status run_iterations(vpfft_batch* b) {
  IterLists L;
  build_iter_lists<S>(b, L);
  if (L.cls.empty()) return VPFFT_OK;
  const int iters = std::max(1, b->bopt.iterations_per_tick);
  if (b->bopt.use_graphs && b->graph && b->graph_generation == b->iter_generation) {
    BCK(b, cudaGraphLaunch(b->graph, b->stream));
    b->graph_replays++;
    return VPFFT_OK;
  }
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  std::vector<HostList*> lists;
  for (ClassList& c : L.cls)
    for (HostList* h : {&c.z, &c.y, &c.x}) lists.push_back(h);
  for (HostList* h : {&L.nr[0], &L.nr[1], &L.fin[0], &L.fin[1]}) lists.push_back(h);
  std::vector<BatchLaunch> bl;
  if (vpfft_status s = upload_lists(b, b->iter_lists, lists, bl)) return s;
  if (b->bopt.use_graphs && b->eager_generation == b->iter_generation) {
    cudaGraph_t graph = nullptr;
    BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int n = enqueue_iterations<S>(b, bl, L, iters);
    cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (e != cudaSuccess)
      return bfail(b, VPFFT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess)
      return bfail(b, VPFFT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    b->graph_generation = b->iter_generation;
    BCK(b, cudaGraphLaunch(b->graph, b->stream));
    b->graph_replays++;
    b->launches += n;
    return VPFFT_OK;
  }
  b->launches += enqueue_iterations<S>(b, bl, L, iters);
  b->eager_generation = b->iter_generation;
  BCK(b, cudaGetLastError());
  return VPFFT_OK;
}

template <typename S>
vpfft_status tick(vpfft_batch* b) {
  BCK(b, cudaSetDevice(b->device));
  b->ticks++;
  // cancelled requests still queued complete at once
  for (auto it = b->queue.begin(); it != b->queue.end();) {
    if (it->cancelled) {
      Active a;
      a.r = *it;
      a.slot = -1;
      vpfft_batch_result r{};
      r.request_id = it->id;
      r.status = VPFFT_ERR_CANCELLED;
      r.seconds_total = now_s() - it->t_submit;
      b->results.push_back(r);
      b->completed++;
      it = b->queue.erase(it);
    } else {
      ++it;
    }
  }
  // cancelled active requests leave before any work of this tick
  for (size_t i = 0; i < b->active.size();) {
    Active& a = b->active[i];
    if (a.r.cancelled) {
      record(b, a, VPFFT_ERR_CANCELLED, now_s());
      if (a.phase == kIter) b->iter_generation++;
      release(b, a);
      b->active.erase(b->active.begin() + i);
    } else {
      ++i;
    }
  }
  // 1. admission and the initialisation of the new slots
  std::vector<int> admitted;
  if (vpfft_status s = admit<S>(b, admitted)) return s;
  if (vpfft_status s = assign_tiles<S>(b, admitted)) return s;
  if (!admitted.empty()) {
    HostList init[2], rm, rms;
    for (int idx : admitted) {
      const Active& a = b->active[idx];
      const SlotDesc<S>& d = *host_desc<S>(b, a.slot);
      init[a.tau].add(a.slot, d.init_blocks);
      rm.add(a.slot, (int)((d.vox.n + 127) / 128));
      rms.add(a.slot, 1);
    }
    std::vector<BatchLaunch> bl;
    if (vpfft_status s = upload_lists(b, b->setup_lists, {&init[0], &init[1], &rm, &rms}, bl))
      return s;
    for (int t = 0; t < 2; ++t)
      b->launches += launch_init_batch<S>(dev_desc<S>(b), bl[t], b->nexp, t == 1, b->stream);
    b->launches += launch_ref_medium_batch<S>(dev_desc<S>(b), bl[2], bl[3], b->stream);
    BCK(b, cudaGetLastError());
  }
  // 2. the iterations of the slots already iterating
  if (vpfft_status s = run_iterations<S>(b)) return s;
  // 3. read back control blocks and reference-medium sums
  const int ms = b->bopt.max_slots;
  BCK(b, cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, sizeof(IterCtrl) * ms, cudaMemcpyDeviceToHost,
                         b->stream));
  BCK(b, cudaMemcpyAsync(b->h_sum25, b->d_sum25, sizeof(double) * 25 * ms,
                         cudaMemcpyDeviceToHost, b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  const double t_now = now_s();
  // 4. finished loops: post-increment update (one launch) and results
  HostList post;
  std::vector<size_t> finishing;
  for (size_t i = 0; i < b->active.size(); ++i) {
    Active& a = b->active[i];
    const IterCtrl& c = b->h_ctrl[a.slot];
    if (a.phase != kIter || !c.done) continue;
    if (c.status & (kStatusNonFinite | kStatusMaxRssTiny)) continue;  // no post on error
    post.add(a.slot, (int)((a.r.g->n + 127) / 128));
    finishing.push_back(i);
  }
  if (post.m()) {
    std::vector<BatchLaunch> bl;
    if (vpfft_status s = upload_lists(b, b->setup_lists, {&post}, bl)) return s;
    b->launches += launch_post_batch<S>(dev_desc<S>(b), bl[0], b->stream);
    BCK(b, cudaGetLastError());
    BCK(b, cudaStreamSynchronize(b->stream));
  }
  // 5. phase transitions
  const double t_end = now_s();
  std::vector<Active> keep;
  keep.reserve(b->active.size());
  for (Active& a : b->active) {
    const IterCtrl& c = b->h_ctrl[a.slot];
    if (a.phase == kInit) {
      vpfft_status st = VPFFT_OK;
      if (c.status & kStatusNonFinite) st = VPFFT_ERR_NONFINITE;
      else if (c.status & kStatusMaxRssTiny) st = VPFFT_ERR_MAX_RSS_TINY;
      if (st == VPFFT_OK) st = start_loop<S>(b, a);
      if (st != VPFFT_OK) {
        record(b, a, st, t_now);
        release(b, a);
        continue;
      }
      keep.push_back(a);
    } else if (a.phase == kIter && c.done) {
      vpfft_status st = VPFFT_OK;
      if (c.status & kStatusNonFinite) st = VPFFT_ERR_NONFINITE;
      else if (c.status & kStatusMaxRssTiny) st = VPFFT_ERR_MAX_RSS_TINY;
      if (st == VPFFT_OK) finish_post(a.r.g, a.r.edot, a.r.dt);
      record(b, a, st, t_end);
      b->iter_generation++;
      release(b, a);
    } else {
      keep.push_back(a);
    }
  }
  b->active.swap(keep);
  return VPFFT_OK;
}

void free_batch(vpfft_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  void* ptrs[] = {b->arena_base, b->d_desc, b->d_ctrl, b->d_sum25, b->setup_lists.d,
                  b->iter_lists.d};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  void* hptrs[] = {b->h_ctrl, b->h_sum25, b->h_desc, b->setup_lists.h, b->iter_lists.h};
  for (void* p : hptrs)
    if (p) cudaFreeHost(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (int a = 0; a < vpfft_batch::kAux; ++a) {
    if (b->aux[a]) cudaStreamDestroy(b->aux[a]);
    if (b->ev_join[a]) cudaEventDestroy(b->ev_join[a]);
  }
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_t0) cudaEventDestroy(b->ev_t0);
  if (b->ev_t1) cudaEventDestroy(b->ev_t1);
}

}  // namespace

extern "C" {

void vpfft_batch_options_default(vpfft_batch_options* o) {
  if (!o) return;
  o->max_slots = 256;
  o->iterations_per_tick = 8;
  o->hbm_budget_bytes = 8LL << 30;
  o->use_graphs = 1;
  o->fft_tiles = -1;
}

vpfft_status vpfft_batch_create(vpfft_precision precision, const vpfft_material* material,
                                const vpfft_solver_options* options,
                                const vpfft_batch_options* bopt, vpfft_batch** out) {
  if (!out) return bfail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (precision != VPFFT_PREC_FP64 && precision != VPFFT_PREC_MIXED)
    return bfail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "unknown precision");
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt <= 0) {
    cudaGetLastError();
    return bfail(nullptr, VPFFT_ERR_NO_DEVICE,
                 "no CUDA device available (vpfft_b200 has no CPU fallback)");
  }
  vpfft_batch* b = new vpfft_batch();
  b->prec = precision;
  if (material)
    b->mat = *material;
  else
    vpfft_material_default(&b->mat);
  if (options)
    b->opt = *options;
  else
    vpfft_solver_options_default(&b->opt);
  if (bopt)
    b->bopt = *bopt;
  else
    vpfft_batch_options_default(&b->bopt);
  if (b->bopt.max_slots < 1 || b->bopt.max_slots > 65536 || b->bopt.hbm_budget_bytes < 0 ||
      b->bopt.fft_tiles < -1 || b->bopt.fft_tiles > 2) {
    delete b;
    return bfail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "bad batch options");
  }
  {
    NRParams p{};
    for (int q = 0; q < kNS; ++q) p.nexp[q] = b->mat.rate_sensitivity[q];
    b->nexp = uniform_exponent(p);
  }
  cudaGetDevice(&b->device);
  auto bail = [&](cudaError_t e, const char* what) {
    g_batch_err = std::string(what) + ": " + cudaGetErrorString(e);
    free_batch(b);
    delete b;
    return e == cudaErrorMemoryAllocation ? VPFFT_ERR_OUT_OF_MEMORY : VPFFT_ERR_CUDA;
  };
  const int ms = b->bopt.max_slots;
  const size_t desc_bytes = precision == VPFFT_PREC_FP64 ? sizeof(SlotDesc<double>)
                                                         : sizeof(SlotDesc<float>);
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(e, "stream");
  for (int a = 0; a < vpfft_batch::kAux; ++a) {
    if ((e = cudaStreamCreateWithFlags(&b->aux[a], cudaStreamNonBlocking)) != cudaSuccess)
      return bail(e, "stream");
    if ((e = cudaEventCreateWithFlags(&b->ev_join[a], cudaEventDisableTiming)) != cudaSuccess)
      return bail(e, "event");
  }
  if ((e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming)) != cudaSuccess)
    return bail(e, "event");
  if ((e = cudaEventCreate(&b->ev_t0)) != cudaSuccess) return bail(e, "event");
  if ((e = cudaEventCreate(&b->ev_t1)) != cudaSuccess) return bail(e, "event");
  if (b->bopt.hbm_budget_bytes > 0 &&
      (e = cudaMalloc(&b->arena_base, (size_t)b->bopt.hbm_budget_bytes)) != cudaSuccess)
    return bail(e, "arena");
  b->arena = Arena((size_t)b->bopt.hbm_budget_bytes);
  if ((e = cudaMalloc(&b->d_desc, desc_bytes * ms)) != cudaSuccess) return bail(e, "descriptors");
  if ((e = cudaMalloc(&b->d_ctrl, sizeof(IterCtrl) * ms)) != cudaSuccess) return bail(e, "ctrl");
  if ((e = cudaMalloc(&b->d_sum25, sizeof(double) * 25 * ms)) != cudaSuccess) return bail(e, "sums");
  if ((e = cudaMallocHost(&b->h_ctrl, sizeof(IterCtrl) * ms)) != cudaSuccess) return bail(e, "pinned");
  if ((e = cudaMallocHost(&b->h_sum25, sizeof(double) * 25 * ms)) != cudaSuccess)
    return bail(e, "pinned");
  // block lists sized for a full batch (a tick then never allocates)
  for (DeviceLists* dl : {&b->setup_lists, &b->iter_lists}) {
    const int cap = 16 * ms + 64;
    if ((e = cudaMalloc(&dl->d, sizeof(int) * cap)) != cudaSuccess) return bail(e, "lists");
    if ((e = cudaMallocHost(&dl->h, sizeof(int) * cap)) != cudaSuccess) return bail(e, "pinned");
    dl->cap = cap;
  }
  std::memset(b->h_ctrl, 0, sizeof(IterCtrl) * ms);
  if ((e = cudaMemset(b->d_ctrl, 0, sizeof(IterCtrl) * ms)) != cudaSuccess) return bail(e, "ctrl");
  if ((e = cudaMallocHost(&b->h_desc, desc_bytes * ms)) != cudaSuccess) return bail(e, "pinned");
  std::memset(b->h_desc, 0, desc_bytes * ms);
  for (int s = ms - 1; s >= 0; --s) b->free_slots.push_back(s);
  *out = b;
  return VPFFT_OK;
}

vpfft_status vpfft_batch_destroy(vpfft_batch* b) {
  if (!b) return VPFFT_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (Active& a : b->active) a.r.g->in_batch = false;
  free_batch(b);
  delete b;
  return VPFFT_OK;
}

vpfft_status vpfft_batch_submit(vpfft_batch* b, vpfft_grid* g, const double edot[5], int max_iter,
                                double dt, double eps, int64_t* id) {
  if (!b || !g || !edot) return bfail(b, VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (g->prec != b->prec) return bfail(b, VPFFT_ERR_INVALID_ARGUMENT, "grid precision differs from the batch's");
  if (g->device != b->device) return bfail(b, VPFFT_ERR_INVALID_ARGUMENT, "grid lives on another device");
  // the solver constants must agree (field by field: the struct has padding);
  // green_operator does not apply to batched solves (they compute the operator)
  const vpfft_solver_options& go = g->opt;
  const vpfft_solver_options& bo = b->opt;
  const bool same_opt = go.init_nr_epsilon == bo.init_nr_epsilon &&
                        go.init_nr_max_iter == bo.init_nr_max_iter &&
                        go.nr_epsilon == bo.nr_epsilon && go.nr_max_resolved == bo.nr_max_resolved &&
                        go.nr_max_iter == bo.nr_max_iter &&
                        go.mixed_certify_step == bo.mixed_certify_step;
  if (std::memcmp(&g->mat, &b->mat, sizeof(vpfft_material)) != 0 || !same_opt)
    return bfail(b, VPFFT_ERR_INVALID_ARGUMENT, "grid material or solver options differ from the batch's");
  if (!g->fields_set) return bfail(b, VPFFT_ERR_NOT_INITIALIZED, "grid fields not set");
  if (max_iter < 1) return bfail(b, VPFFT_ERR_INVALID_ARGUMENT, "max_iter must be >= 1");
  const size_t need = 2 * ((spectrum_bytes(g) + 255) & ~size_t(255));
  if (need > b->arena.size())
    return bfail(b, VPFFT_ERR_OUT_OF_MEMORY, "the grid's spectra exceed the batch's HBM budget");
  Request r;
  r.id = b->next_id++;
  r.g = g;
  std::memcpy(r.edot, edot, sizeof(r.edot));
  r.max_iter = max_iter;
  r.dt = dt;
  r.eps = eps;
  r.t_submit = now_s();
  b->queue.push_back(r);
  if (id) *id = r.id;
  return VPFFT_OK;
}

vpfft_status vpfft_batch_step(vpfft_batch* b, int* pending) {
  if (!b) return bfail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL batch");
  nvtxRangePushA("vpfft batch tick");  // NVTX range per tick (Nsight timelines)
  vpfft_status s = b->prec == VPFFT_PREC_FP64 ? tick<double>(b) : tick<float>(b);
  nvtxRangePop();
  if (pending) *pending = (int)(b->queue.size() + b->active.size());
  return s;
}

vpfft_status vpfft_batch_run(vpfft_batch* b) {
  if (!b) return bfail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL batch");
  int pending = 1;
  while (pending > 0) {
    vpfft_status s = vpfft_batch_step(b, &pending);
    if (s != VPFFT_OK) return s;
  }
  return VPFFT_OK;
}

vpfft_status vpfft_batch_poll(vpfft_batch* b, vpfft_batch_result* out, int cap, int* n_out) {
  if (!b || (!out && cap > 0)) return bfail(b, VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  int n = 0;
  while (n < cap && !b->results.empty()) {
    out[n++] = b->results.front();
    b->results.pop_front();
  }
  if (n_out) *n_out = n;
  return VPFFT_OK;
}

vpfft_status vpfft_batch_cancel(vpfft_batch* b, int64_t id) {
  if (!b) return bfail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL batch");
  for (Request& r : b->queue)
    if (r.id == id) {
      r.cancelled = true;
      return VPFFT_OK;
    }
  for (Active& a : b->active)
    if (a.r.id == id) {
      a.r.cancelled = true;
      return VPFFT_OK;
    }
  return bfail(b, VPFFT_ERR_INVALID_ARGUMENT, "no such pending request");
}

vpfft_status vpfft_batch_get_info(const vpfft_batch* b, vpfft_batch_info* info) {
  if (!b || !info) return VPFFT_ERR_INVALID_ARGUMENT;
  info->queued = (int64_t)b->queue.size();
  info->active = (int64_t)b->active.size();
  info->completed = b->completed;
  info->ticks = b->ticks;
  info->graph_replays = b->graph_replays;
  info->kernel_launches = b->launches;
  info->arena_bytes_in_use = (int64_t)b->arena.in_use();
  info->arena_bytes = (int64_t)b->arena.size();
  info->admissions_deferred_for_memory = b->deferred;
  return VPFFT_OK;
}

vpfft_status vpfft_batch_get_tunings(const vpfft_batch* b, vpfft_tile_tuning* out, int cap,
                                     int* n_out) {
  if (!b || !n_out || cap < 0 || (cap > 0 && !out))
    return bfail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "bad arguments");
  const int n = std::min(cap, (int)b->tunings.size());
  for (int i = 0; i < n; ++i) out[i] = b->tunings[i];
  *n_out = (int)b->tunings.size();
  return VPFFT_OK;
}

const char* vpfft_batch_last_error(const vpfft_batch* b) {
  return b ? b->err.c_str() : g_batch_err.c_str();
}

}  // extern "C"
