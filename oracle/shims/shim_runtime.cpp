// shim_runtime.cpp -- implementations of the MPI and FFTW stand-ins declared in
// mpi.h / fftw3-mpi.h, plus the observation hooks.  Test-oracle infrastructure
// only.
//
// Two modes:
//   * one rank (the default): MPI_Allreduce copies, point-to-point calls are
//     never reached, fftw_execute runs the oracle's 3D DFT in place;
//   * P ranks (vpfft_shim_configure(P, ...) before MPI_Init): MPI_Init forks
//     P - 1 processes that share one anonymous mapping made before the fork
//     (so every rank sees every other rank's FFT slabs at the same address).
//     The FFTW-MPI slab decomposition is FFTW's default (blocks of
//     ceil(n0 / P) planes along the first axis), fftw_execute is collective:
//     each rank transforms the z and y lines of its own planes, then a share
//     of the x lines gathered across all slabs, with barriers between.  Every
//     line uses the same 1D transform in the same axis order as the one-rank
//     3D DFT (z, y, x), so each element comes out bit for bit the same.
//     MPI_Allreduce sums the ranks' contributions in rank order; sends are
//     buffered in a shared mailbox (FIFO per sender, receiver and tag).
//   All waits poll with back-off and give up (the whole job exits with an
//   error) when a rank dies or nothing moves for ten minutes.
#include <atomic>
#include <chrono>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <sched.h>
#include <signal.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#include "../common/dft.h"
#include "fftw3-mpi.h"
#include "mpi.h"
#include "shim_hooks.h"

namespace {
vpfft_shim_exec_hook g_exec_hook = nullptr;
void *g_exec_user = nullptr;
vpfft_shim_allreduce_hook g_ar_hook = nullptr;
void *g_ar_user = nullptr;
vpfft_shim_barrier_hook g_bar_hook = nullptr;
void *g_bar_user = nullptr;
long g_exec_count = 0;
long g_ar_count = 0;
double g_fft_seconds = 0.0;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

[[noreturn]] void die(const char *what) {
  std::fprintf(stderr, "[vpfft shim] %s\n", what);
  std::fflush(stderr);
  _exit(3);
}

// ---------------------------------------------------------------- multi-rank state
constexpr int kMaxRanks = 256;
constexpr int kMaxReduce = 64;   // doubles per MPI_Allreduce
constexpr int kMaxPlans = 64;
constexpr int kMaxMsgs = 4096;
constexpr double kStallSeconds = 600.0;

struct PlanSlot {
  fftw_complex *in, *out;
};
struct Msg {
  std::atomic<int> state;  // 0 free, 1 published, 2 consumed
  int src, dst, tag;
  size_t off, size;
};
struct Shared {
  std::atomic<int> abort;
  std::atomic<unsigned> bar_count;
  std::atomic<unsigned> bar_gen;
  std::atomic<int> msg_count;
  std::atomic<size_t> mbox_top;
  double red[kMaxRanks][kMaxReduce];
  PlanSlot plans[kMaxPlans][kMaxRanks];
  Msg msgs[kMaxMsgs];
};

int g_ranks = 1, g_rank = 0;
size_t g_arena_per_rank = 0, g_mailbox = 0;
Shared *g_sh = nullptr;
char *g_arena = nullptr;  // rank r's heap at g_arena + r * g_arena_per_rank
char *g_mbox = nullptr;
size_t g_arena_top = 0;
int g_plan_count = 0;
pid_t g_parent = 0;
std::vector<pid_t> g_children;

struct PendingRecv {
  void *buf;
  size_t size;
  int src, tag;
};
std::vector<PendingRecv> g_pending;

void check_peers() {
  if (g_sh->abort.load(std::memory_order_relaxed)) _exit(3);
  if (g_rank == 0) {
    int st = 0;
    pid_t p = waitpid(-1, &st, WNOHANG);
    if (p > 0 && !(WIFEXITED(st) && WEXITSTATUS(st) == 0)) {
      g_sh->abort.store(1);
      die("a rank died; stopping the job");
    }
  } else if (getppid() != g_parent) {
    _exit(3);
  }
}

// Polls `done` with back-off: spin, then yield, then sleep 50 us.
template <class F>
void wait_until(F done) {
  const double t0 = now_s();
  for (long it = 0; !done(); ++it) {
    if (it < 2000) {
#if defined(__x86_64__)
      __builtin_ia32_pause();
#endif
      continue;
    }
    if ((it & 63) == 0) {
      check_peers();
      if (now_s() - t0 > kStallSeconds) {
        g_sh->abort.store(1);
        die("a wait made no progress for ten minutes; stopping the job");
      }
    }
    if (it < 20000) {
      sched_yield();
    } else {
      struct timespec ts = {0, 50000};
      nanosleep(&ts, nullptr);
    }
  }
}

void barrier() {
  if (g_ranks == 1) return;
  const unsigned gen = g_sh->bar_gen.load(std::memory_order_acquire);
  if (g_sh->bar_count.fetch_add(1, std::memory_order_acq_rel) == (unsigned)g_ranks - 1) {
    g_sh->bar_count.store(0, std::memory_order_relaxed);
    g_sh->bar_gen.fetch_add(1, std::memory_order_acq_rel);
  } else {
    wait_until([&] { return g_sh->bar_gen.load(std::memory_order_acquire) != gen; });
  }
}

// FFTW's default slab distribution: blocks of ceil(n0 / P) planes.
void slab(ptrdiff_t n0, int rank, ptrdiff_t *local_n0, ptrdiff_t *start) {
  const ptrdiff_t block = (n0 + g_ranks - 1) / g_ranks;
  ptrdiff_t s = block * rank;
  if (s > n0) s = n0;
  ptrdiff_t e = s + block;
  if (e > n0) e = n0;
  *start = s;
  *local_n0 = e - s;
}

size_t dtype_size(MPI_Datatype dt) {
  return dt == MPI_DOUBLE ? sizeof(double)
         : dt == MPI_FLOAT ? sizeof(float)
         : dt == MPI_INT   ? sizeof(int)
                           : 1;
}

void post(const void *buf, size_t size, int dest, int tag) {
  const size_t off = g_sh->mbox_top.fetch_add((size + 63) & ~size_t(63));
  if (off + size > g_mailbox) die("message mailbox exhausted");
  std::memcpy(g_mbox + off, buf, size);
  const int k = g_sh->msg_count.fetch_add(1);
  if (k >= kMaxMsgs) die("too many messages");
  Msg &m = g_sh->msgs[k];
  m.src = g_rank;
  m.dst = dest;
  m.tag = tag;
  m.off = off;
  m.size = size;
  m.state.store(1, std::memory_order_release);
}

void take(void *buf, size_t size, int src, int tag, MPI_Status *st) {
  // the oldest published message from src to this rank with this tag; a
  // sender publishes in order, so scanning by slot index is FIFO per sender
  Msg *found = nullptr;
  wait_until([&] {
    const int n = g_sh->msg_count.load(std::memory_order_acquire);
    for (int k = 0; k < n && k < kMaxMsgs; ++k) {
      Msg &m = g_sh->msgs[k];
      const int s = m.state.load(std::memory_order_acquire);
      if (s == 0) return false;  // an older slot not yet published: keep order
      if (s != 1 || m.dst != g_rank || m.src != src || m.tag != tag) continue;
      int one = 1;
      if (m.state.compare_exchange_strong(one, 2)) {
        found = &m;
        return true;
      }
    }
    return false;
  });
  if (found->size > size) die("received message longer than the receive buffer");
  std::memcpy(buf, g_mbox + found->off, found->size);
  if (st) {
    st->MPI_SOURCE = src;
    st->MPI_TAG = tag;
    st->MPI_ERROR = MPI_SUCCESS;
  }
}
}  // namespace

struct vpfft_shim_plan_s {
  ptrdiff_t n0, n1, n2;
  fftw_complex *in;
  fftw_complex *out;
  int sign;
  int id;  // collective plan index (multi-rank mode)
};

extern "C" {

void vpfft_shim_set_exec_hook(vpfft_shim_exec_hook h, void *user) {
  g_exec_hook = h;
  g_exec_user = user;
}
void vpfft_shim_set_allreduce_hook(vpfft_shim_allreduce_hook h, void *user) {
  g_ar_hook = h;
  g_ar_user = user;
}
void vpfft_shim_set_barrier_hook(vpfft_shim_barrier_hook h, void *user) {
  g_bar_hook = h;
  g_bar_user = user;
}
long vpfft_shim_exec_count(void) { return g_exec_count; }
long vpfft_shim_allreduce_count(void) { return g_ar_count; }
double vpfft_shim_fft_seconds(void) { return g_fft_seconds; }

int vpfft_shim_configure(int ranks, size_t arena_bytes_per_rank, size_t mailbox_bytes) {
  if (ranks < 1 || ranks > kMaxRanks || g_sh) return 1;
  g_ranks = ranks;
  g_arena_per_rank = (arena_bytes_per_rank + 4095) & ~size_t(4095);
  g_mailbox = (mailbox_bytes + 4095) & ~size_t(4095);
  return 0;
}

// ---------------------------------------------------------------- MPI
int MPI_Init(int *, char ***) {
  if (g_ranks == 1 || g_sh) return MPI_SUCCESS;
  const size_t hdr = (sizeof(Shared) + 4095) & ~size_t(4095);
  const size_t total = hdr + g_arena_per_rank * (size_t)g_ranks + g_mailbox;
  void *p = mmap(nullptr, total, PROT_READ | PROT_WRITE,
                 MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
  if (p == MAP_FAILED) die("cannot map the shared arena");
  g_sh = static_cast<Shared *>(p);  // zero-filled by the kernel: atomics start at 0
  g_arena = static_cast<char *>(p) + hdr;
  g_mbox = g_arena + g_arena_per_rank * (size_t)g_ranks;
  g_parent = getpid();
  std::fflush(stdout);
  std::fflush(stderr);
  for (int r = 1; r < g_ranks; ++r) {
    const pid_t c = fork();
    if (c < 0) die("fork failed");
    if (c == 0) {
      g_rank = r;
      g_children.clear();
      return MPI_SUCCESS;
    }
    g_children.push_back(c);
  }
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  if (g_ranks == 1) return MPI_SUCCESS;
  barrier();
  if (g_rank != 0) {
    std::fflush(stdout);
    std::fflush(stderr);
    _exit(0);
  }
  int bad = 0;
  for (pid_t c : g_children) {
    int st = 0;
    if (waitpid(c, &st, 0) < 0 || !(WIFEXITED(st) && WEXITSTATUS(st) == 0)) bad = 1;
  }
  if (bad) die("a rank failed");
  return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = g_rank;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int *size) {
  *size = g_ranks;
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op,
                  MPI_Comm) {
  const size_t esz = dtype_size(dt);
  if (g_ranks == 1) {
    std::memmove(recvbuf, sendbuf, esz * (size_t)count);
  } else {
    if (count > kMaxReduce || !(dt == MPI_DOUBLE || dt == MPI_INT))
      die("MPI_Allreduce: only sums of up to 64 doubles or ints are supported");
    std::memcpy(g_sh->red[g_rank], sendbuf, esz * (size_t)count);
    barrier();
    if (dt == MPI_DOUBLE) {
      double *out = static_cast<double *>(recvbuf);
      for (int i = 0; i < count; ++i) {
        double s = g_sh->red[0][i];
        for (int r = 1; r < g_ranks; ++r) s += g_sh->red[r][i];
        out[i] = s;
      }
    } else {
      int *out = static_cast<int *>(recvbuf);
      for (int i = 0; i < count; ++i) {
        long long s = 0;
        for (int r = 0; r < g_ranks; ++r) s += reinterpret_cast<const int *>(g_sh->red[r])[i];
        out[i] = (int)s;
      }
    }
    barrier();
  }
  ++g_ar_count;
  if (g_ar_hook && dt == MPI_DOUBLE) g_ar_hook((const double *)recvbuf, count, g_ar_user);
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm) {
  barrier();
  if (g_bar_hook) g_bar_hook(g_bar_user);
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm) {
  if (g_ranks == 1) die("MPI_Send is not available with one rank");
  post(buf, dtype_size(dt) * (size_t)count, dest, tag);
  return MPI_SUCCESS;
}
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm, MPI_Status *st) {
  if (g_ranks == 1) die("MPI_Recv is not available with one rank");
  take(buf, dtype_size(dt) * (size_t)count, src, tag, st);
  return MPI_SUCCESS;
}
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm,
              MPI_Request *req) {
  if (g_ranks == 1) die("MPI_Isend is not available with one rank");
  post(buf, dtype_size(dt) * (size_t)count, dest, tag);  // buffered: complete at once
  *req = 0;
  return MPI_SUCCESS;
}
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm,
              MPI_Request *req) {
  if (g_ranks == 1) die("MPI_Irecv is not available with one rank");
  g_pending.push_back(PendingRecv{buf, dtype_size(dt) * (size_t)count, src, tag});
  *req = (int)g_pending.size();
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *req, MPI_Status *st) {
  if (req && *req > 0) {
    const PendingRecv r = g_pending[(size_t)*req - 1];
    take(r.buf, r.size, r.src, r.tag, st);
    *req = 0;
  }
  return MPI_SUCCESS;
}

// ---------------------------------------------------------------- FFTW
void fftw_mpi_init(void) {}
void fftw_cleanup(void) {}

ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start) {
  if (g_ranks == 1) {
    *local_n0 = n0;
    *local_0_start = 0;
    return n0 * n1 * n2;
  }
  slab(n0, g_rank, local_n0, local_0_start);
  const ptrdiff_t n = *local_n0 * n1 * n2;
  return n > 0 ? n : 1;
}

void *fftw_malloc(size_t n) {
  if (g_ranks > 1) {
    // from this rank's part of the shared arena, so other ranks can reach it
    const size_t sz = (n + 63) & ~size_t(63);
    if (g_arena_top + sz > g_arena_per_rank) die("shared FFT arena exhausted");
    void *p = g_arena + (size_t)g_rank * g_arena_per_rank + g_arena_top;
    g_arena_top += sz;
    return p;
  }
  void *p = nullptr;
  if (posix_memalign(&p, 64, n ? n : 1) != 0) return nullptr;
  return p;
}
fftw_complex *fftw_alloc_complex(size_t n) {
  return (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
}
void fftw_free(void *p) {
  if (g_ranks == 1) std::free(p);  // arena memory lives until the process ends
}

fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in,
                               fftw_complex *out, MPI_Comm, int sign, unsigned) {
  auto *p = new vpfft_shim_plan_s{n0, n1, n2, in, out, sign, -1};
  if (g_ranks > 1) {
    // plans are made collectively in the same order on every rank
    if (g_plan_count >= kMaxPlans) die("too many FFT plans");
    p->id = g_plan_count++;
    g_sh->plans[p->id][g_rank] = PlanSlot{in, out};
    barrier();
  }
  return p;
}

void fftw_execute(const fftw_plan p) {
  ++g_exec_count;
  ptrdiff_t ln0 = p->n0, start0 = 0;
  if (g_ranks > 1) slab(p->n0, g_rank, &ln0, &start0);
  const long total = (long)(ln0 * p->n1 * p->n2);
  if (g_exec_hook) g_exec_hook(p->sign, p->in, total, g_exec_user);
  const double t0 = now_s();
  if (g_ranks == 1) {
    if (p->out != p->in) std::memcpy(p->out, p->in, sizeof(fftw_complex) * (size_t)total);
    oracle_dft3d_inplace(reinterpret_cast<oracle_cplx *>(p->out), (size_t)p->n0, (size_t)p->n1,
                         (size_t)p->n2, p->sign);
    g_fft_seconds += now_s() - t0;
    return;
  }
  barrier();
  if (p->out != p->in && total > 0)
    std::memcpy(p->out, p->in, sizeof(fftw_complex) * (size_t)total);
  // z then y lines of this rank's planes: the 3D routine on one plane at a
  // time (a first axis of length 1 is skipped)
  const size_t plane = (size_t)p->n1 * (size_t)p->n2;
  for (ptrdiff_t x = 0; x < ln0; ++x)
    oracle_dft3d_inplace(reinterpret_cast<oracle_cplx *>(p->out) + (size_t)x * plane, 1,
                         (size_t)p->n1, (size_t)p->n2, p->sign);
  barrier();
  // x lines: this rank's share of the n1*n2 columns, gathered across slabs in
  // runs of consecutive z (contiguous within every plane)
  const size_t n0 = (size_t)p->n0;
  const size_t c0 = plane * (size_t)g_rank / (size_t)g_ranks;
  const size_t c1 = plane * (size_t)(g_rank + 1) / (size_t)g_ranks;
  if (n0 > 1 && c1 > c0) {
    constexpr size_t kRun = 16;
    oracle_dft1d *d = oracle_dft1d_plan(n0, p->sign);
    std::vector<oracle_cplx> tile(n0 * kRun), line(n0), res(n0);
    std::vector<oracle_cplx *> row(n0);
    for (size_t x = 0; x < n0; ++x) {
      ptrdiff_t owner_n0, owner_start;
      int owner = (int)(x / (size_t)((p->n0 + g_ranks - 1) / g_ranks));
      slab(p->n0, owner, &owner_n0, &owner_start);
      row[x] = reinterpret_cast<oracle_cplx *>(g_sh->plans[p->id][owner].out) +
               (x - (size_t)owner_start) * plane;
    }
    for (size_t c = c0; c < c1; c += kRun) {
      const size_t w = (c1 - c) < kRun ? (c1 - c) : kRun;
      for (size_t x = 0; x < n0; ++x)
        std::memcpy(&tile[x * kRun], row[x] + c, sizeof(oracle_cplx) * w);
      for (size_t b = 0; b < w; ++b) {
        for (size_t x = 0; x < n0; ++x) line[x] = tile[x * kRun + b];
        oracle_dft1d_exec(d, line.data(), 1, res.data(), 1);
        for (size_t x = 0; x < n0; ++x) tile[x * kRun + b] = res[x];
      }
      for (size_t x = 0; x < n0; ++x)
        std::memcpy(row[x] + c, &tile[x * kRun], sizeof(oracle_cplx) * w);
    }
    oracle_dft1d_free(d);
  }
  barrier();
  g_fft_seconds += now_s() - t0;
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
