// shim_runtime.cpp -- implementations of the single-process MPI and FFTW
// stand-ins declared in mpi.h / fftw3-mpi.h, plus the observation hooks.
// Test-oracle infrastructure only.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../common/dft.h"
#include "fftw3-mpi.h"
#include "mpi.h"
#include "shim_hooks.h"

namespace {
vpfft_shim_exec_hook g_exec_hook = nullptr;
void *g_exec_user = nullptr;
vpfft_shim_allreduce_hook g_ar_hook = nullptr;
void *g_ar_user = nullptr;
long g_exec_count = 0;
long g_ar_count = 0;

[[noreturn]] void die(const char *what) {
  std::fprintf(stderr, "[vpfft shim] %s is not available in the single-process stand-in\n", what);
  std::abort();
}
}  // namespace

struct vpfft_shim_plan_s {
  ptrdiff_t n0, n1, n2;
  fftw_complex *in;
  fftw_complex *out;
  int sign;
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
long vpfft_shim_exec_count(void) { return g_exec_count; }
long vpfft_shim_allreduce_count(void) { return g_ar_count; }

// ---------------------------------------------------------------- MPI
int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int *size) {
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op,
                  MPI_Comm) {
  size_t esz = dt == MPI_DOUBLE ? sizeof(double)
               : dt == MPI_FLOAT ? sizeof(float)
               : dt == MPI_INT   ? sizeof(int)
                                 : 1;
  std::memmove(recvbuf, sendbuf, esz * (size_t)count);
  ++g_ar_count;
  if (g_ar_hook && dt == MPI_DOUBLE) g_ar_hook((const double *)recvbuf, count, g_ar_user);
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { die("MPI_Send"); }
int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { die("MPI_Recv"); }
int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  die("MPI_Isend");
}
int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { die("MPI_Irecv"); }
int MPI_Wait(MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }

// ---------------------------------------------------------------- FFTW
void fftw_mpi_init(void) {}
void fftw_cleanup(void) {}

ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start) {
  *local_n0 = n0;
  *local_0_start = 0;
  return n0 * n1 * n2;
}

void *fftw_malloc(size_t n) {
  void *p = nullptr;
  if (posix_memalign(&p, 64, n ? n : 1) != 0) return nullptr;
  return p;
}
fftw_complex *fftw_alloc_complex(size_t n) {
  return (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
}
void fftw_free(void *p) { std::free(p); }

fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in,
                               fftw_complex *out, MPI_Comm, int sign, unsigned) {
  auto *p = new vpfft_shim_plan_s{n0, n1, n2, in, out, sign};
  return p;
}

void fftw_execute(const fftw_plan p) {
  ++g_exec_count;
  const long total = (long)(p->n0 * p->n1 * p->n2);
  if (g_exec_hook) g_exec_hook(p->sign, p->in, total, g_exec_user);
  if (p->out != p->in) std::memcpy(p->out, p->in, sizeof(fftw_complex) * (size_t)total);
  oracle_dft3d_inplace(reinterpret_cast<oracle_cplx *>(p->out), (size_t)p->n0, (size_t)p->n1,
                       (size_t)p->n2, p->sign);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
