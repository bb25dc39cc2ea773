// noalloc.cu -- vpfft_solve_constrained_constitutive_noalloc: the batched
// constrained constitutive solve with no device memory allocation.
//
// Who needs it: a macro-scale driver (a finite-element code that calls the
// crystal-plasticity point solve at every integration point of every global
// Newton iteration) usually hands the whole device to its own memory pool,
// so a cudaMalloc inside the call can fail, and each cudaFree synchronises
// the device and stalls the driver's other streams.  This entry point stages
// the caller's host arrays in a fixed device array that exists as long as the
// library is loaded, so it calls neither cudaMalloc nor cudaFree nor any
// library routine that allocates.
//
// Limits and rules:
//  * at most VPFFT_NOALLOC_MAX_POINTS points per call (larger n is refused
//    with VPFFT_ERR_UNSUPPORTED_SIZE; split the batch);
//  * the first call on each device sets up: it looks up the array's device
//    address (cudaGetSymbolAddress, with that device current) and makes the
//    CUDA runtime load the array and the kernels this call launches.  Under
//    the runtime's default lazy module loading that load is what allocates
//    (about 3 MiB per device), so make the first call -- one with n = 0 is
//    enough -- before the caller's memory pool takes the device; later calls
//    allocate nothing;
//  * every copy and launch of a call runs on the legacy default stream, so no
//    call may overlap a stream capture anywhere in the process, on any
//    device, and a call is ordered after the work of the caller's blocking
//    streams (only streams made with cudaStreamNonBlocking are not stalled);
//  * there is one array per device per process, so two calls that overlapped
//    in time would race on it: the entry point holds a process-wide lock for
//    the whole call, and concurrent callers run one after another;
//  * the array keeps the previous call's contents; the only value that must
//    start at zero (the count of non-converged points) is cleared each call;
//  * the call synchronises the legacy default stream, not the whole device,
//    and does not return until the results are on the host.
//  * the looked-up address belongs to the device's primary context: after a
//    cudaDeviceReset the library (its grids, batches and this entry point)
//    must not be used again in the process.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/vpfft_capi.h"
#include "kernels.h"

namespace vpfft {
vpfft_status lib_fail(vpfft_status s, const std::string& msg);
}

namespace {

constexpr int kMaxPoints = VPFFT_NOALLOC_MAX_POINTS;
constexpr int kMaxDevices = 64;
// doubles per point: stress0 5, schmid 60, crss 12, lambda 5, d~ 5, out 5, NR error 1
constexpr long long kOffS0 = 0;
constexpr long long kOffSchmid = kOffS0 + 5LL * kMaxPoints;
constexpr long long kOffCrss = kOffSchmid + 60LL * kMaxPoints;
constexpr long long kOffLambda = kOffCrss + 12LL * kMaxPoints;
constexpr long long kOffDtilde = kOffLambda + 5LL * kMaxPoints;
constexpr long long kOffOut = kOffDtilde + 5LL * kMaxPoints;
constexpr long long kOffErr = kOffOut + 5LL * kMaxPoints;
constexpr long long kOffCount = kOffErr + 1LL * kMaxPoints;  // one 64-bit counter
constexpr long long kScratchDoubles = kOffCount + 32;       // counter + padding

// 93 doubles x 4096 points + 256 bytes = 2.9 MiB per device.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_noalloc_lock;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Points whose final NR error is not below eps (or is NaN) -- the batch's
// "not converged" count, accumulated into the scratch counter.
__global__ void k_count_not_converged(const double* __restrict__ err, int n, double eps,
                                      unsigned long long* count) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const bool bad = v < n && !(err[v] < eps);
  const unsigned mask = __ballot_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0 && mask) atomicAdd(count, (unsigned long long)__popc(mask));
}

vpfft_status cuda_fail(cudaError_t e, const char* what) {
  return vpfft::lib_fail(e == cudaErrorMemoryAllocation ? VPFFT_ERR_OUT_OF_MEMORY : VPFFT_ERR_CUDA,
                         std::string(what) + ": " + cudaGetErrorString(e));
}

#define NA_CK(call)                                   \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

// Device address of the scratch array on the current device (looked up once
// per device; the caller holds g_noalloc_lock).
vpfft_status scratch_for_current_device(double** out) {
  int dev = -1;
  NA_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return vpfft::lib_fail(VPFFT_ERR_UNSUPPORTED_SIZE, "device ordinal out of range");
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    NA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    // load this unit's count kernel and the solve kernels now, not at the
    // first launch of a later call
    cudaFuncAttributes attr;
    NA_CK(cudaFuncGetAttributes(&attr, k_count_not_converged));
    NA_CK(vpfft::load_solvers_kernels());
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return VPFFT_OK;
}

}  // namespace

extern "C" vpfft_status vpfft_solve_constrained_constitutive_noalloc(
    int n, const double* s0, const double* schmid, const double* crss, const vpfft_material* m,
    const double edot[5], const double* lambda, const double* dtilde, const double L0[25],
    double eps, double max_rss, int max_iter, double* out, double* nr_error,
    int64_t* not_converged) {
  if (n < 0 || !s0 || !schmid || !crss || !m || !edot || !lambda || !dtilde || !L0 || !out)
    return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (n > kMaxPoints)
    return vpfft::lib_fail(VPFFT_ERR_UNSUPPORTED_SIZE,
                           "n = " + std::to_string(n) + " exceeds the no-allocation scratch of " +
                               std::to_string(kMaxPoints) +
                               " points; split the batch or call "
                               "vpfft_solve_constrained_constitutive");
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt <= 0) {
    cudaGetLastError();
    return vpfft::lib_fail(VPFFT_ERR_NO_DEVICE,
                           "no CUDA device available (vpfft_b200 has no CPU fallback)");
  }
  if (not_converged) *not_converged = 0;

  std::lock_guard<std::mutex> lock(g_noalloc_lock);
  double* base = nullptr;
  if (vpfft_status s = scratch_for_current_device(&base)) return s;
  if (n == 0) return VPFFT_OK;
  double* d_s0 = base + kOffS0;
  double* d_schmid = base + kOffSchmid;
  double* d_crss = base + kOffCrss;
  double* d_lambda = base + kOffLambda;
  double* d_dtilde = base + kOffDtilde;
  double* d_out = base + kOffOut;
  double* d_err = base + kOffErr;
  auto* d_count = reinterpret_cast<unsigned long long*>(base + kOffCount);

  const size_t b5 = sizeof(double) * 5 * (size_t)n;
  NA_CK(cudaMemcpy(d_s0, s0, b5, cudaMemcpyHostToDevice));
  NA_CK(cudaMemcpy(d_schmid, schmid, sizeof(double) * 60 * (size_t)n, cudaMemcpyHostToDevice));
  NA_CK(cudaMemcpy(d_crss, crss, sizeof(double) * 12 * (size_t)n, cudaMemcpyHostToDevice));
  NA_CK(cudaMemcpy(d_lambda, lambda, b5, cudaMemcpyHostToDevice));
  NA_CK(cudaMemcpy(d_dtilde, dtilde, b5, cudaMemcpyHostToDevice));
  NA_CK(cudaMemset(d_count, 0, sizeof(unsigned long long)));

  vpfft::MaterialParams mp;
  for (int k = 0; k < vpfft::kNS; ++k) {
    mp.gdot[k] = m->gamma_dot_base[k];
    mp.nexp[k] = m->rate_sensitivity[k];
  }
  vpfft::launch_solvers_constrained(n, d_s0, d_schmid, d_crss, mp, edot, d_lambda, d_dtilde, L0,
                                    eps, max_rss, max_iter, d_out, d_err, nullptr);
  NA_CK(cudaGetLastError());
  k_count_not_converged<<<(n + 255) / 256, 256>>>(d_err, n, eps, d_count);
  NA_CK(cudaGetLastError());
  // the copies, the solve and the count all ran on the legacy default stream:
  // wait for that stream only, not for the caller's own (non-blocking) streams
  NA_CK(cudaStreamSynchronize(0));
  NA_CK(cudaMemcpy(out, d_out, b5, cudaMemcpyDeviceToHost));
  if (nr_error) NA_CK(cudaMemcpy(nr_error, d_err, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (not_converged) {
    unsigned long long c = 0;
    NA_CK(cudaMemcpy(&c, d_count, sizeof(c), cudaMemcpyDeviceToHost));
    *not_converged = (int64_t)c;
  }
  return VPFFT_OK;
}
