// capi.cu -- host implementation of the C ABI declared in include/vpfft_capi.h.
//
// A vpfft_grid owns the device-resident state of one RVE (representative
// volume element): orientation, stress, Lagrange multiplier, CRSS and
// accumulated shear as component-major arrays, one real work field (P / d~),
// the half spectrum and the twiddle tables, plus a CUDA stream.  The host only
// sequences kernels; all per-voxel and per-wave-vector arithmetic runs on the
// device.  There is no CPU fallback: without a CUDA device every entry point
// that needs one returns VPFFT_ERR_NO_DEVICE.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <map>
#include <mutex>
#include <tuple>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "grid.h"

using namespace vpfft;
using namespace vpfft::grid_ops;

// NVTX range over one phase of a solve (initialisation, reference medium,
// fixed-point loop, post-increment update), visible in Nsight timelines.
struct PhaseRange {
  explicit PhaseRange(const char* name) { nvtxRangePushA(name); }
  ~PhaseRange() { nvtxRangePop(); }
  PhaseRange(const PhaseRange&) = delete;
  PhaseRange& operator=(const PhaseRange&) = delete;
};

static_assert(VPFFT_STATUS_MAX_RSS_TINY == vpfft::kStatusMaxRssTiny &&
                  VPFFT_STATUS_NONFINITE == vpfft::kStatusNonFinite &&
                  VPFFT_STATUS_DEVICE_TIMEOUT == vpfft::kStatusDeviceTimeout,
              "device status bits and the C ABI's bits agree");

namespace {

thread_local std::string g_lib_err;

size_t elem_size(vpfft_precision p) { return p == VPFFT_PREC_FP64 ? sizeof(double) : sizeof(float); }

vpfft_status fail(vpfft_grid* g, vpfft_status s, const std::string& msg) {
  if (g)
    g->err = msg;
  else
    g_lib_err = msg;
  return s;
}

#define CK(g, call)                                                                       \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      return fail((g), e_ == cudaErrorMemoryAllocation ? VPFFT_ERR_OUT_OF_MEMORY          \
                                                       : VPFFT_ERR_CUDA,                  \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                    \
    }                                                                                     \
  } while (0)

#define CKL(g) CK(g, cudaGetLastError())

vpfft_status busy(vpfft_grid* g) {
  return fail(g, VPFFT_ERR_BUSY, "the grid has a request in flight in a batch");
}

vpfft_status need_device(vpfft_grid* g) {
  int cnt = 0;
  cudaError_t e = cudaGetDeviceCount(&cnt);
  if (e != cudaSuccess || cnt <= 0) {
    cudaGetLastError();
    return fail(g, VPFFT_ERR_NO_DEVICE,
                "no CUDA device available (vpfft_b200 has no CPU fallback)");
  }
  return VPFFT_OK;
}

// twiddle table exp(-2 pi i e / n), e in [0, n), from long double
template <typename R>
std::vector<R> twiddles(int n) {
  std::vector<R> t(2 * (size_t)n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int e = 0; e < n; ++e) {
    const long double a = two_pi * (long double)e / (long double)n;
    t[2 * e] = (R)cosl(a);
    t[2 * e + 1] = (R)(-sinl(a));
  }
  return t;
}

// LU with row pivoting inverse of a column-major 5x5 (host, FP64)
void inverse5_host(const double* a, double* out) {
  double lu[5][5];
  int perm[5];
  for (int i = 0; i < 5; ++i) {
    perm[i] = i;
    for (int j = 0; j < 5; ++j) lu[i][j] = a[j * 5 + i];
  }
  for (int k = 0; k < 5; ++k) {
    int piv = k;
    double best = std::fabs(lu[k][k]);
    for (int i = k + 1; i < 5; ++i)
      if (std::fabs(lu[i][k]) > best) {
        best = std::fabs(lu[i][k]);
        piv = i;
      }
    if (piv != k) {
      for (int j = 0; j < 5; ++j) std::swap(lu[k][j], lu[piv][j]);
      std::swap(perm[k], perm[piv]);
    }
    for (int i = k + 1; i < 5; ++i) {
      lu[i][k] /= lu[k][k];
      for (int j = k + 1; j < 5; ++j) lu[i][j] -= lu[i][k] * lu[k][j];
    }
  }
  for (int col = 0; col < 5; ++col) {
    double y[5];
    for (int i = 0; i < 5; ++i) {
      double s = (perm[i] == col) ? 1.0 : 0.0;
      for (int j = 0; j < i; ++j) s -= lu[i][j] * y[j];
      y[i] = s;
    }
    for (int i = 4; i >= 0; --i) {
      double s = y[i];
      for (int j = i + 1; j < 5; ++j) s -= lu[i][j] * y[j];
      y[i] = s / lu[i][i];
    }
    for (int i = 0; i < 5; ++i) out[col * 5 + i] = y[i];
  }
}

}  // namespace

void vpfft::inverse5_colmajor(const double* a, double* out) { inverse5_host(a, out); }

// Library-level error slot (vpfft_last_error(NULL)) for entry points in other files.
namespace vpfft {
vpfft_status lib_fail(vpfft_status s, const std::string& msg) { return fail(nullptr, s, msg); }
}  // namespace vpfft

namespace {

}  // namespace

namespace vpfft {
namespace grid_ops {

VoxelParams voxel_params(const vpfft_grid* g, const double edot[5]) {
  VoxelParams p{};
  p.n = g->n;
  for (int c = 0; c < 5; ++c) p.edot[c] = edot[c];
  for (int k = 0; k < 25; ++k) p.L0[k] = g->L0[k];
  p.mat = mat_params(g->mat);
  for (int k = 0; k < kNS; ++k) p.crss[k] = g->mat.crss[k];
  p.nr_eps = g->opt.nr_epsilon;
  p.nr_max_rss = g->opt.nr_max_resolved;
  p.nr_max_iter = g->opt.nr_max_iter;
  p.init_max_iter = g->opt.init_nr_max_iter;
  p.init_eps = g->opt.init_nr_epsilon;
  // MaterialGrid.cpp:162-166
  int min_n = g->mat.rate_sensitivity[0];
  for (int k = 1; k < kNS; ++k) min_n = std::min(min_n, (int)g->mat.rate_sensitivity[k]);
  const double ee = edot[0] * edot[0] + edot[1] * edot[1] + edot[2] * edot[2] +
                    edot[3] * edot[3] + edot[4] * edot[4];
  double imposed = 2.0 * std::pow(ee / g->mat.gamma_dot_base[0], (double)(1. / (float)min_n));
  p.imposed_max_rss = (2.0 < imposed) ? imposed : 2.0;
  return p;
}

// Launch constants of the Newton kernels: the initialisation solve
// (InitializeComputation, MaterialGrid.cpp:159-166) or the loop solve (909-911).
NRParams nr_params(const vpfft_grid* g, const double edot[5], bool init) {
  VoxelParams v = voxel_params(g, edot);
  NRParams p{};
  p.n = g->n;
  for (int c = 0; c < 5; ++c) p.edot[c] = edot[c];
  for (int k = 0; k < 25; ++k) p.L0[k] = g->L0[k];
  for (int k = 0; k < 15; ++k) p.L0inv[k] = g->L0inv_sym[k];
  for (int q = 0; q < kNS; ++q) {
    p.gdot[q] = g->mat.gamma_dot_base[q];
    p.nexp[q] = g->mat.rate_sensitivity[q];
    p.crss[q] = g->mat.crss[q];
    p.icrss[q] = 1.0 / g->mat.crss[q];
  }
  if (init) {
    p.eps = g->opt.init_nr_epsilon;
    p.max_rss = v.imposed_max_rss;
    p.max_iter = g->opt.init_nr_max_iter;
  } else {
    p.eps = g->opt.nr_epsilon;
    p.max_rss = g->opt.nr_max_resolved;
    p.max_iter = g->opt.nr_max_iter;
  }
  set_fp32_copies(p);
  p.cert2_f = (float)(g->opt.mixed_certify_step * g->opt.mixed_certify_step);
  return p;
}

PostParams post_params(const vpfft_grid* g, double dt) {
  PostParams p{};
  p.n = g->n;
  p.dt = dt;
  p.mat = mat_params(g->mat);
  for (int k = 0; k < kNS; ++k) {
    p.crss[k] = g->mat.crss[k];
    p.tau0[k] = g->mat.tau0[k];
    p.tau1[k] = g->mat.tau1[k];
    p.theta0[k] = g->mat.theta0[k];
    p.theta1[k] = g->mat.theta1[k];
  }
  for (int k = 0; k < kNS * kNS; ++k) p.H[k] = g->mat.hardening[k];
  return p;
}

vpfft_status grid_fail(vpfft_grid* g, vpfft_status s, const std::string& msg) {
  return fail(g, s, msg);
}

// The operators formed from L0: inverse(-L0) for the Nyquist planes
// (StrainRateEvolutionWithFFT, MaterialGrid.cpp:628-632) and the symmetric
// part of L0^-1 for the Newton step.
void derive_L0_inverses(vpfft_grid* g) {
  double negL[25];
  for (int k = 0; k < 25; ++k) negL[k] = -g->L0[k];
  inverse5_host(negL, g->Linv);
  double inv[25];
  inverse5_host(g->L0, inv);
  for (int i = 0; i < 5; ++i)
    for (int j = i; j < 5; ++j) g->L0inv_sym[sym5(i, j)] = 0.5 * (inv[j * 5 + i] + inv[i * 5 + j]);
}

vpfft_status finish_ref_medium(vpfft_grid* g, const double sums[25]) {
  const double N = (double)g->n;
  for (int k = 0; k < 25; ++k) {
    double m = sums[k] / N;                        // mean of the per-voxel inverses (H4)
    double tmp = m * (double)g->nx;                // * DimXLocal   (MaterialGrid.cpp:262)
    m = tmp / (double)g->nx;                       // / DimX        (269)
    g->L0[k] = std::fabs(m) < 1e-10 ? 0.0 : m;     // NormalizeValues (LinearAlgebra.h:605-613)
  }
  for (int k = 0; k < 25; ++k)
    if (!std::isfinite(g->L0[k]))
      return fail(g, VPFFT_ERR_NONFINITE, "reference medium is not finite (singular voxel compliance)");
  derive_L0_inverses(g);
  g->have_L0 = true;
  return VPFFT_OK;
}

void finish_post(vpfft_grid* g, const double edot[5], double dt) {
  g->crss_per_voxel = true;
  // UpdateVoxelLength (MaterialGrid.cpp:1190-1196) with Edot as a 3x3 matrix
  double E[9];
  vpfft_matrix_from_edot(edot, E);
  g->h[0] *= (1.0 + E[0] * dt);
  g->h[1] *= (1.0 + E[4] * dt);
  g->h[2] *= (1.0 + E[8] * dt);
}

// like the reference's do { } while (StepsTaken < NumMaxIterations && ...)
// (MaterialGrid.cpp:930-1068), at least one iteration always runs
IterCtrl loop_ctrl(const vpfft_grid* g, const double edot[5], int max_iter, double eps) {
  IterCtrl h{};
  h.iter = 0;
  h.done = 0;
  h.max_iter = max_iter;
  h.eps = eps;
  h.edot_norm = std::sqrt(edot[0] * edot[0] + edot[1] * edot[1] + edot[2] * edot[2] +
                          edot[3] * edot[3] + edot[4] * edot[4]);
  h.n_voxels = (double)g->n;
  return h;
}

vpfft_status ensure_hist(vpfft_grid* g, int max_iter) {
  if (std::max(max_iter, 1) > g->hist_cap) {
    if (g->hist) cudaFree(g->hist);
    g->hist = nullptr;
    CK(g, cudaMalloc(&g->hist, sizeof(double) * 12 * (size_t)std::max(max_iter, 1)));
    g->hist_cap = std::max(max_iter, 1);
  }
  return VPFFT_OK;
}

vpfft_status ensure_crss_array(vpfft_grid* g) {
  const size_t es = g->prec == VPFFT_PREC_FP64 ? sizeof(double) : sizeof(float);
  if (!g->crss) CK(g, cudaMalloc(&g->crss, es * (size_t)g->n * kNS));
  return VPFFT_OK;
}

}  // namespace grid_ops
}  // namespace vpfft

namespace {

// The spectrum buffers of the single-grid path: allocated on first use and
// kept (a grid solved only through a batch never allocates them).
vpfft_status ensure_spectrum(vpfft_grid* g) {
  const size_t b = spectrum_bytes(g);
  if (!g->X) CK(g, cudaMalloc(&g->X, b));
  if (!g->X2) CK(g, cudaMalloc(&g->X2, b));
  return VPFFT_OK;
}

template <typename S>
vpfft_status upload_twiddles(vpfft_grid* g) {
  const int dims[3] = {g->nx, g->ny, g->nz};
  void** dst[3] = {&g->twx, &g->twy, &g->twz};
  for (int a = 0; a < 3; ++a) {
    std::vector<S> t = twiddles<S>(dims[a]);
    CK(g, cudaMalloc(dst[a], t.size() * sizeof(S)));
    CK(g, cudaMemcpy(*dst[a], t.data(), t.size() * sizeof(S), cudaMemcpyHostToDevice));
  }
  return VPFFT_OK;
}

void free_grid_buffers(vpfft_grid* g) {
  void* ptrs[] = {g->R,   g->sigma, g->lambda, g->work,     g->dkeep, g->crss,
                  g->acc, g->X,     g->X2,     g->twx,      g->twy,   g->twz,
                  g->partials, g->sum25, g->ctrl, g->hist, g->staging, g->gtab};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (g->h_ctrl) cudaFreeHost(g->h_ctrl);
  if (g->loop_graph) cudaGraphExecDestroy(g->loop_graph);
  for (cudaEvent_t e : g->ev) cudaEventDestroy(e);
  g->ev.clear();
  if (g->stream) cudaStreamDestroy(g->stream);
}

// Lines up to 512 points keep every FFT tile (5 components, FP64, ping-pong
// buffers) inside one block's shared memory.
bool valid_dim(int n) {
  LinePlan p;
  return n >= 1 && n <= 512 && make_line_plan(n, &p);
}

// The staging buffer holds one voxel-major FP64 field (up to 12 values per
// voxel); it is allocated on first use and kept, so field uploads and
// read-backs do not allocate.
vpfft_status ensure_staging(vpfft_grid* g) {
  if (!g->staging) CK(g, cudaMalloc(&g->staging, sizeof(double) * (size_t)g->n * 12));
  return VPFFT_OK;
}

template <typename S>
vpfft_status to_device_field(vpfft_grid* g, const double* host_or_dev, bool is_device, S* dst,
                             int width) {
  const size_t bytes = sizeof(double) * (size_t)g->n * width;
  vpfft_status s = ensure_staging(g);
  if (s != VPFFT_OK) return s;
  CK(g, cudaMemcpyAsync(g->staging, host_or_dev, bytes,
                        is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, g->stream));
  g->launches += launch_to_soa<S>(g->staging, dst, g->n, width, g->stream);
  CKL(g);
  CK(g, cudaStreamSynchronize(g->stream));
  return VPFFT_OK;
}

template <typename S>
vpfft_status from_device_field(vpfft_grid* g, const S* src, int width, double* host) {
  const size_t bytes = sizeof(double) * (size_t)g->n * width;
  vpfft_status s = ensure_staging(g);
  if (s != VPFFT_OK) return s;
  g->launches += launch_from_soa<S>(src, g->staging, g->n, width, g->stream);
  CKL(g);
  CK(g, cudaMemcpyAsync(host, g->staging, bytes, cudaMemcpyDeviceToHost, g->stream));
  CK(g, cudaStreamSynchronize(g->stream));
  return VPFFT_OK;
}


// ---------------------------------------------------------------- phases
template <typename S>
vpfft_status do_init(vpfft_grid* g, const double edot[5]) {
  PhaseRange range("vpfft InitializeComputation");
  if (!g->fields_set) return fail(g, VPFFT_ERR_NOT_INITIALIZED, "fields not set");
  NRParams p = nr_params(g, edot, true);
  IterCtrl h{};
  h.n_voxels = (double)g->n;
  CK(g, cudaMemcpyAsync(g->ctrl, &h, sizeof(h), cudaMemcpyHostToDevice, g->stream));
  g->launches += launch_init<S>(p, fields<S>(g), g->ctrl, g->stream);
  CKL(g);
  CK(g, cudaMemcpyAsync(g->h_ctrl, g->ctrl, sizeof(IterCtrl), cudaMemcpyDeviceToHost, g->stream));
  CK(g, cudaStreamSynchronize(g->stream));
  if (g->h_ctrl->status & kStatusNonFinite)
    return fail(g, VPFFT_ERR_NONFINITE,
                "initial guess is not finite (zero or non-finite macroscopic strain rate)");
  if (g->h_ctrl->status & kStatusMaxRssTiny)
    return fail(g, VPFFT_ERR_MAX_RSS_TINY, "max resolved shear stress < 1e-10 in the initial guess");
  for (int c = 0; c < 5; ++c) g->last_edot[c] = edot[c];
  return VPFFT_OK;
}

template <typename S>
vpfft_status do_ref_medium(vpfft_grid* g, double* L0_out) {
  PhaseRange range("vpfft BuildLinearRefMediumStiffness");
  VoxelParams p = voxel_params(g, g->last_edot);
  g->launches += launch_ref_medium<S>(p, fields<S>(g), g->partials, g->sum25, g->stream);
  CKL(g);
  double sums[25];
  CK(g, cudaMemcpyAsync(sums, g->sum25, sizeof(sums), cudaMemcpyDeviceToHost, g->stream));
  CK(g, cudaStreamSynchronize(g->stream));
  if (vpfft_status r = finish_ref_medium(g, sums)) return r;
  if (L0_out) std::memcpy(L0_out, g->L0, sizeof(g->L0));
  return VPFFT_OK;
}

// ---- the x pass's Green operator: computed per wave vector or stored.
// A stored table costs kGreenStored values per wave vector of the half
// spectrum in HBM traffic per iteration against the ~200 operations of
// (V L0 V^T)^-1 and 1/(k.C k) recomputed per wave vector.  Both give the same
// bits; which is faster depends on the size (a table that stays in L2 can
// win), so it is timed: the first solve of a size (per device and precision) times the
// x pass both ways on the spare spectrum buffer A (free between the forward y
// pass and the inverse one; not read before the next z pass rewrites it) and
// keeps the faster.  Tables above kGreenTableMax bytes are not tried.
constexpr size_t kGreenTableMax = 512ull << 20;
std::mutex g_green_mu;
std::map<std::tuple<int, int, int, int, int>, std::pair<int, std::pair<double, double>>>
    g_green_choice;  // (device, bytes, nx, ny, nz) -> (mode, (ms computed, ms stored))

template <typename S>
size_t green_table_bytes(const vpfft_grid* g) {
  return sizeof(S) * kGreenStored * (size_t)g->nh * g->ny * g->nx;
}

template <typename S>
vpfft_status time_x_pass(vpfft_grid* g, const Spectral<S>& sp, const GreenParams<S>& gp,
                         const S* tab, double* ms) {
  cudaEvent_t e0, e1;
  CK(g, cudaEventCreate(&e0));
  CK(g, cudaEventCreate(&e1));
  launch_x_pass<S>(sp, gp, tab, g->X, 5, g->stream);  // warm-up
  CK(g, cudaEventRecord(e0, g->stream));
  constexpr int kReps = 3;
  for (int r = 0; r < kReps; ++r) launch_x_pass<S>(sp, gp, tab, g->X, 5, g->stream);
  CK(g, cudaEventRecord(e1, g->stream));
  CKL(g);
  CK(g, cudaEventSynchronize(e1));
  float t = 0.f;
  CK(g, cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = (double)t / kReps;
  return VPFFT_OK;
}

// Picks the operator (if not done for this grid) and, when it is the stored
// one, rebuilds the table for the current L0 and voxel lengths.
template <typename S>
vpfft_status prepare_green(vpfft_grid* g, const Spectral<S>& sp, const GreenParams<S>& gp) {
  const size_t bytes = green_table_bytes<S>(g);
  auto ensure_table = [&]() -> vpfft_status {
    if (!g->gtab) CK(g, cudaMalloc(&g->gtab, bytes));
    g->launches += launch_green_table<S>(gp, (S*)g->gtab, g->nh, g->stream);
    CKL(g);
    return VPFFT_OK;
  };
  if (g->green_mode == 0) {
    const int opt = g->opt.green_operator;
    if (opt == 1 || opt == 2) {
      g->green_mode = opt;
    } else if (bytes > kGreenTableMax) {
      g->green_mode = 1;
    } else {
      const auto key = std::make_tuple(g->device, (int)sizeof(S), g->nx, g->ny, g->nz);
      bool cached = false;
      {
        std::lock_guard<std::mutex> lk(g_green_mu);
        auto it = g_green_choice.find(key);
        if (it != g_green_choice.end()) {
          g->green_mode = it->second.first;
          g->green_ms[0] = it->second.second.first;
          g->green_ms[1] = it->second.second.second;
          cached = true;
        }
      }
      if (!cached) {
        if (vpfft_status r = ensure_table()) return r;
        if (vpfft_status r = time_x_pass<S>(g, sp, gp, nullptr, &g->green_ms[0])) return r;
        if (vpfft_status r = time_x_pass<S>(g, sp, gp, (const S*)g->gtab, &g->green_ms[1]))
          return r;
        g->green_mode = g->green_ms[1] < g->green_ms[0] ? 2 : 1;
        std::lock_guard<std::mutex> lk(g_green_mu);
        g_green_choice.emplace(key, std::make_pair(g->green_mode,
                                                   std::make_pair(g->green_ms[0], g->green_ms[1])));
      }
    }
  }
  if (g->green_mode == 2) return ensure_table();
  if (g->gtab) {  // computed operator chosen: the table is not needed
    CK(g, cudaStreamSynchronize(g->stream));
    cudaFree(g->gtab);
    g->gtab = nullptr;
  }
  return VPFFT_OK;
}

template <typename S>
vpfft_status do_fixed_point(vpfft_grid* g, const double edot[5], int max_iter, double eps,
                            double* history, vpfft_stats* st) {
  PhaseRange range("vpfft fixed-point loop");
  if (!g->have_L0) return fail(g, VPFFT_ERR_NOT_INITIALIZED, "reference medium not built");
  if (vpfft_status r = ensure_hist(g, max_iter)) return r;
  if (vpfft_status r = ensure_spectrum(g)) return r;
  IterCtrl h = loop_ctrl(g, edot, max_iter, eps);
  CK(g, cudaMemcpyAsync(g->ctrl, &h, sizeof(h), cudaMemcpyHostToDevice, g->stream));
  NRParams p = nr_params(g, edot, false);
  GreenParams<S> gp = green_params<S>(g->nx, g->ny, g->nz, g->h, g->L0, g->Linv);
  Spectral<S> sp = spectral<S>(g, g->X, g->X2);
  if (vpfft_status r = prepare_green<S>(g, sp, gp)) return r;
  const S* gtab = g->green_mode == 2 ? (const S*)g->gtab : nullptr;
  FieldPtrs<S> f = fields<S>(g);
  const int batch = g->n >= (1LL << 21) ? 4 : 16;
  constexpr int kEv = 8;  // events per iteration when profiling
  if (g->profile && (int)g->ev.size() < batch * kEv) {
    while ((int)g->ev.size() < batch * kEv) {
      cudaEvent_t e;
      CK(g, cudaEventCreate(&e));
      g->ev.push_back(e);
    }
  }
  // The first chunk runs eagerly; when the loop goes on, the chunk is captured
  // once into a CUDA graph (updating the grid's executable graph in place when
  // only the parameters changed) and replayed: the kernels return at once when
  // the device-side control block says the loop is done.  Profiling keeps the
  // eager launches (events between the kernels).
  auto enqueue_chunk = [&](bool profiled) {
    int n = 0;
    for (int b = 0; b < batch; ++b) {
      cudaEvent_t* e = profiled ? &g->ev[(size_t)b * kEv] : nullptr;
      n += launch_spectral_iteration<S>(sp, gp, (S*)g->work, g->ctrl, g->stream, 5, e, gtab);
      n += launch_nr_update<S>(p, f, g->partials, g->ctrl, g->hist, g->stream,
                               e ? e + 6 : nullptr);
    }
    return n;
  };
  int done_before = 0, chunk = 0, chunk_launches = 0;
  bool graph_ready = false;
  for (;;) {
    if (g->profile || chunk == 0) {
      chunk_launches = enqueue_chunk(g->profile);
    } else {
      if (!graph_ready) {
        cudaGraph_t graph = nullptr;
        CK(g, cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_chunk(false);
        CK(g, cudaStreamEndCapture(g->stream, &graph));
        bool updated = false;
        if (g->loop_graph) {
          cudaGraphExecUpdateResultInfo info;
          updated = cudaGraphExecUpdate(g->loop_graph, graph, &info) == cudaSuccess;
          if (!updated) {
            cudaGetLastError();
            cudaGraphExecDestroy(g->loop_graph);
            g->loop_graph = nullptr;
          }
        }
        cudaError_t e = updated ? cudaSuccess : cudaGraphInstantiate(&g->loop_graph, graph, 0);
        cudaGraphDestroy(graph);
        CK(g, e);
        graph_ready = true;
      }
      CK(g, cudaGraphLaunch(g->loop_graph, g->stream));
    }
    g->launches += chunk_launches;
    ++chunk;
    CKL(g);
    CK(g, cudaMemcpyAsync(g->h_ctrl, g->ctrl, sizeof(IterCtrl), cudaMemcpyDeviceToHost, g->stream));
    CK(g, cudaStreamSynchronize(g->stream));
    if (g->profile) {
      // only the iterations that ran (the rest returned at once on `done`)
      const int ran = g->h_ctrl->iter - done_before;
      for (int b = 0; b < ran && b < batch; ++b) {
        const cudaEvent_t* e = &g->ev[(size_t)b * kEv];
        for (int k = 0; k < VPFFT_NUM_PHASES; ++k) {
          float ms = 0.f;
          CK(g, cudaEventElapsedTime(&ms, e[k], e[k + 1]));
          g->phase_ms[k] += ms;
          g->phase_n[k] += 1;
        }
      }
    }
    done_before = g->h_ctrl->iter;
    if (g->h_ctrl->done) break;
  }
  const IterCtrl& c = *g->h_ctrl;
  if (history && c.iter > 0)
    CK(g, cudaMemcpy(history, g->hist, sizeof(double) * 12 * (size_t)c.iter, cudaMemcpyDeviceToHost));
  if (st) {
    st->iterations = c.iter;
    st->stress_error = c.last[10];
    st->strain_rate_error = c.last[11];
    st->converged = (c.last[10] <= eps && c.last[11] <= eps) ? 1 : 0;
    for (int k = 0; k < 5; ++k) st->avg_strain_rate[k] = c.last[5 + k];
    st->nr_not_converged = (int64_t)c.nr_capped;
    st->nr_fp64_steps = (int64_t)c.nr_fp64;
    st->status_bits = c.status | (st->converged ? 0 : VPFFT_STATUS_LOOP_NOT_CONVERGED) |
                      (c.nr_capped ? VPFFT_STATUS_NR_CAPPED : 0);
    std::memcpy(st->L0, g->L0, sizeof(g->L0));
  }
  if (c.status & kStatusDeviceTimeout)
    return fail(g, VPFFT_ERR_CUDA, "a bounded device-side wait timed out in a transform pass");
  if (c.status & kStatusNonFinite) return fail(g, VPFFT_ERR_NONFINITE, "non-finite stress or strain rate");
  if (c.status & kStatusMaxRssTiny)
    return fail(g, VPFFT_ERR_MAX_RSS_TINY, "max resolved shear stress < 1e-10 during the iteration");
  return VPFFT_OK;
}

template <typename S>
vpfft_status do_post(vpfft_grid* g, const double edot[5], double dt) {
  PhaseRange range("vpfft post-increment (texture, voxel length, hardening)");
  vpfft_status s = ensure_crss_array(g);
  if (s != VPFFT_OK) return s;
  PostParams p = post_params(g, dt);
  g->launches += launch_post<S>(p, fields<S>(g), (S*)g->crss, g->stream);
  CKL(g);
  finish_post(g, edot, dt);
  CK(g, cudaStreamSynchronize(g->stream));
  return VPFFT_OK;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename S>
vpfft_status do_step(vpfft_grid* g, const double edot[5], int max_iter, double dt, double eps,
                     double avg[5], vpfft_stats* st) {
  vpfft_stats local{};
  vpfft_stats* s = st ? st : &local;
  std::memset(s, 0, sizeof(*s));
  const double t0 = now_s();
  vpfft_status r = do_init<S>(g, edot);
  if (r != VPFFT_OK) return r;
  r = do_ref_medium<S>(g, nullptr);
  if (r != VPFFT_OK) return r;
  const double t1 = now_s();
  r = do_fixed_point<S>(g, edot, max_iter, eps, nullptr, s);
  if (r != VPFFT_OK) return r;
  const double t2 = now_s();
  if (avg)
    for (int c = 0; c < 5; ++c) avg[c] = g->h_ctrl->last[c];
  r = do_post<S>(g, edot, dt);
  if (r != VPFFT_OK) return r;
  const double t3 = now_s();
  s->seconds_init = t1 - t0;
  s->seconds_loop = t2 - t1;
  s->seconds_post = t3 - t2;
  return VPFFT_OK;
}

#define DISPATCH(g, fn, ...) \
  ((g)->prec == VPFFT_PREC_FP64 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

}  // namespace

// ================================================================== C ABI
extern "C" {

const char* vpfft_version(void) { return "vpfft_b200 0.1 (sm_100a)"; }

const char* vpfft_status_string(vpfft_status s) {
  switch (s) {
    case VPFFT_OK: return "ok";
    case VPFFT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case VPFFT_ERR_UNSUPPORTED_SIZE: return "unsupported grid size";
    case VPFFT_ERR_CUDA: return "CUDA error";
    case VPFFT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case VPFFT_ERR_NO_DEVICE: return "no CUDA device";
    case VPFFT_ERR_MAX_RSS_TINY: return "max resolved shear stress < 1e-10";
    case VPFFT_ERR_NONFINITE: return "non-finite values";
    case VPFFT_ERR_NOT_INITIALIZED: return "not initialized";
    case VPFFT_ERR_IO: return "I/O or parse error";
    case VPFFT_ERR_CANCELLED: return "cancelled";
    case VPFFT_ERR_BUSY: return "grid busy in a batch";
  }
  return "unknown status";
}

int vpfft_device_count(void) {
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return cnt;
}

void vpfft_material_default(vpfft_material* m) {
  if (!m) return;
  for (int k = 0; k < kNS; ++k) {
    m->gamma_dot_base[k] = 15.5;  // MaterialGrid.cpp:322
    m->rate_sensitivity[k] = 10;  // 323
    m->crss[k] = 11.0;            // 390
    m->tau0[k] = 11.0;            // 329
    m->tau1[k] = 11.0;            // 330
    m->theta0[k] = 430.0;         // 331
    m->theta1[k] = 110.0;         // 332
  }
  for (int k = 0; k < kNS * kNS; ++k) m->hardening[k] = 1.0;  // 334-336
}

void vpfft_solver_options_default(vpfft_solver_options* o) {
  if (!o) return;
  o->init_nr_epsilon = 5e-4;  // MaterialGrid.cpp:159
  o->init_nr_max_iter = 1000; // 160
  o->nr_epsilon = 5e-4;       // 909
  o->nr_max_resolved = 1e9;   // 910
  o->nr_max_iter = 100;       // 911
  o->green_operator = 0;      // chosen per grid size
  o->mixed_certify_step = 1e-5;
}

vpfft_status vpfft_grid_create(int nx, int ny, int nz, const vpfft_material* material,
                               const vpfft_solver_options* options, vpfft_precision precision,
                               vpfft_grid** out) {
  if (!out) return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "out is NULL");
  *out = nullptr;
  if (precision != VPFFT_PREC_FP64 && precision != VPFFT_PREC_MIXED)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "unknown precision");
  if (!valid_dim(nx) || !valid_dim(ny) || !valid_dim(nz))
    return fail(nullptr, VPFFT_ERR_UNSUPPORTED_SIZE,
                "grid dimensions must be in [1, 512] and products of 2, 3 and 5");
  if (material) {
    for (int k = 0; k < kNS; ++k)
      if (!(material->crss[k] > 0) || !(material->gamma_dot_base[k] > 0))
        return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "CRSS and reference rates must be > 0");
  }
  if (options && (options->green_operator < 0 || options->green_operator > 2))
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "green_operator must be 0, 1 or 2");
  if (options && !(options->mixed_certify_step >= 0.0 && options->mixed_certify_step <= 1e-2))
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "mixed_certify_step must be in [0, 1e-2]");
  vpfft_status s = need_device(nullptr);
  if (s != VPFFT_OK) return s;
  vpfft_grid* g = new vpfft_grid();
  g->nx = nx;
  g->ny = ny;
  g->nz = nz;
  g->nh = nz / 2 + 1;
  g->n = (long long)nx * ny * nz;
  g->prec = precision;
  if (material)
    g->mat = *material;
  else
    vpfft_material_default(&g->mat);
  if (options)
    g->opt = *options;
  else
    vpfft_solver_options_default(&g->opt);
  make_line_plan(nx, &g->px);
  make_line_plan(ny, &g->py);
  make_line_plan(nz, &g->pz);
  g->keep_d = g->n <= (1LL << 21);
  cudaGetDevice(&g->device);
  auto bail = [&](vpfft_status st) {
    free_grid_buffers(g);
    g_lib_err = g->err;
    delete g;
    return st;
  };
#define CKC(call)                                                                            \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      g->err = std::string(#call) + ": " + cudaGetErrorString(e_);                           \
      return bail(e_ == cudaErrorMemoryAllocation ? VPFFT_ERR_OUT_OF_MEMORY : VPFFT_ERR_CUDA); \
    }                                                                                        \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  const size_t es = elem_size(precision);
  const size_t n = (size_t)g->n;
  CKC(cudaMalloc(&g->R, es * n * 9));
  CKC(cudaMalloc(&g->sigma, es * n * 5));
  CKC(cudaMalloc(&g->lambda, es * n * 5));
  CKC(cudaMalloc(&g->work, es * n * 5));
  if (g->keep_d) CKC(cudaMalloc(&g->dkeep, es * n * 5));
  // the per-voxel CRSS (written by the first hardening update) and the
  // iteration history are allocated here, so that no solve -- in particular
  // no batch request -- allocates device memory
  CKC(cudaMalloc(&g->crss, es * n * kNS));
  CKC(cudaMalloc(&g->hist, sizeof(double) * 12 * 128));
  g->hist_cap = 128;
  CKC(cudaMalloc(&g->acc, sizeof(double) * n));
  const size_t nparts = (size_t)std::max(nr_blocks(g->n), ref_medium_blocks(g->n));
  CKC(cudaMalloc(&g->partials, sizeof(double) * nparts * 25));
  CKC(cudaMalloc(&g->sum25, sizeof(double) * 25));
  CKC(cudaMalloc(&g->ctrl, sizeof(IterCtrl)));
  CKC(cudaMallocHost(&g->h_ctrl, sizeof(IterCtrl)));
  CKC(cudaMemset(g->acc, 0, sizeof(double) * n));
#undef CKC
  s = precision == VPFFT_PREC_FP64 ? upload_twiddles<double>(g) : upload_twiddles<float>(g);
  if (s != VPFFT_OK) return bail(s);
  *out = g;
  return VPFFT_OK;
}

vpfft_status vpfft_grid_destroy(vpfft_grid* g) {
  if (g && g->in_batch) return busy(g);
  if (!g) return VPFFT_OK;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  free_grid_buffers(g);
  delete g;
  return VPFFT_OK;
}

vpfft_status vpfft_grid_dims(const vpfft_grid* g, int* nx, int* ny, int* nz) {
  if (!g) return VPFFT_ERR_INVALID_ARGUMENT;
  if (nx) *nx = g->nx;
  if (ny) *ny = g->ny;
  if (nz) *nz = g->nz;
  return VPFFT_OK;
}

static vpfft_status set_fields_impl(vpfft_grid* g, const double* R, const double* sigma,
                                    bool device) {
  if (g && g->in_batch) return busy(g);
  if (!g) return VPFFT_ERR_INVALID_ARGUMENT;
  if (!R) return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "Orientation array not initialized");
  cudaSetDevice(g->device);
  vpfft_status s;
  if (g->prec == VPFFT_PREC_FP64) {
    s = to_device_field<double>(g, R, device, (double*)g->R, 9);
    if (s == VPFFT_OK && sigma) s = to_device_field<double>(g, sigma, device, (double*)g->sigma, 5);
    if (s == VPFFT_OK && !sigma) g->launches += launch_fill<double>((double*)g->sigma, g->n * 5, 0.0, g->stream);
  } else {
    s = to_device_field<float>(g, R, device, (float*)g->R, 9);
    if (s == VPFFT_OK && sigma) s = to_device_field<float>(g, sigma, device, (float*)g->sigma, 5);
    if (s == VPFFT_OK && !sigma) g->launches += launch_fill<float>((float*)g->sigma, g->n * 5, 0.0, g->stream);
  }
  if (s != VPFFT_OK) return s;
  CK(g, cudaMemsetAsync(g->acc, 0, sizeof(double) * (size_t)g->n, g->stream));
  g->crss_per_voxel = false;
  g->have_L0 = false;
  CK(g, cudaStreamSynchronize(g->stream));
  g->fields_set = true;
  return VPFFT_OK;
}

vpfft_status vpfft_grid_set_fields(vpfft_grid* g, const double* R, const double* sigma) {
  return set_fields_impl(g, R, sigma, false);
}
vpfft_status vpfft_grid_set_fields_device(vpfft_grid* g, const double* R, const double* sigma) {
  return set_fields_impl(g, R, sigma, true);
}

vpfft_status vpfft_grid_set_voxel_length(vpfft_grid* g, double hx, double hy, double hz) {
  if (g && g->in_batch) return busy(g);
  if (!g) return VPFFT_ERR_INVALID_ARGUMENT;
  if (!(hx > 0) || !(hy > 0) || !(hz > 0))
    return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "voxel lengths must be > 0");
  g->h[0] = hx;
  g->h[1] = hy;
  g->h[2] = hz;
  return VPFFT_OK;
}
vpfft_status vpfft_grid_get_voxel_length(const vpfft_grid* g, double h[3]) {
  if (!g || !h) return VPFFT_ERR_INVALID_ARGUMENT;
  std::memcpy(h, g->h, sizeof(g->h));
  return VPFFT_OK;
}

vpfft_status vpfft_grid_set_crss(vpfft_grid* g, const double* crss) {
  if (g && g->in_batch) return busy(g);
  if (!g) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  if (!crss) {
    g->crss_per_voxel = false;
    return VPFFT_OK;
  }
  vpfft_status s = ensure_crss_array(g);
  if (s != VPFFT_OK) return s;
  s = g->prec == VPFFT_PREC_FP64 ? to_device_field<double>(g, crss, false, (double*)g->crss, kNS)
                                 : to_device_field<float>(g, crss, false, (float*)g->crss, kNS);
  if (s == VPFFT_OK) g->crss_per_voxel = true;
  return s;
}

static int field_width(vpfft_field f) {
  switch (f) {
    case VPFFT_FIELD_STRESS:
    case VPFFT_FIELD_LAGRANGE:
    case VPFFT_FIELD_POLARIZATION:
    case VPFFT_FIELD_STRAIN_RATE_VARIATION:
    case VPFFT_FIELD_STRAIN_RATE: return 5;
    case VPFFT_FIELD_ORIENTATION: return 9;
    case VPFFT_FIELD_CRSS: return kNS;
    case VPFFT_FIELD_ACCUMULATED_SHEAR: return 1;
    case VPFFT_FIELD_SCHMID: return 60;
  }
  return -1;
}

}  // extern "C"
template <typename S>
static vpfft_status get_field_impl(vpfft_grid* g, vpfft_field which, double* dst) {
  const long long n = g->n;
  switch (which) {
    case VPFFT_FIELD_STRESS: return from_device_field<S>(g, (S*)g->sigma, 5, dst);
    case VPFFT_FIELD_LAGRANGE: return from_device_field<S>(g, (S*)g->lambda, 5, dst);
    case VPFFT_FIELD_ORIENTATION: return from_device_field<S>(g, (S*)g->R, 9, dst);
    case VPFFT_FIELD_POLARIZATION: return from_device_field<S>(g, (S*)g->work, 5, dst);
    case VPFFT_FIELD_STRAIN_RATE_VARIATION:
      if (!g->keep_d || !g->dkeep)
        return fail(g, VPFFT_ERR_INVALID_ARGUMENT,
                    "d~ is kept only when enabled (grids up to 128^3 by default)");
      return from_device_field<S>(g, (S*)g->dkeep, 5, dst);
    case VPFFT_FIELD_CRSS:
      if (!g->crss_per_voxel) {
        for (long long v = 0; v < n; ++v)
          for (int k = 0; k < kNS; ++k) dst[v * kNS + k] = g->mat.crss[k];
        return VPFFT_OK;
      }
      return from_device_field<S>(g, (S*)g->crss, kNS, dst);
    case VPFFT_FIELD_ACCUMULATED_SHEAR:
      CK(g, cudaMemcpy(dst, g->acc, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
      return VPFFT_OK;
    case VPFFT_FIELD_STRAIN_RATE: {
      S* tmp = nullptr;
      CK(g, cudaMalloc(&tmp, sizeof(S) * (size_t)n * 5));
      VoxelParams p = voxel_params(g, g->last_edot);
      g->launches += launch_strain_rate<S>(p, fields<S>(g), tmp, g->stream);
      vpfft_status s = from_device_field<S>(g, tmp, 5, dst);
      cudaFree(tmp);
      return s;
    }
    case VPFFT_FIELD_SCHMID: {
      double* tmp = nullptr;
      CK(g, cudaMalloc(&tmp, sizeof(double) * (size_t)n * 60));
      g->launches += launch_schmid_field<S>(n, (S*)g->R, tmp, g->stream);
      cudaError_t e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(dst, tmp, sizeof(double) * (size_t)n * 60, cudaMemcpyDeviceToHost, g->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
      cudaFree(tmp);
      if (e != cudaSuccess) return fail(g, VPFFT_ERR_CUDA, cudaGetErrorString(e));
      return VPFFT_OK;
    }
  }
  return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "unknown field");
}

extern "C" {

vpfft_status vpfft_grid_get_field(vpfft_grid* g, vpfft_field which, double* dst) {
  if (g && g->in_batch) return busy(g);
  if (!g || !dst || field_width(which) < 0) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  return g->prec == VPFFT_PREC_FP64 ? get_field_impl<double>(g, which, dst)
                                    : get_field_impl<float>(g, which, dst);
}

}  // extern "C"
template <typename S>
static vpfft_status set_field_impl(vpfft_grid* g, vpfft_field which, const double* src) {
  switch (which) {
    case VPFFT_FIELD_STRESS: return to_device_field<S>(g, src, false, (S*)g->sigma, 5);
    case VPFFT_FIELD_LAGRANGE: return to_device_field<S>(g, src, false, (S*)g->lambda, 5);
    case VPFFT_FIELD_ORIENTATION: return to_device_field<S>(g, src, false, (S*)g->R, 9);
    case VPFFT_FIELD_POLARIZATION: return to_device_field<S>(g, src, false, (S*)g->work, 5);
    case VPFFT_FIELD_CRSS: return vpfft_grid_set_crss(g, src);
    case VPFFT_FIELD_ACCUMULATED_SHEAR:
      CK(g, cudaMemcpy(g->acc, src, sizeof(double) * (size_t)g->n, cudaMemcpyHostToDevice));
      return VPFFT_OK;
    default: return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "field is derived and cannot be set");
  }
}

extern "C" {

vpfft_status vpfft_grid_set_field(vpfft_grid* g, vpfft_field which, const double* src) {
  if (g && g->in_batch) return busy(g);
  if (!g || !src || field_width(which) < 0) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  vpfft_status s = g->prec == VPFFT_PREC_FP64 ? set_field_impl<double>(g, which, src)
                                              : set_field_impl<float>(g, which, src);
  if (s == VPFFT_OK && which == VPFFT_FIELD_ORIENTATION) g->fields_set = true;
  return s;
}

}  // extern "C"

namespace {

// Binary snapshot of a grid: this header, then FP64 voxel-major fields in the
// order stress (5), Lagrange multiplier (5), orientation (9), polarization /
// work field (5), accumulated shear (1) and, when the CRSS is per voxel, the
// CRSS (12).
struct SnapshotHeader {
  char magic[8];
  int32_t version, precision, nx, ny, nz, flags, pad;
  double h[3];
  double L0[25];
  double last_edot[5];
};
constexpr char kSnapMagic[8] = {'V', 'P', 'F', 'F', 'T', 'S', 'N', '1'};
constexpr int32_t kSnapFieldsSet = 1, kSnapCrssPerVoxel = 2, kSnapHaveL0 = 4;

size_t snapshot_bytes(long long n, bool crss_per_voxel) {
  const size_t per = 5 + 5 + 9 + 5 + 1 + (crss_per_voxel ? kNS : 0);
  return sizeof(SnapshotHeader) + sizeof(double) * per * (size_t)n;
}

struct SnapField {
  vpfft_field f;
  int width;
};
constexpr SnapField kSnapFields[] = {{VPFFT_FIELD_STRESS, 5},
                                     {VPFFT_FIELD_LAGRANGE, 5},
                                     {VPFFT_FIELD_ORIENTATION, 9},
                                     {VPFFT_FIELD_POLARIZATION, 5},
                                     {VPFFT_FIELD_ACCUMULATED_SHEAR, 1},
                                     {VPFFT_FIELD_CRSS, kNS}};

}  // namespace

extern "C" {

vpfft_status vpfft_grid_snapshot_size(const vpfft_grid* g, size_t* bytes) {
  if (!g || !bytes) return VPFFT_ERR_INVALID_ARGUMENT;
  *bytes = snapshot_bytes(g->n, g->crss_per_voxel);
  return VPFFT_OK;
}

vpfft_status vpfft_grid_snapshot(vpfft_grid* g, void* buf, size_t cap) {
  if (g && g->in_batch) return busy(g);
  if (!g || !buf) return VPFFT_ERR_INVALID_ARGUMENT;
  const size_t need = snapshot_bytes(g->n, g->crss_per_voxel);
  if (cap < need)
    return fail(g, VPFFT_ERR_INVALID_ARGUMENT,
                "snapshot buffer too small: " + std::to_string(need) + " bytes needed");
  SnapshotHeader hd{};
  std::memcpy(hd.magic, kSnapMagic, sizeof(kSnapMagic));
  hd.version = 1;
  hd.precision = (int32_t)g->prec;
  hd.nx = g->nx;
  hd.ny = g->ny;
  hd.nz = g->nz;
  hd.flags = (g->fields_set ? kSnapFieldsSet : 0) | (g->crss_per_voxel ? kSnapCrssPerVoxel : 0) |
             (g->have_L0 ? kSnapHaveL0 : 0);
  std::memcpy(hd.h, g->h, sizeof(hd.h));
  std::memcpy(hd.L0, g->L0, sizeof(hd.L0));
  std::memcpy(hd.last_edot, g->last_edot, sizeof(hd.last_edot));
  unsigned char* out = static_cast<unsigned char*>(buf);
  std::memcpy(out, &hd, sizeof(hd));
  double* d = reinterpret_cast<double*>(out + sizeof(hd));
  for (const SnapField& sf : kSnapFields) {
    if (sf.f == VPFFT_FIELD_CRSS && !g->crss_per_voxel) continue;
    if (vpfft_status s = vpfft_grid_get_field(g, sf.f, d)) return s;
    d += (size_t)sf.width * (size_t)g->n;
  }
  return VPFFT_OK;
}

vpfft_status vpfft_grid_restore(vpfft_grid* g, const void* buf, size_t size) {
  if (g && g->in_batch) return busy(g);
  if (!g || !buf) return VPFFT_ERR_INVALID_ARGUMENT;
  SnapshotHeader hd{};
  if (size < sizeof(hd)) return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "snapshot truncated");
  std::memcpy(&hd, buf, sizeof(hd));
  if (std::memcmp(hd.magic, kSnapMagic, sizeof(kSnapMagic)) != 0 || hd.version != 1)
    return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "not a vpfft grid snapshot");
  if (hd.precision != (int32_t)g->prec || hd.nx != g->nx || hd.ny != g->ny || hd.nz != g->nz)
    return fail(g, VPFFT_ERR_INVALID_ARGUMENT,
                "snapshot of a grid of other dimensions or precision");
  const bool crss_pv = (hd.flags & kSnapCrssPerVoxel) != 0;
  if (size != snapshot_bytes(g->n, crss_pv))
    return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "snapshot size does not match its header");
  if (!(hd.h[0] > 0) || !(hd.h[1] > 0) || !(hd.h[2] > 0))
    return fail(g, VPFFT_ERR_INVALID_ARGUMENT, "snapshot voxel lengths must be > 0");
  const double* d =
      reinterpret_cast<const double*>(static_cast<const unsigned char*>(buf) + sizeof(hd));
  // From here the grid's fields are overwritten one at a time: if a copy
  // fails part-way the grid holds a mix of old and new state, so it is marked
  // unusable (no fields, no reference medium) until it is restored or its
  // fields are set again.
  for (const SnapField& sf : kSnapFields) {
    vpfft_status s = sf.f == VPFFT_FIELD_CRSS ? vpfft_grid_set_crss(g, crss_pv ? d : nullptr)
                                              : vpfft_grid_set_field(g, sf.f, d);
    if (s != VPFFT_OK) {
      g->fields_set = false;
      g->have_L0 = false;
      return s;
    }
    if (sf.f != VPFFT_FIELD_CRSS || crss_pv) d += (size_t)sf.width * (size_t)g->n;
  }
  std::memcpy(g->h, hd.h, sizeof(g->h));
  std::memcpy(g->L0, hd.L0, sizeof(g->L0));
  std::memcpy(g->last_edot, hd.last_edot, sizeof(g->last_edot));
  g->have_L0 = (hd.flags & kSnapHaveL0) != 0;
  if (g->have_L0) derive_L0_inverses(g);
  g->fields_set = (hd.flags & kSnapFieldsSet) != 0;
  return VPFFT_OK;
}

vpfft_status vpfft_run_single_strain_step(vpfft_grid* g, const double edot[5], int max_iter,
                                          double dt, double eps, double avg[5], vpfft_stats* st) {
  if (g && g->in_batch) return busy(g);
  if (!g || !edot) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  return DISPATCH(g, do_step, g, edot, max_iter, dt, eps, avg, st);
}

vpfft_status vpfft_run(vpfft_grid* g, const double edot[5], int max_iter, int n_steps, double dt,
                       double eps, const char* path, vpfft_step_callback cb, void* user) {
  if (g && g->in_batch) return busy(g);
  if (!g || !edot || n_steps < 0) return VPFFT_ERR_INVALID_ARGUMENT;
  FILE* os = nullptr;
  if (path) {
    os = std::fopen(path, "w");
    if (!os) return fail(g, VPFFT_ERR_IO, std::string("cannot open ") + path);
  }
  double strain[5] = {0, 0, 0, 0, 0};
  vpfft_status s = VPFFT_OK;
  for (int i = 0; i < n_steps; ++i) {
    double avg[5];
    s = vpfft_run_single_strain_step(g, edot, max_iter, dt, eps, avg, nullptr);
    if (s != VPFFT_OK) break;
    for (int c = 0; c < 5; ++c) strain[c] += edot[c] * dt;  // MaterialGrid.cpp:1217
    if (os) {
      // one row per increment like MaterialGrid.cpp:1221-1225
      double ne = 0, ns = 0;
      for (int c = 0; c < 5; ++c) {
        ne += strain[c] * strain[c];
        ns += avg[c] * avg[c];
      }
      std::fprintf(os, "%d ", i);
      for (int c = 0; c < 5; ++c) std::fprintf(os, "%g ", strain[c]);
      std::fprintf(os, " ");
      for (int c = 0; c < 5; ++c) std::fprintf(os, "%g ", avg[c]);
      std::fprintf(os, " %g %g \n", std::sqrt(ne), std::sqrt(ns));
    }
    if (cb && cb(i, strain, avg, user)) break;
  }
  if (os) std::fclose(os);
  return s;
}

vpfft_status vpfft_initialize_computation(vpfft_grid* g, const double edot[5]) {
  if (g && g->in_batch) return busy(g);
  if (!g || !edot) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  return DISPATCH(g, do_init, g, edot);
}
vpfft_status vpfft_build_reference_medium(vpfft_grid* g, double L0_out[25]) {
  if (g && g->in_batch) return busy(g);
  if (!g) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  return DISPATCH(g, do_ref_medium, g, L0_out);
}
vpfft_status vpfft_fixed_point(vpfft_grid* g, const double edot[5], int max_iter, double eps,
                               double* history, vpfft_stats* st) {
  if (g && g->in_batch) return busy(g);
  if (!g || !edot) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  return DISPATCH(g, do_fixed_point, g, edot, max_iter, eps, history, st);
}
vpfft_status vpfft_post_increment(vpfft_grid* g, const double edot[5], double dt) {
  if (g && g->in_batch) return busy(g);
  if (!g || !edot) return VPFFT_ERR_INVALID_ARGUMENT;
  cudaSetDevice(g->device);
  return DISPATCH(g, do_post, g, edot, dt);
}
vpfft_status vpfft_grid_synchronize(vpfft_grid* g) {
  if (!g) return VPFFT_ERR_INVALID_ARGUMENT;
  CK(g, cudaStreamSynchronize(g->stream));
  return VPFFT_OK;
}
void* vpfft_grid_stream(vpfft_grid* g) { return g ? (void*)g->stream : nullptr; }

vpfft_status vpfft_grid_set_profiling(vpfft_grid* g, int enabled) {
  if (!g) return VPFFT_ERR_INVALID_ARGUMENT;
  g->profile = enabled != 0;
  for (int k = 0; k < VPFFT_NUM_PHASES; ++k) {
    g->phase_ms[k] = 0;
    g->phase_n[k] = 0;
  }
  return VPFFT_OK;
}

vpfft_status vpfft_grid_phase_times(const vpfft_grid* g, double* ms, int64_t* counts) {
  if (!g || !ms || !counts) return VPFFT_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < VPFFT_NUM_PHASES; ++k) {
    ms[k] = g->phase_ms[k];
    counts[k] = g->phase_n[k];
  }
  return VPFFT_OK;
}

const char* vpfft_phase_name(int phase) {
  static const char* names[VPFFT_NUM_PHASES] = {"fft_z_r2c", "fft_y_forward", "fft_x_green",
                                                "fft_y_inverse", "fft_z_c2r", "nr_update",
                                                "iter_finish"};
  return (phase >= 0 && phase < VPFFT_NUM_PHASES) ? names[phase] : "";
}
int64_t vpfft_grid_launch_count(const vpfft_grid* g) { return g ? g->launches : 0; }
const char* vpfft_last_error(const vpfft_grid* g) { return g ? g->err.c_str() : g_lib_err.c_str(); }

// ------------------------------------------------------------------ Solvers batch
namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
vpfft_status upload(DevBuf& b, const void* src, size_t bytes) {
  if (cudaMalloc(&b.p, bytes ? bytes : 8) != cudaSuccess)
    return fail(nullptr, VPFFT_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
  if (src && bytes && cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(nullptr, VPFFT_ERR_CUDA, "cudaMemcpy failed");
  return VPFFT_OK;
}
vpfft_status finish_batch(void* dst, const DevBuf& b, size_t bytes) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess && dst) e = cudaMemcpy(dst, b.p, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(nullptr, VPFFT_ERR_CUDA, cudaGetErrorString(e));
  return VPFFT_OK;
}
#define UP(buf, ptr, bytes)                        \
  do {                                             \
    vpfft_status s_ = upload(buf, ptr, bytes);     \
    if (s_ != VPFFT_OK) return s_;                 \
  } while (0)
}  // namespace

vpfft_status vpfft_solve_constrained_constitutive(int n, const double* s0, const double* schmid,
                                                  const double* crss, const vpfft_material* m,
                                                  const double edot[5], const double* lambda,
                                                  const double* dtilde, const double L0[25],
                                                  double eps, double max_rss, int max_iter,
                                                  double* out, double* nr_error) {
  if (n < 0 || !s0 || !schmid || !crss || !m || !edot || !lambda || !dtilde || !L0 || !out)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (vpfft_status s = need_device(nullptr)) return s;
  if (n == 0) return VPFFT_OK;
  DevBuf a, b, c, d, e, o, r;
  UP(a, s0, sizeof(double) * 5 * n);
  UP(b, schmid, sizeof(double) * 60 * n);
  UP(c, crss, sizeof(double) * 12 * n);
  UP(d, lambda, sizeof(double) * 5 * n);
  UP(e, dtilde, sizeof(double) * 5 * n);
  UP(o, nullptr, sizeof(double) * 5 * n);
  UP(r, nullptr, sizeof(double) * n);
  launch_solvers_constrained(n, (double*)a.p, (double*)b.p, (double*)c.p, mat_params(*m), edot,
                             (double*)d.p, (double*)e.p, L0, eps, max_rss, max_iter, (double*)o.p,
                             (double*)r.p, nullptr);
  vpfft_status s = finish_batch(out, o, sizeof(double) * 5 * n);
  if (s == VPFFT_OK && nr_error) s = finish_batch(nr_error, r, sizeof(double) * n);
  return s;
}

vpfft_status vpfft_solve_constitutive(int n, const double* s0, const double* schmid,
                                      const double* crss, const vpfft_material* m,
                                      const double edot[5], double eps, double max_rss,
                                      int max_iter, double* out) {
  if (n < 0 || !s0 || !schmid || !crss || !m || !edot || !out)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (vpfft_status s = need_device(nullptr)) return s;
  if (n == 0) return VPFFT_OK;
  DevBuf a, b, c, o;
  UP(a, s0, sizeof(double) * 5 * n);
  UP(b, schmid, sizeof(double) * 60 * n);
  UP(c, crss, sizeof(double) * 12 * n);
  UP(o, nullptr, sizeof(double) * 5 * n);
  launch_solvers_unconstrained(n, (double*)a.p, (double*)b.p, (double*)c.p, mat_params(*m), edot,
                               eps, max_rss, max_iter, (double*)o.p, nullptr);
  return finish_batch(out, o, sizeof(double) * 5 * n);
}

vpfft_status vpfft_apply_constitutive(int n, const double* s, const double* schmid,
                                      const double* crss, const vpfft_material* m, double* out) {
  if (n < 0 || !s || !schmid || !crss || !m || !out)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (vpfft_status st = need_device(nullptr)) return st;
  if (n == 0) return VPFFT_OK;
  DevBuf a, b, c, o;
  UP(a, s, sizeof(double) * 5 * n);
  UP(b, schmid, sizeof(double) * 60 * n);
  UP(c, crss, sizeof(double) * 12 * n);
  UP(o, nullptr, sizeof(double) * 5 * n);
  launch_solvers_apply(n, (double*)a.p, (double*)b.p, (double*)c.p, mat_params(*m), (double*)o.p, nullptr);
  return finish_batch(out, o, sizeof(double) * 5 * n);
}

vpfft_status vpfft_solve_sachs(int n, const double* schmid, const double* crss,
                               const double edot[5], double* out) {
  if (n < 0 || !schmid || !crss || !edot || !out)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (vpfft_status s = need_device(nullptr)) return s;
  if (n == 0) return VPFFT_OK;
  DevBuf b, c, o;
  UP(b, schmid, sizeof(double) * 60 * n);
  UP(c, crss, sizeof(double) * 12 * n);
  UP(o, nullptr, sizeof(double) * 5 * n);
  launch_solvers_sachs(n, (double*)b.p, (double*)c.p, edot, (double*)o.p, nullptr);
  return finish_batch(out, o, sizeof(double) * 5 * n);
}

vpfft_status vpfft_schmid_tensors(int n, const double* R, double* out) {
  if (n < 0 || !R || !out) return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "NULL argument");
  if (vpfft_status s = need_device(nullptr)) return s;
  if (n == 0) return VPFFT_OK;
  DevBuf a, o;
  UP(a, R, sizeof(double) * 9 * n);
  UP(o, nullptr, sizeof(double) * 60 * n);
  launch_solvers_schmid(n, (double*)a.p, (double*)o.p, nullptr);
  return finish_batch(out, o, sizeof(double) * 60 * n);
}

vpfft_status vpfft_green_apply(int n, const int32_t* kidx, int nx, int ny, int nz,
                               const double h[3], const double L0[25], const double* phat,
                               double* dhat, vpfft_precision prec) {
  if (n < 0 || !kidx || !h || !L0 || !phat || !dhat || nx < 1 || ny < 1 || nz < 1)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  if (vpfft_status s = need_device(nullptr)) return s;
  if (n == 0) return VPFFT_OK;
  double negL[25], Linv[25];
  for (int k = 0; k < 25; ++k) negL[k] = -L0[k];
  inverse5_host(negL, Linv);
  DevBuf k, p, o;
  UP(k, kidx, sizeof(int32_t) * 3 * n);
  UP(p, phat, sizeof(double) * 10 * n);
  UP(o, nullptr, sizeof(double) * 10 * n);
  if (prec == VPFFT_PREC_FP64)
    launch_green_batch<double>(n, (int32_t*)k.p, green_params<double>(nx, ny, nz, h, L0, Linv),
                               (double*)p.p, (double*)o.p, nullptr);
  else
    launch_green_batch<float>(n, (int32_t*)k.p, green_params<float>(nx, ny, nz, h, L0, Linv),
                              (double*)p.p, (double*)o.p, nullptr);
  return finish_batch(dhat, o, sizeof(double) * 10 * n);
}

// ------------------------------------------------------------------ FFT (testing)
}  // extern "C"
template <typename S>
static vpfft_status fft_impl(int nx, int ny, int nz, int ncomp, const double* in, double* out,
                             int mode) {
  vpfft_grid tmp;  // only used for the twiddle upload / error string
  tmp.nx = nx;
  tmp.ny = ny;
  tmp.nz = nz;
  tmp.nh = nz / 2 + 1;
  make_line_plan(nx, &tmp.px);
  make_line_plan(ny, &tmp.py);
  make_line_plan(nz, &tmp.pz);
  const int nh = tmp.nh;
  const long long n = (long long)nx * ny * nz;
  const size_t nspec = (size_t)ncomp * nx * ny * nh;
  vpfft_status s = upload_twiddles<S>(&tmp);
  DevBuf X, X2, real, io;
  if (s == VPFFT_OK) s = upload(X, nullptr, 2 * sizeof(S) * nspec);
  if (s == VPFFT_OK) s = upload(X2, nullptr, 2 * sizeof(S) * nspec);
  if (s == VPFFT_OK) s = upload(real, nullptr, sizeof(S) * n * ncomp);
  const size_t in_count = mode == 0 ? (size_t)n * ncomp : 2 * nspec;
  const size_t out_count = mode == 0 ? 2 * nspec : (size_t)n * ncomp;
  if (s == VPFFT_OK) s = upload(io, nullptr, sizeof(double) * std::max(in_count, out_count));
  // the device keeps the spectrum as B[c][kz][ky][x]; the API uses [c][x][y][kz]
  auto b_index = [&](size_t c, size_t x, size_t y, size_t k) {
    return 2 * (((c * nh + k) * ny + y) * nx + x);
  };
  auto api_index = [&](size_t c, size_t x, size_t y, size_t k) {
    return 2 * (((c * nx + x) * ny + y) * nh + k);
  };
  std::vector<double> host(std::max(in_count, out_count));
  if (s == VPFFT_OK) {
    Spectral<S> sp = spectral<S>(&tmp, X.p, X2.p);
    if (mode == 0) {
      cudaMemcpy(io.p, in, sizeof(double) * in_count, cudaMemcpyHostToDevice);
      launch_to_soa<S>((double*)io.p, (S*)real.p, (long long)in_count, 1, nullptr);
      launch_fft3d<S>(sp, (S*)real.p, ncomp, 0, nullptr);
      launch_from_soa<S>((S*)X2.p, (double*)io.p, (long long)out_count, 1, nullptr);
      s = finish_batch(host.data(), io, sizeof(double) * out_count);
      if (s == VPFFT_OK)
        for (int c = 0; c < ncomp; ++c)
          for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
              for (int k = 0; k < nh; ++k) {
                out[api_index(c, x, y, k)] = host[b_index(c, x, y, k)];
                out[api_index(c, x, y, k) + 1] = host[b_index(c, x, y, k) + 1];
              }
    } else {
      for (int c = 0; c < ncomp; ++c)
        for (int x = 0; x < nx; ++x)
          for (int y = 0; y < ny; ++y)
            for (int k = 0; k < nh; ++k) {
              host[b_index(c, x, y, k)] = in[api_index(c, x, y, k)];
              host[b_index(c, x, y, k) + 1] = in[api_index(c, x, y, k) + 1];
            }
      cudaMemcpy(io.p, host.data(), sizeof(double) * in_count, cudaMemcpyHostToDevice);
      launch_to_soa<S>((double*)io.p, (S*)X2.p, (long long)in_count, 1, nullptr);
      launch_fft3d<S>(sp, (S*)real.p, ncomp, 1, nullptr);
      launch_from_soa<S>((S*)real.p, (double*)io.p, (long long)out_count, 1, nullptr);
      s = finish_batch(out, io, sizeof(double) * out_count);
    }
  }
  if (tmp.twx) cudaFree(tmp.twx);
  if (tmp.twy) cudaFree(tmp.twy);
  if (tmp.twz) cudaFree(tmp.twz);
  tmp.twx = tmp.twy = tmp.twz = nullptr;
  return s;
}

extern "C" {

vpfft_status vpfft_fft3d_r2c(int nx, int ny, int nz, int ncomp, const double* real, double* spec,
                             vpfft_precision prec) {
  if (!valid_dim(nx) || !valid_dim(ny) || !valid_dim(nz) || ncomp < 1 || ncomp > 5 || !real || !spec)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  if (vpfft_status s = need_device(nullptr)) return s;
  return prec == VPFFT_PREC_FP64 ? fft_impl<double>(nx, ny, nz, ncomp, real, spec, 0)
                                 : fft_impl<float>(nx, ny, nz, ncomp, real, spec, 0);
}
int vpfft_set_tma_passes(int enable) { return vpfft::set_tma_passes(enable); }

vpfft_status vpfft_grid_green_operator(const vpfft_grid* g, int* mode, double* ms_compute,
                                       double* ms_table) {
  if (!g || !mode) return VPFFT_ERR_INVALID_ARGUMENT;
  *mode = g->green_mode;
  if (ms_compute) *ms_compute = g->green_ms[0];
  if (ms_table) *ms_table = g->green_ms[1];
  return VPFFT_OK;
}

vpfft_status vpfft_fft3d_c2r(int nx, int ny, int nz, int ncomp, const double* spec, double* real,
                             vpfft_precision prec) {
  if (!valid_dim(nx) || !valid_dim(ny) || !valid_dim(nz) || ncomp < 1 || ncomp > 5 || !real || !spec)
    return fail(nullptr, VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  if (vpfft_status s = need_device(nullptr)) return s;
  return prec == VPFFT_PREC_FP64 ? fft_impl<double>(nx, ny, nz, ncomp, spec, real, 1)
                                 : fft_impl<float>(nx, ny, nz, ncomp, spec, real, 1);
}

}  // extern "C"
