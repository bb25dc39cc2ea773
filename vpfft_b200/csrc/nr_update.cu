// nr_update.cu -- the Newton-Raphson kernels of the initialisation and of the
// fixed-point loop (see nr_kernel.cuh for the per-voxel arithmetic), their
// launchers, and the batched Solvers entry points built on the same code.
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

#include "kernel_common.cuh"
#include "nr_kernel.cuh"

namespace vpfft {

// Shared memory of the NR kernels per thread: 60 Schmid components, plus 12
// reciprocal CRSS values when the CRSS is per voxel.
template <typename MS>
__host__ __device__ constexpr int nr_smem_per_thread(bool tau) {
  return (60 + (tau ? 12 : 0)) * (int)sizeof(MS);
}
// Blocks per SM the NR kernels are compiled for: the FP64 Schmid tile
// (61 KB per 128-thread block) fits three blocks in an SM's shared memory.
template <typename MS>
constexpr int nr_min_blocks() {
  return sizeof(MS) == 8 ? 3 : 4;
}
// The batched initialisation kernel reads all of the slot's constants from
// shared memory instead of the constant bank, which costs registers: three
// blocks per SM.
template <typename MS>
constexpr int nr_batch_min_blocks() {
  return 3;
}
// The fixed-point NR sweep: three blocks per SM for the single grid (168
// registers, no spills; measured 3 % faster at 256^3 mixed than four blocks
// of 128 registers, which spill), four for the batched FP32 sweep (measured
// 3 % faster than three there).
template <typename MS>
constexpr int nr_loop_min_blocks() {
  return 3;
}
template <typename MS>
constexpr int nr_loop_batch_min_blocks() {
  return sizeof(MS) == 8 ? 3 : 4;
}

template <bool kTauSmem, typename S, typename MS>
__device__ __forceinline__ void voxel_schmid(const FieldPtrs<S>& f, long long n, long long v,
                                             MS* msm, MS* tsm, int bs) {
  MS R[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) R[k] = (MS)f.R[k * n + v];
  if constexpr (sizeof(MS) == 4)
    schmid_to_smem_pairs(R, msm, bs);
  else
    schmid_to_smem<MS>(R, msm, bs);
  if constexpr (kTauSmem) {
    // 1/CRSS: IEEE FP64 division for the FP64 path, the correctly rounded
    // FP32 reciprocal of the FP32 CRSS for the mixed path's FP32 staging
#pragma unroll
    for (int q = 0; q < kNS; ++q) {
      if constexpr (sizeof(MS) == 4)
        tsm[SL<MS>::t(q, bs)] = __frcp_rn((float)f.crss[q * n + v]);
      else
        tsm[SL<MS>::t(q, bs)] = (MS)(1.0 / (double)f.crss[q * n + v]);
    }
  }
}

// InitializeComputation (MaterialGrid.cpp:153-210): Sachs guess, scaled to the
// yield surface when MaxRSS > 1.1, unconstrained NR; lambda = P = sigma.
// Persistent grid-stride loop over voxels: block blk of nblk.
template <typename S, typename MS, int NEXP, bool kTauSmem>
__device__ __forceinline__ void init_body(const NRParams& p, const FieldPtrs<S>& f,
                                          IterCtrl* ctrl, int blk, int nblk, MS* msm, MS* tsm) {
  constexpr int bs = kVoxelBlock;  // every launch of these kernels uses kVoxelBlock threads
  const long long n = p.n;
  unsigned long long capped_count = 0;
  int status = 0;
  for (long long v = (long long)blk * bs + threadIdx.x; v < n; v += (long long)nblk * bs) {
    voxel_schmid<kTauSmem>(f, n, v, msm, tsm, bs);
    const double mxs = max_resolved<kTauSmem>(msm, tsm, bs, p, p.edot);
    double g[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) g[c] = p.edot[c] / mxs;
    const double mx = max_resolved<kTauSmem>(msm, tsm, bs, p, g);
    if (mx > 1.1) {
#pragma unroll
      for (int c = 0; c < 5; ++c) g[c] /= mx;
    }
    if (mx < 1e-10) status |= kStatusMaxRssTiny;
    // a zero strain rate makes the Sachs guess 0/0 (Solvers.cpp:241)
    if (!isfinite(mx)) status |= kStatusNonFinite;
    bool capped;
    if constexpr (sizeof(S) == 4) {
      // mixed precision: FP32 Newton predictor from the Sachs guess, then the
      // reference's FP64 iteration from its iterate (from the guess if it failed)
      nr_predict_unconstrained_fp32<NEXP, kTauSmem>(msm, tsm, bs, p, p.edot, g, 60);
    }
    nr_unconstrained_smem<NEXP, kTauSmem>(msm, tsm, bs, p, p.edot, g, &capped);
    capped_count += capped ? 1 : 0;
    store5(f.sigma, n, v, g);
    store5(f.lambda, n, v, g);
    store5(f.work, n, v, g);
  }
  if (status) atomicOr(&ctrl->status, status);
  if (capped_count) atomicAdd(&ctrl->nr_capped, capped_count);
}

template <typename S, typename MS, int NEXP, bool kTauSmem>
__global__ void __launch_bounds__(kVoxelBlock, nr_min_blocks<MS>())
    k_init(const __grid_constant__ NRParams p, const __grid_constant__ FieldPtrs<S> f,
           IterCtrl* ctrl) {
  extern __shared__ __align__(16) unsigned char nr_smem[];
  MS* msm = reinterpret_cast<MS*>(nr_smem) + SL<MS>::kThreadStride * threadIdx.x;
  MS* tsm = msm + 60 * kVoxelBlock;
  init_body<S, MS, NEXP, kTauSmem>(p, f, ctrl, blockIdx.x, gridDim.x, msm, tsm);
}

// The same over a batch of RVEs: each block finds its slot and works on the
// slot's voxels with the slot's block count.
template <typename S, typename MS, int NEXP, bool kTauSmem>
__global__ void __launch_bounds__(kVoxelBlock, nr_batch_min_blocks<MS>())
    k_init_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  extern __shared__ __align__(16) unsigned char nr_smem[];
  __shared__ NRParams sp;
  __shared__ FieldPtrs<S> sf;
  int lb;
  const SlotDesc<S>& d = desc[batch_slot(bl, blockIdx.x, &lb)];
  copy_struct(&sp, &d.nr_init);
  copy_struct(&sf, &d.f);
  __syncthreads();
  MS* msm = reinterpret_cast<MS*>(nr_smem) + SL<MS>::kThreadStride * threadIdx.x;
  MS* tsm = msm + 60 * kVoxelBlock;
  init_body<S, MS, NEXP, kTauSmem>(sp, sf, d.ctrl, lb, d.init_blocks, msm, tsm);
}

// The end of a voxel's update in the fixed-point loop (MaterialGrid.cpp:982-1003):
//   P = sigma - L0 d~;  lambda += L0 (Edot + d~ - edot);
// stores sigma, lambda and P (into `work`) and adds the voxel's terms to the
// block sums acc: sigma (5), edot (5), |sigma - lambda|, |edot - Edot - d~|
// (lambda already updated).  ed = Edot + d~.  The sums live at acc[k * kStride]
// (registers for kStride 1, the thread's column of a shared-memory array else).
template <int kStride = 1, typename S, class C>
__device__ __forceinline__ void finish_voxel(const C& cs, long long n, const FieldPtrs<S>& f,
                                             long long v, const double s[5], const double e[5],
                                             double lam[5], const double d[5],
                                             const double ed[5], double* acc) {
  double P[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double ld = 0.0, lt = 0.0;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const double l0 = cs.L0(j * 5 + i);
      ld += l0 * d[j];
      lt += l0 * (ed[j] - e[j]);
    }
    P[i] = s[i] - ld;
    lam[i] += lt;
  }
  store5(f.sigma, n, v, s);
  store5(f.lambda, n, v, lam);
  store5(f.work, n, v, P);
  double es = 0.0, ee = 0.0;
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    acc[c * kStride] += s[c];
    acc[(5 + c) * kStride] += e[c];
    const double ds = s[c] - lam[c];
    const double de = e[c] - cs.edot(c) - d[c];
    es += ds * ds;
    ee += de * de;
  }
  acc[10 * kStride] += sqrt(es);
  acc[11 * kStride] += sqrt(ee);
}

// The per-voxel body of the fixed-point loop, FP64 (MaterialGrid.cpp:946-1003):
//   sigma /= MaxRSS(sigma); sigma = SolveConstrained(...); edot = Apply(sigma);
//   P = sigma - L0 d~; lambda += L0 (Edot + d~ - edot);
// and the block partials of sum sigma, sum edot, sum |sigma - lambda|,
// sum |edot - Edot - d~| (lambda already updated).  `work` holds d~ on entry
// and P on exit.  Persistent grid-stride loop: every thread solves many voxels
// and the block reduces once, so the spread of Newton iteration counts between
// voxels averages out instead of idling warps at a barrier.
// p: the material and solver constants; cs: the RVE's strain rate and
// reference medium; n: its voxel count.
template <typename S, typename MS, int NEXP, bool kTauSmem, bool kFull, class C>
__device__ __forceinline__ void nr_update_body(const NRParams& p, const C& cs, long long n,
                                               const FieldPtrs<S>& f, double* partials,
                                               IterCtrl* ctrl, int blk, int nblk, MS* msm,
                                               MS* tsm) {
  static_assert(sizeof(S) == 8, "the mixed path is nr_update_body_mixed");
  constexpr int bs = kVoxelBlock;  // every launch of these kernels uses kVoxelBlock threads
  double acc[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k] = 0.0;
  unsigned long long capped_count = 0;
  int status = 0;
  for (long long v = (long long)blk * bs + threadIdx.x; v < n; v += (long long)nblk * bs) {
    voxel_schmid<kTauSmem>(f, n, v, msm, tsm, bs);
    double s[5], lam[5], d[5];
    load5(f.sigma, n, v, s);
    load5(f.lambda, n, v, lam);
    load5(f.work, n, v, d);
    if (f.dkeep) store5(f.dkeep, n, v, d);
    double ed[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) ed[c] = cs.edot(c) + d[c];
    double e[5];
    bool capped;
    const double mx = max_resolved<kTauSmem>(msm, tsm, bs, p, s);
    if (mx < 1e-10) status |= kStatusMaxRssTiny;
#pragma unroll
    for (int c = 0; c < 5; ++c) s[c] /= mx;
    nr_constrained_smem<NEXP, kTauSmem>(msm, tsm, bs, p, cs, lam, ed, s, nullptr, &capped);
    apply_smem<NEXP, kTauSmem>(msm, tsm, bs, p, s, e);
    capped_count += capped ? 1 : 0;
    finish_voxel(cs, n, f, v, s, e, lam, d, ed, acc);
  }
  if (status) atomicOr(&ctrl->status, status);
  if (capped_count) atomicAdd(&ctrl->nr_capped, capped_count);
  block_reduce_store<12, kVoxelBlock>(acc, partials + (long long)blk * 12);
}

// Shared memory of the mixed sweep beyond the Schmid staging: the threads' 12
// running sums (double [12][kVoxelBlock]) and, per warp, the queue of its
// voxels that take the FP64 Newton step: kDeferCap voxel indices, with
// kDeferRestart set when the FP32 predictor failed (the FP64 solve then starts
// at sigma / MaxRSS from the previous stress; otherwise from the predicted
// stress, which the voxel's lane has stored into sigma).
constexpr int kDeferCap = 64;  // at most 31 waiting + 32 added in one round
constexpr uint32_t kDeferRestart = 0x80000000u;
template <typename MS>
__host__ __device__ constexpr int nr_defer_smem_per_block() {
  return sizeof(MS) == 4 ? kVoxelBlock * 12 * 8 + (kVoxelBlock / 32) * kDeferCap * 4 : 0;
}

// The FP64 Newton solve of one queued voxel (q: its warp's queue, k: the entry)
// and the end of its update.  Returns whether its NR stopped at the cap.
template <int NEXP, bool kTauSmem, class C>
__device__ __forceinline__ bool fp64_step_queued(const NRParams& p, const C& cs, long long n,
                                                 const FieldPtrs<float>& f, const uint32_t* q,
                                                 int k, float* msm, float* tsm, double* acc) {
  constexpr int bs = kVoxelBlock;
  const uint32_t code = q[k];
  const long long v = (long long)(code & ~kDeferRestart);
  double s[5], lam[5], d[5], ed[5];
  load5(f.sigma, n, v, s);
  load5(f.lambda, n, v, lam);
  load5(f.work, n, v, d);
#pragma unroll
  for (int c = 0; c < 5; ++c) ed[c] = cs.edot(c) + d[c];
  voxel_schmid<kTauSmem>(f, n, v, msm, tsm, bs);
  if (code & kDeferRestart) {
    const double mx = max_resolved<kTauSmem>(msm, tsm, bs, p, s);
#pragma unroll
    for (int c = 0; c < 5; ++c) s[c] /= mx;
  }
  double el[5], e[5];
  bool capped, tight;
  nr_constrained_smem<NEXP, kTauSmem, float, C, true>(msm, tsm, bs, p, cs, lam, ed, s, nullptr,
                                                      &capped, el, &tight);
  if (!capped && tight) {
#pragma unroll
    for (int c = 0; c < 5; ++c) e[c] = el[c];
  } else {
    apply_smem<NEXP, kTauSmem>(msm, tsm, bs, p, s, e);
  }
  finish_voxel<kVoxelBlock>(cs, n, f, v, s, e, lam, d, ed, acc);
  return capped;
}

// The per-voxel body of the fixed-point loop in mixed precision.  Each voxel
// runs an FP32 Newton predictor from its previous stress (the reference's
// iteration and stopping rule in single precision), then the FP64 residual at
// the predicted point: the strain rate S(sigma) in FP64 and
// y = L0^-1 (sigma - lambda) + S - Edot - d~.  Where the Newton step that
// residual asks for, estimated with the predictor's last FP32 factors, is
// below the certification bound (|step|^2 <= cert2 |sigma|^2), the predicted
// stress is accepted with its FP64 strain rate and no step is taken.  Every
// other voxel (and every voxel whose predictor failed) takes the FP64 Newton
// step (FP64 residual and Jacobian, the small system solved in FP32): it is
// queued in its warp's shared-memory queue, and whenever 32 are waiting the
// warp solves them together, one per lane, so that the FP64 work runs in full
// warps instead of the few lanes that need it in each group of 32 voxels.
// The voxel -> warp assignment and the order of every sum are fixed, so the
// results are deterministic run to run.
// kPrefetch: each thread copies its next voxel's fields (R, sigma, lambda, d~)
// into its column of pf with asynchronous copies while it solves the current
// one, so their global-memory latency is not exposed at the start of a voxel.
template <int NEXP, bool kTauSmem, bool kFull, bool kPrefetch, class C>
__device__ __forceinline__ void nr_update_body_mixed(const NRParams& p, const C& cs, long long n,
                                                     const FieldPtrs<float>& f, double* partials,
                                                     IterCtrl* ctrl, int blk, int nblk,
                                                     float* msm, float* tsm, uint32_t* q,
                                                     double* acc, float* pf) {
  constexpr int bs = kVoxelBlock;  // every launch of these kernels uses kVoxelBlock threads
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k * bs] = 0.0;
  unsigned long long capped_count = 0, fp64_count = 0;
  int status = 0;
  int waiting = 0;  // queued voxels of this warp (warp-uniform)
  const long long stride = (long long)nblk * bs;
  auto prefetch = [&](long long w) {
    if (w < n) {
#pragma unroll
      for (int k = 0; k < 9; ++k) __pipeline_memcpy_async(&pf[k * bs], &f.R[k * n + w], 4);
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        __pipeline_memcpy_async(&pf[(9 + c) * bs], &f.sigma[c * n + w], 4);
        __pipeline_memcpy_async(&pf[(14 + c) * bs], &f.lambda[c * n + w], 4);
        __pipeline_memcpy_async(&pf[(19 + c) * bs], &f.work[c * n + w], 4);
      }
    }
    __pipeline_commit();
  };
  if constexpr (kPrefetch) prefetch((long long)blk * bs + threadIdx.x);
  for (long long base = (long long)blk * bs + (threadIdx.x & ~31); base < n; base += stride) {
    const long long v = base + lane;
    bool defer = false;
    uint32_t code = 0;
    // the voxel's FP32 fields; sp: the predictor's stress (from the previous one)
    float sp[5], lam[5], d[5];
    if constexpr (kPrefetch) __pipeline_wait_prior(0);
    if (v < n) {
      if constexpr (kPrefetch) {
        float R[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) R[k] = pf[k * bs];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          sp[c] = pf[(9 + c) * bs];
          lam[c] = pf[(14 + c) * bs];
          d[c] = pf[(19 + c) * bs];
        }
        prefetch(v + stride);
        schmid_to_smem_pairs(R, msm, bs);
        if constexpr (kTauSmem) {
#pragma unroll
          for (int q2 = 0; q2 < kNS; ++q2)
            tsm[SL<float>::t(q2, bs)] = __frcp_rn(f.crss[q2 * n + v]);
        }
      } else {
        voxel_schmid<kTauSmem>(f, n, v, msm, tsm, bs);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          sp[c] = f.sigma[c * n + v];
          lam[c] = f.lambda[c * n + v];
          d[c] = f.work[c * n + v];
        }
      }
      if (f.dkeep) {
#pragma unroll
        for (int c = 0; c < 5; ++c) f.dkeep[c * n + v] = d[c];
      }
      float e32[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) e32[c] = (float)(cs.edot(c) + (double)d[c]);
      float mx0;
      Ldl5<float> fac;
      const bool ok = nr_predict_fp32<NEXP, kTauSmem, kFull>(msm, tsm, bs, p, cs, lam, e32, sp, 8,
                                                             &mx0, &fac);
      if (mx0 < 1e-10f) status |= kStatusMaxRssTiny;
      bool certified = false;
      double s64[5], e[5];
      if (ok) {
#pragma unroll
        for (int c = 0; c < 5; ++c) s64[c] = (double)sp[c];
        const bool adm = strain_rate_fp64<NEXP, kTauSmem, kFull>(msm, tsm, bs, p, s64, e);
        float y[5], st[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
          double a = e[i] - (cs.edot(i) + (double)d[i]);
#pragma unroll
          for (int j = 0; j < 5; ++j) a += cs.L0inv(sym5(i, j)) * (s64[j] - (double)lam[j]);
          y[i] = (float)(-a);
        }
        ldlt5_subst(fac, y, st);
        float dn = 0.f, sn = 0.f;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          dn += st[c] * st[c];
          sn += sp[c] * sp[c];
        }
        certified = adm && dn <= p.cert2_f * sn;
      }
      if (certified) {
        double lamd[5], dd[5], ed[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          lamd[c] = (double)lam[c];
          dd[c] = (double)d[c];
          ed[c] = cs.edot(c) + dd[c];
        }
        finish_voxel<bs>(cs, n, f, v, s64, e, lamd, dd, ed, acc);
      } else {
        defer = true;
        code = (uint32_t)v | (ok ? 0u : kDeferRestart);
        if (ok) {  // the FP64 step starts at the predicted stress
#pragma unroll
          for (int c = 0; c < 5; ++c) f.sigma[c * n + v] = sp[c];
        }
      }
    }
    const unsigned dm = __ballot_sync(0xffffffffu, defer);
    if (defer) q[waiting + __popc(dm & ((1u << lane) - 1u))] = code;
    waiting += __popc(dm);
    if (waiting >= 32) {
      __syncwarp();
      waiting -= 32;
      capped_count += fp64_step_queued<NEXP, kTauSmem>(p, cs, n, f, q, waiting + lane, msm, tsm,
                                                       acc) ? 1 : 0;
      fp64_count++;
      __syncwarp();
    }
  }
  __syncwarp();
  if (lane < waiting) {
    capped_count +=
        fp64_step_queued<NEXP, kTauSmem>(p, cs, n, f, q, lane, msm, tsm, acc) ? 1 : 0;
    fp64_count++;
  }
  if (status) atomicOr(&ctrl->status, status);
  if (capped_count) atomicAdd(&ctrl->nr_capped, capped_count);
  if (fp64_count) atomicAdd(&ctrl->nr_fp64, fp64_count);
  double sums[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) sums[k] = acc[k * bs];
  block_reduce_store<12, kVoxelBlock>(sums, partials + (long long)blk * 12);
}

// Dynamic shared memory of the loop's NR kernels: the Schmid staging, plus the
// FP64-step queues and running sums of the mixed sweep, plus (single-grid
// mixed sweep) the prefetch staging of the next voxel's fields.
constexpr int kPrefetchWords = 24;  // R (9), sigma, lambda, d~ (5 each)
template <typename MS>
__host__ __device__ constexpr size_t nr_loop_smem(bool tau, bool prefetch = false) {
  return (size_t)kVoxelBlock * nr_smem_per_thread<MS>(tau) + nr_defer_smem_per_block<MS>() +
         (prefetch && sizeof(MS) == 4 ? (size_t)kVoxelBlock * kPrefetchWords * 4 : 0);
}

// The loop's per-voxel body for either precision.
template <typename S, typename MS, int NEXP, bool kTauSmem, bool kFull, class C>
__device__ __forceinline__ void nr_loop_body(const NRParams& p, const C& cs, long long n,
                                             const FieldPtrs<S>& f, double* partials,
                                             IterCtrl* ctrl, int blk, int nblk,
                                             unsigned char* smem) {
  MS* msm = reinterpret_cast<MS*>(smem) + SL<MS>::kThreadStride * threadIdx.x;
  MS* tsm = msm + 60 * kVoxelBlock;
  if constexpr (sizeof(S) == 4) {
    unsigned char* extra = smem + (size_t)kVoxelBlock * nr_smem_per_thread<MS>(kTauSmem);
    double* acc = reinterpret_cast<double*>(extra) + threadIdx.x;
    uint32_t* q = reinterpret_cast<uint32_t*>(extra + kVoxelBlock * 12 * sizeof(double)) +
                  (threadIdx.x >> 5) * kDeferCap;
    // the single-grid sweep (kFull) prefetches; the batched one, whose threads
    // have one or two voxels each in small RVEs, does not
    float* pf = kFull ? reinterpret_cast<float*>(extra + (size_t)nr_defer_smem_per_block<MS>()) +
                            threadIdx.x
                      : nullptr;
    nr_update_body_mixed<NEXP, kTauSmem, kFull, kFull>(p, cs, n, f, partials, ctrl, blk, nblk,
                                                       msm, tsm, q, acc, pf);
  } else {
    nr_update_body<S, MS, NEXP, kTauSmem, kFull>(p, cs, n, f, partials, ctrl, blk, nblk, msm,
                                                 tsm);
  }
}

template <typename S, typename MS, int NEXP, bool kTauSmem>
__global__ void __launch_bounds__(kVoxelBlock, nr_loop_min_blocks<MS>())
    k_nr_update(const __grid_constant__ NRParams p, const __grid_constant__ FieldPtrs<S> f,
                double* partials, IterCtrl* ctrl) {
  if (ctrl->done) return;
  extern __shared__ __align__(16) unsigned char nr_smem[];
  nr_loop_body<S, MS, NEXP, kTauSmem, true>(p, ParamConsts{p}, p.n, f, partials, ctrl, blockIdx.x,
                                            gridDim.x, nr_smem);
}

template <typename S, typename MS, int NEXP, bool kTauSmem>
__global__ void __launch_bounds__(kVoxelBlock, nr_loop_batch_min_blocks<MS>())
    k_nr_update_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl,
                      const __grid_constant__ NRParams pm) {
  int lb;
  const SlotDesc<S>& d = desc[batch_slot(bl, blockIdx.x, &lb)];
  if (d.ctrl->done) return;
  extern __shared__ __align__(16) unsigned char nr_smem[];
  __shared__ NRParams sp;
  __shared__ FieldPtrs<S> sf;
  copy_struct(&sp, &d.nr);
  copy_struct(&sf, &d.f);
  __syncthreads();
  // material and solver constants (the same for every RVE of a batch) from the
  // kernel parameter; the slot's strain rate and reference medium from shared memory
  nr_loop_body<S, MS, NEXP, kTauSmem, false>(pm, SharedConsts{&sp}, sp.n, sf, d.partials, d.ctrl,
                                             lb, d.nr_blocks, nr_smem);
}


int uniform_exponent(const NRParams& p) {
  for (int q = 1; q < kNS; ++q)
    if (p.nexp[q] != p.nexp[0]) return 0;
  return (p.nexp[0] == 10 || p.nexp[0] == 20) ? p.nexp[0] : 0;
}

namespace {

// Blocks of a persistent grid-stride launch: as many as are resident at once.
int persistent_blocks(const void* kern, size_t smem, long long n) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, size_t, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  int per_sm = 0, sms = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_tuple(kern, smem, dev);
    auto it = cache.find(key);
    if (it == cache.end()) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kVoxelBlock, smem);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      per_sm = per_sm < 1 ? 1 : per_sm;
      it = cache.emplace(key, per_sm * sms).first;
    }
    per_sm = it->second;
  }
  const long long need = (n + kVoxelBlock - 1) / kVoxelBlock;
  return (int)(need < per_sm ? (need < 1 ? 1 : need) : per_sm);
}


template <typename S, int NEXP, bool TAU>
int init_t(const NRParams& p, const FieldPtrs<S>& f, IterCtrl* ctrl, cudaStream_t st) {
  auto kern = k_init<S, S, NEXP, TAU>;
  const size_t smem = (size_t)kVoxelBlock * nr_smem_per_thread<S>(TAU);
  const int nb = persistent_blocks((const void*)kern, smem, p.n);
  kern<<<nb, kVoxelBlock, smem, st>>>(p, f, ctrl);
  return 1;
}

template <typename S, int NEXP, bool TAU>
int nr_t(const NRParams& p, const FieldPtrs<S>& f, double* partials, IterCtrl* ctrl, double* hist,
         cudaStream_t st, cudaEvent_t* ev) {
  auto kern = k_nr_update<S, S, NEXP, TAU>;
  const size_t smem = nr_loop_smem<S>(TAU, true);
  const int nb = persistent_blocks((const void*)kern, smem, p.n);
  kern<<<nb, kVoxelBlock, smem, st>>>(p, f, partials, ctrl);
  if (ev) cudaEventRecord(ev[0], st);
  k_iter_finish<<<1, kFinishThreads, 0, st>>>(partials, nb, ctrl, hist);
  if (ev) cudaEventRecord(ev[1], st);
  return 2;
}

template <typename S, int NEXP, bool TAU>
int blocks_t(const NRParams& p, bool init) {
  const size_t smem = init ? (size_t)kVoxelBlock * nr_smem_per_thread<S>(TAU)
                           : nr_loop_smem<S>(TAU, true);
  const void* kern = init ? (const void*)k_init<S, S, NEXP, TAU>
                          : (const void*)k_nr_update<S, S, NEXP, TAU>;
  return persistent_blocks(kern, smem, p.n);
}

// Batched launches: same kernels' bodies, one block list over all slots.
template <typename K>
void smem_optin(K kern, size_t smem) {
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <typename S, int NEXP, bool TAU>
int init_batch_t(const SlotDesc<S>* d, const BatchLaunch& bl, cudaStream_t st) {
  auto kern = k_init_batch<S, S, NEXP, TAU>;
  const size_t smem = (size_t)kVoxelBlock * nr_smem_per_thread<S>(TAU);
  smem_optin(kern, smem);
  kern<<<bl.blocks, kVoxelBlock, smem, st>>>(d, bl);
  return 1;
}

template <typename S, int NEXP, bool TAU>
int nr_batch_t(const SlotDesc<S>* d, const BatchLaunch& bl, const BatchLaunch& bls,
               const NRParams& material, cudaStream_t st) {
  auto kern = k_nr_update_batch<S, S, NEXP, TAU>;
  const size_t smem = nr_loop_smem<S>(TAU);
  smem_optin(kern, smem);
  kern<<<bl.blocks, kVoxelBlock, smem, st>>>(d, bl, material);
  k_iter_finish_batch<S><<<bls.m, kFinishThreads, 0, st>>>(d, bls);
  return 2;
}

}  // namespace

template <typename S>
int nr_launch_blocks(const NRParams& p, bool tau, bool init) {
  switch (uniform_exponent(p)) {
    case 10: return tau ? blocks_t<S, 10, true>(p, init) : blocks_t<S, 10, false>(p, init);
    case 20: return tau ? blocks_t<S, 20, true>(p, init) : blocks_t<S, 20, false>(p, init);
    default: return tau ? blocks_t<S, 0, true>(p, init) : blocks_t<S, 0, false>(p, init);
  }
}

template <typename S>
int launch_init_batch(const SlotDesc<S>* d, const BatchLaunch& bl, int nexp, bool tau,
                      cudaStream_t st) {
  if (bl.blocks <= 0) return 0;
  switch (nexp) {
    case 10: return tau ? init_batch_t<S, 10, true>(d, bl, st) : init_batch_t<S, 10, false>(d, bl, st);
    case 20: return tau ? init_batch_t<S, 20, true>(d, bl, st) : init_batch_t<S, 20, false>(d, bl, st);
    default: return tau ? init_batch_t<S, 0, true>(d, bl, st) : init_batch_t<S, 0, false>(d, bl, st);
  }
}

template <typename S>
int launch_nr_update_batch(const SlotDesc<S>* d, const BatchLaunch& bl, const BatchLaunch& bls,
                           const NRParams& material, int nexp, bool tau, cudaStream_t st) {
  if (bl.blocks <= 0) return 0;
  const NRParams& m = material;
  switch (nexp) {
    case 10:
      return tau ? nr_batch_t<S, 10, true>(d, bl, bls, m, st)
                 : nr_batch_t<S, 10, false>(d, bl, bls, m, st);
    case 20:
      return tau ? nr_batch_t<S, 20, true>(d, bl, bls, m, st)
                 : nr_batch_t<S, 20, false>(d, bl, bls, m, st);
    default:
      return tau ? nr_batch_t<S, 0, true>(d, bl, bls, m, st)
                 : nr_batch_t<S, 0, false>(d, bl, bls, m, st);
  }
}

template int nr_launch_blocks<double>(const NRParams&, bool, bool);
template int nr_launch_blocks<float>(const NRParams&, bool, bool);
template int launch_init_batch<double>(const SlotDesc<double>*, const BatchLaunch&, int, bool,
                                       cudaStream_t);
template int launch_init_batch<float>(const SlotDesc<float>*, const BatchLaunch&, int, bool,
                                      cudaStream_t);
template int launch_nr_update_batch<double>(const SlotDesc<double>*, const BatchLaunch&,
                                            const BatchLaunch&, const NRParams&, int, bool,
                                            cudaStream_t);
template int launch_nr_update_batch<float>(const SlotDesc<float>*, const BatchLaunch&,
                                           const BatchLaunch&, const NRParams&, int, bool,
                                           cudaStream_t);

template <typename S>
int launch_init(const NRParams& p, const FieldPtrs<S>& f, IterCtrl* ctrl, cudaStream_t st) {
  const bool tau = f.crss != nullptr;
  switch (uniform_exponent(p)) {
    case 10: return tau ? init_t<S, 10, true>(p, f, ctrl, st) : init_t<S, 10, false>(p, f, ctrl, st);
    case 20: return tau ? init_t<S, 20, true>(p, f, ctrl, st) : init_t<S, 20, false>(p, f, ctrl, st);
    default: return tau ? init_t<S, 0, true>(p, f, ctrl, st) : init_t<S, 0, false>(p, f, ctrl, st);
  }
}

template <typename S>
int launch_nr_update(const NRParams& p, const FieldPtrs<S>& f, double* partials, IterCtrl* ctrl,
                     double* hist, cudaStream_t st, cudaEvent_t* ev) {
  const bool tau = f.crss != nullptr;
  switch (uniform_exponent(p)) {
    case 10:
      return tau ? nr_t<S, 10, true>(p, f, partials, ctrl, hist, st, ev)
                 : nr_t<S, 10, false>(p, f, partials, ctrl, hist, st, ev);
    case 20:
      return tau ? nr_t<S, 20, true>(p, f, partials, ctrl, hist, st, ev)
                 : nr_t<S, 20, false>(p, f, partials, ctrl, hist, st, ev);
    default:
      return tau ? nr_t<S, 0, true>(p, f, partials, ctrl, hist, st, ev)
                 : nr_t<S, 0, false>(p, f, partials, ctrl, hist, st, ev);
  }
}

template int launch_init<double>(const NRParams&, const FieldPtrs<double>&, IterCtrl*, cudaStream_t);
template int launch_init<float>(const NRParams&, const FieldPtrs<float>&, IterCtrl*, cudaStream_t);
template int launch_nr_update<double>(const NRParams&, const FieldPtrs<double>&, double*,
                                      IterCtrl*, double*, cudaStream_t, cudaEvent_t*);
template int launch_nr_update<float>(const NRParams&, const FieldPtrs<float>&, double*, IterCtrl*,
                                     double*, cudaStream_t, cudaEvent_t*);

// ---------------------------------------------------------------- Solvers batch
// One thread per voxel; the caller's Schmid tensors (n x 12 x 5) and CRSS
// (n x 12) are staged into the same shared-memory layout the grid kernels use.
template <bool kConstrained>
__global__ void __launch_bounds__(kVoxelBlock, 3)
    k_solvers_nr(const __grid_constant__ NRParams p, int n, const double* s0, const double* schmid,
                 const double* crss, const double* lambda, const double* dtilde, double* out,
                 double* nr_err) {
  extern __shared__ __align__(16) unsigned char nr_smem[];
  constexpr int bs = kVoxelBlock;  // every launch of these kernels uses kVoxelBlock threads
  double* msm = reinterpret_cast<double*>(nr_smem) + threadIdx.x;
  double* tsm = msm + 60 * bs;
  const long long v = (long long)blockIdx.x * bs + threadIdx.x;  // 64-bit: v * 60 below
  if (v >= n) return;
  for (int k = 0; k < 60; ++k) msm[k * bs] = schmid[v * 60 + k];
  for (int q = 0; q < kNS; ++q) tsm[q * bs] = 1.0 / crss[v * kNS + q];
  double s[5];
  for (int c = 0; c < 5; ++c) s[c] = s0[v * 5 + c];
  bool capped;
  if (kConstrained) {
    double lam[5], ed[5], rel;
    for (int c = 0; c < 5; ++c) {
      lam[c] = lambda[v * 5 + c];
      ed[c] = p.edot[c] + dtilde[v * 5 + c];
    }
    nr_constrained_smem<0, true>(msm, tsm, bs, p, ParamConsts{p}, lam, ed, s, &rel, &capped);
    if (nr_err) nr_err[v] = rel;
  } else {
    nr_unconstrained_smem<0, true>(msm, tsm, bs, p, p.edot, s, &capped);
  }
  for (int c = 0; c < 5; ++c) out[v * 5 + c] = s[c];
}

static NRParams batch_params(const MaterialParams& mp, const double edot[5], const double* L0,
                             double eps, double max_rss, int max_iter) {
  NRParams p{};
  for (int c = 0; c < 5; ++c) p.edot[c] = edot[c];
  if (L0) {
    for (int k = 0; k < 25; ++k) p.L0[k] = L0[k];
    double inv[25];
    inverse5_colmajor(L0, inv);
    for (int i = 0; i < 5; ++i)
      for (int j = i; j < 5; ++j) p.L0inv[sym5(i, j)] = 0.5 * (inv[j * 5 + i] + inv[i * 5 + j]);
  }
  for (int q = 0; q < kNS; ++q) {
    p.gdot[q] = mp.gdot[q];
    p.nexp[q] = mp.nexp[q];
    p.crss[q] = 1.0;
    p.icrss[q] = 1.0;
  }
  p.eps = eps;
  p.max_rss = max_rss;
  p.max_iter = max_iter;
  set_fp32_copies(p);
  return p;
}

cudaError_t load_solvers_kernels() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k_solvers_nr<true>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_solvers_nr<false>);
  return e;
}

int launch_solvers_constrained(int n, const double* s0, const double* schmid, const double* crss,
                               const MaterialParams& mp, const double edot[5],
                               const double* lambda, const double* dtilde, const double L0[25],
                               double eps, double max_rss, int max_iter, double* out,
                               double* nr_err, cudaStream_t st) {
  NRParams p = batch_params(mp, edot, L0, eps, max_rss, max_iter);
  p.n = n;
  const size_t smem = (size_t)kVoxelBlock * 72 * sizeof(double);
  cudaFuncSetAttribute(k_solvers_nr<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_solvers_nr<true><<<(n + kVoxelBlock - 1) / kVoxelBlock, kVoxelBlock, smem, st>>>(
      p, n, s0, schmid, crss, lambda, dtilde, out, nr_err);
  return 1;
}

int launch_solvers_unconstrained(int n, const double* s0, const double* schmid,
                                 const double* crss, const MaterialParams& mp,
                                 const double edot[5], double eps, double max_rss, int max_iter,
                                 double* out, cudaStream_t st) {
  NRParams p = batch_params(mp, edot, nullptr, eps, max_rss, max_iter);
  p.n = n;
  const size_t smem = (size_t)kVoxelBlock * 72 * sizeof(double);
  cudaFuncSetAttribute(k_solvers_nr<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_solvers_nr<false><<<(n + kVoxelBlock - 1) / kVoxelBlock, kVoxelBlock, smem, st>>>(
      p, n, s0, schmid, crss, nullptr, nullptr, out, nullptr);
  return 1;
}

}  // namespace vpfft
