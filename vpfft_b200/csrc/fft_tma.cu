// fft_tma.cu -- the forward y pass of the fixed-point loop (A -> B, see
// fft_passes.cuh) with its tiles moved by the Tensor Memory Accelerator.
//
// Each persistent block walks its tiles (TY consecutive x of one kz and one
// component, TY = the pass's lines per tile); per tile:
//   * a 3D tiled TMA load brings the TY y-lines A[c][x0..x0+TY)[kz][0..ny)
//     into shared memory (dense rows), completing on an mbarrier; the load of
//     the block's next tile is issued before the current one is transformed,
//     into the other of two input buffers, so HBM reads overlap the FFT;
//   * the line FFT (the same fixed engine and arithmetic as the warp-copy
//     pass, so the spectrum is the same bit for bit) reads the dense rows in
//     its first stage;
//   * the result is transposed in shared memory into the box of the output,
//     B[c][kz][0..ny)[x0..x0+TY), and a 3D tiled TMA store writes it; the store
//     drains while the next tile is loaded and transformed (bulk async-group,
//     waited on only before the staging buffer is rewritten).
// Only this GPU's memory is addressed; no load uses cluster multicast.
//
// Every wait on an mbarrier is bounded: after kWaitPolls failed polls the
// block stops, waits (bounded) for its own copies in flight and reports
// kStatusDeviceTimeout in the loop's control block.
#include <cuda.h>  // CUtensorMap and its enums (types only; the encoder is fetched at run time)
#include <cuda_runtime.h>

#include <atomic>

#include "fft_passes.cuh"

namespace vpfft {
namespace fft {
namespace {

constexpr int kTmaThreads = 256;
constexpr long long kWaitPolls = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of bar; false when it did not complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < kWaitPolls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int c0,
                                             int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src))
      : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Shared memory of the kernel for line length N (bytes): two input tiles, the
// output staging tile, the FFT's two padded buffers, the twiddles, two
// mbarriers, and slack for aligning the tiles.
template <int N>
constexpr size_t tma_y_smem() {
  using Ti = Tiles<float, FixedEngine<N>>;
  return sizeof(float2) * (3 * (size_t)Ti::kY * N + 2 * (size_t)Ti::kY * line_stride(N) + N) +
         2 * sizeof(uint64_t) + 128;
}

template <int N>
__global__ void __launch_bounds__(kTmaThreads)
    k_pass_y_fwd_tma(const __grid_constant__ CUtensorMap in_map,
                     const __grid_constant__ CUtensorMap out_map,
                     const float2* __restrict__ twg, int nx, int nh, int ncomp, IterCtrl* ctrl) {
  using E = FixedEngine<N>;
  constexpr int TY = Tiles<float, E>::kY;
  constexpr int LS = line_stride(N);
  constexpr uint32_t kTileBytes = TY * N * sizeof(float2);
  if (ctrl && ctrl->done) return;
  extern __shared__ __align__(128) unsigned char tsm_raw[];
  // TMA tiles start on a 128-byte boundary (the size has 128 bytes of slack)
  unsigned char* tsm = tsm_raw + ((128u - (smem_u32(tsm_raw) & 127u)) & 127u);
  float2* const in0 = reinterpret_cast<float2*>(tsm);
  float2* const in1 = in0 + TY * N;
  float2* const stg = in1 + TY * N;
  float2* const a = stg + TY * N;
  float2* const b = a + TY * LS;
  float2* const tw = b + TY * LS;
  uint64_t* const bar = reinterpret_cast<uint64_t*>(tw + N);
  const int nxb = nx / TY;
  const int tiles = ncomp * nh * nxb;
  auto tile_at = [&](int t, int* c, int* kz, int* x0) {
    *c = t / (nh * nxb);
    const int r = t - *c * nh * nxb;
    *kz = r / nxb;
    *x0 = (r - *kz * nxb) * TY;
  };
  E::load_tw(tw, twg, N, threadIdx.x, blockDim.x);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  // loads issued and waited for per buffer: the m-th use of a buffer's
  // mbarrier completes phase m, waited for with parity m & 1
  int issued0 = 0, issued1 = 0, waited0 = 0, waited1 = 0;
  auto issue = [&](int t, int i) {
    int c, kz, x0;
    tile_at(t, &c, &kz, &x0);
    mbar_expect_tx(&bar[i], kTileBytes);
    tma_load_3d(i ? in1 : in0, &in_map, &bar[i], 0, kz, c * nx + x0);
    if (i) ++issued1; else ++issued0;
  };
  if (threadIdx.x == 0 && (int)blockIdx.x < tiles) issue(blockIdx.x, 0);
  bool failed = false;
  int k = 0;
  for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++k) {
    const int i = k & 1;
    // the next tile into the other buffer: its previous contents (tile k-1)
    // were read by the first FFT stage, behind the barriers of that tile
    if (threadIdx.x == 0 && t + (int)gridDim.x < tiles) issue(t + gridDim.x, i ^ 1);
    const int use = k >> 1;  // this tile is use `use` of buffer i
    const bool ok = mbar_wait(&bar[i], (uint32_t)(use & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    if (i) waited1 = use + 1; else waited0 = use + 1;
    const float2* r = E::template fft_dense_in<-1>(i ? in1 : in0, a, b, tw, TY, LS,
                                                   threadIdx.x, blockDim.x);
    // the staging tile is free once the previous tile's store has read it
    if (threadIdx.x == 0) bulk_wait_read_all();
    __syncthreads();
    for (int e = threadIdx.x; e < TY * N; e += blockDim.x) {
      const int ky = e / TY, l = e - ky * TY;
      stg[e] = r[l * LS + sw(ky)];
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      int c, kz, x0;
      tile_at(t, &c, &kz, &x0);
      tma_store_3d(&out_map, stg, x0, 0, c * nh + kz);
      bulk_commit();
    }
  }
  if (threadIdx.x == 0) {
    bulk_wait_all();
    if (failed) {
      // loads still in flight land in this block's shared memory: wait for
      // them (bounded) before the block exits, then report
      if (issued0 > waited0) mbar_wait(&bar[0], (uint32_t)(waited0 & 1));
      if (issued1 > waited1) mbar_wait(&bar[1], (uint32_t)(waited1 & 1));
      if (ctrl) atomicOr(&ctrl->status, (int)kStatusDeviceTimeout);
    }
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = []() -> EncodeTiled {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// A rank-3 map over 8-byte elements (one FP32 complex value each).
bool map3(CUtensorMap* m, void* base, const uint64_t dims[3], const uint64_t strides[2],
          const uint32_t box[3]) {
  EncodeTiled enc = encoder();
  if (!enc) return false;
  const cuuint64_t d[3] = {dims[0], dims[1], dims[2]};
  const cuuint64_t s[2] = {strides[0], strides[1]};
  const cuuint32_t bx[3] = {box[0], box[1], box[2]};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, base, d, s, bx, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int N>
bool launch_n(const Spectral<float>& sp, IterCtrl* ctrl, cudaStream_t st, int ncomp) {
  constexpr int TY = Tiles<float, FixedEngine<N>>::kY;
  if (sp.ny != N || sp.nx % TY != 0) return false;
  // A[c][x][kz][y] as (y, kz, c nx + x); B[c][kz][ky][x] as (x, ky, c nh + kz)
  const uint64_t e = sizeof(float2);
  CUtensorMap in_map, out_map;
  const uint64_t din[3] = {(uint64_t)N, (uint64_t)sp.nh, (uint64_t)ncomp * sp.nx};
  const uint64_t sin[2] = {N * e, (uint64_t)sp.nh * N * e};
  const uint32_t bin[3] = {(uint32_t)N, 1u, (uint32_t)TY};
  const uint64_t dout[3] = {(uint64_t)sp.nx, (uint64_t)N, (uint64_t)ncomp * sp.nh};
  const uint64_t sout[2] = {sp.nx * e, (uint64_t)N * sp.nx * e};
  const uint32_t bout[3] = {(uint32_t)TY, (uint32_t)N, 1u};
  if (!map3(&in_map, sp.X, din, sin, bin) || !map3(&out_map, sp.X2, dout, sout, bout))
    return false;
  constexpr size_t smem = tma_y_smem<N>();
  static std::atomic<int> blocks{0};
  int nb = blocks.load();
  if (nb == 0) {
    cudaFuncSetAttribute(k_pass_y_fwd_tma<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pass_y_fwd_tma<N>, kTmaThreads,
                                                  smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    nb = (per_sm < 1 ? 1 : per_sm) * sms;
    blocks.store(nb);
  }
  const int tiles = ncomp * sp.nh * (sp.nx / TY);
  k_pass_y_fwd_tma<N><<<tiles < nb ? tiles : nb, kTmaThreads, smem, st>>>(
      in_map, out_map, reinterpret_cast<const float2*>(sp.twy), sp.nx, sp.nh, ncomp, ctrl);
  return true;
}

std::atomic<int> g_tma_enabled{0};

}  // namespace
}  // namespace fft

// The TMA forward y pass for FP32 spectra with y lines of 64, 128 or 256
// points and nx a multiple of the tile's line count; false (nothing launched)
// when it does not apply or the tensor-map encoder is unavailable.
bool launch_y_fwd_tma(const Spectral<float>& sp, const IterCtrl* ctrl, cudaStream_t st,
                      int ncomp) {
  if (!fft::g_tma_enabled.load()) return false;
  // the control block is device memory the loop's kernels update; the pass
  // only ORs a status bit into it
  IterCtrl* c = const_cast<IterCtrl*>(ctrl);
  switch (sp.ny) {
    case 64: return fft::launch_n<64>(sp, c, st, ncomp);
    case 128: return fft::launch_n<128>(sp, c, st, ncomp);
    case 256: return fft::launch_n<256>(sp, c, st, ncomp);
    default: return false;
  }
}

int set_tma_passes(int enable) {
  if (enable < 0) return fft::g_tma_enabled.load();
  return fft::g_tma_enabled.exchange(enable ? 1 : 0);
}

}  // namespace vpfft
