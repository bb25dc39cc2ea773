// fft_tma.cu -- the y and z passes of the fixed-point loop (see fft_passes.cuh
// for the layouts W, A, B) with their tiles moved by the Tensor Memory
// Accelerator, for FP32 lines of 64, 128 or 256 points:
//   z forward   W rows -> A     z inverse   A -> W rows (times 1/N)
//   y forward   A rows -> B     y inverse   B -> A rows
// Each persistent block walks its tiles (the same lines per tile as the
// warp-copy pass); per tile:
//   * a 3D tiled TMA load brings the tile's input box into shared memory,
//     completing on an mbarrier; the loads of the block's next kTmaStages - 1
//     tiles are in flight while the current one is transformed (a ring of
//     kTmaStages input buffers), so HBM reads overlap the FFT;
//   * the line FFT reads the staged box in its first stage (rows, columns, or
//     pairs of real rows packed as complex lines; the same fixed engine and
//     arithmetic as the warp-copy pass, so results are the same bit for bit);
//   * the transformed lines are rearranged in shared memory into the output
//     box, and a 3D tiled TMA store writes it; the store drains while the
//     next tile is loaded and transformed (bulk async-group, waited on only
//     before the staging box is rewritten).
// Only this GPU's memory is addressed; every load fills its own block's
// shared memory only (no cluster-wide delivery).  Box
// coordinates along the innermost axis are multiples of the tile's lines
// (>= 8 complex values), so every box starts on a 16-byte boundary.
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
#ifndef VPFFT_TMA_STAGES
#define VPFFT_TMA_STAGES 3
#endif
constexpr int kTmaStages = VPFFT_TMA_STAGES;  // input buffers per block (loads in flight: kTmaStages - 1)
std::atomic<int> g_tma_enabled{1};
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

// ---------------------------------------------------------------- pass policies
// A policy describes one pass: its tiles (count, and the box coordinates of
// tile t in the input and output tensor maps), how the first FFT stage reads
// the staged input box, the transform's sign, and how the transformed lines
// become the output box.  Line lengths N of 64, 128 or 256 (the fixed
// engines whose boxes fit the TMA limit of 256 elements per dimension).
struct PassDims {
  int nx, ny, nh, ncomp;
  float scale;  // 1 / (nx ny nz) for the last inverse pass
};
struct TileBoxes {
  int in[3], out[3];
};
constexpr int round128(int bytes) { return (bytes + 127) / 128 * 128; }

// y pass, forward: A[c][x][kz][0..ny) rows of TY consecutive x -> B[c][kz][ky][x] box
template <int N>
struct YFwd {
  static constexpr int kLines = Tiles<float, FixedEngine<N>>::kY;
  static constexpr int kSign = -1;
  static constexpr bool kLineFastest = false;
  static constexpr int kInBytes = kLines * N * 8, kOutBytes = kLines * N * 8;
  __device__ static int tiles(const PassDims& d) { return d.ncomp * d.nh * (d.nx / kLines); }
  __device__ static TileBoxes box(const PassDims& d, int t) {
    const int nxb = d.nx / kLines, c = t / (d.nh * nxb), r = t - c * d.nh * nxb;
    const int kz = r / nxb, x0 = (r - kz * nxb) * kLines;
    return TileBoxes{{0, kz, c * d.nx + x0}, {x0, 0, c * d.nh + kz}};
  }
  __device__ static float2 load(const void* in, int l, int i) {
    return static_cast<const float2*>(in)[l * N + i];
  }
  __device__ static void epilogue(const float2* r, void* stg, const PassDims&, int tid, int nthr) {
    float2* o = static_cast<float2*>(stg);
    for (int e = tid; e < kLines * N; e += nthr) {
      const int ky = e / kLines, l = e - ky * kLines;
      o[e] = r[l * line_stride(N) + sw(ky)];
    }
  }
};
// y pass, inverse: B box (lines across its rows, read as columns) -> A rows
template <int N>
struct YInv {
  static constexpr int kLines = Tiles<float, FixedEngine<N>>::kY;
  static constexpr int kSign = 1;
  static constexpr bool kLineFastest = true;
  static constexpr int kInBytes = kLines * N * 8, kOutBytes = kLines * N * 8;
  __device__ static int tiles(const PassDims& d) { return YFwd<N>::tiles(d); }
  __device__ static TileBoxes box(const PassDims& d, int t) {
    const TileBoxes f = YFwd<N>::box(d, t);
    return TileBoxes{{f.out[0], f.out[1], f.out[2]}, {f.in[0], f.in[1], f.in[2]}};
  }
  __device__ static float2 load(const void* in, int l, int i) {
    return static_cast<const float2*>(in)[i * kLines + l];
  }
  __device__ static void epilogue(const float2* r, void* stg, const PassDims&, int tid, int nthr) {
    float2* o = static_cast<float2*>(stg);
    for (int e = tid; e < kLines * N; e += nthr) {
      const int l = e / N, y = e - l * N;
      o[e] = r[l * line_stride(N) + sw(y)];
    }
  }
};
// z pass, forward (real to half-complex): TZ real rows W[c][x][y0..y0+TZ)[0..nz)
// packed in pairs as complex lines -> A[c][x][0..nh)[y0..y0+TZ) box
template <int N>
struct ZR2C {
  static constexpr int kRows = Tiles<float, FixedEngine<N>>::kZ;
  static constexpr int kLines = kRows / 2;
  static constexpr int kNh = N / 2 + 1;
  static constexpr int kSign = -1;
  static constexpr bool kLineFastest = false;
  static constexpr int kInBytes = kRows * N * 4, kOutBytes = kRows * kNh * 8;
  __device__ static int tiles(const PassDims& d) { return d.ncomp * d.nx * (d.ny / kRows); }
  __device__ static TileBoxes box(const PassDims& d, int t) {
    const int nyb = d.ny / kRows, c = t / (d.nx * nyb), r = t - c * d.nx * nyb;
    const int x = r / nyb, y0 = (r - x * nyb) * kRows;
    return TileBoxes{{0, y0, c * d.nx + x}, {y0, 0, c * d.nx + x}};
  }
  __device__ static float2 load(const void* in, int q, int z) {
    const float* w = static_cast<const float*>(in);
    return float2{w[(2 * q) * N + z], w[(2 * q + 1) * N + z]};
  }
  __device__ static void epilogue(const float2* r, void* stg, const PassDims&, int tid, int nthr) {
    float2* o = static_cast<float2*>(stg);
    constexpr int LS = line_stride(N);
    for (int e = tid; e < kNh * kRows; e += nthr) {
      const int k = e / kRows, l = e - k * kRows, p = l >> 1;
      const float2 Z = r[p * LS + sw(k)];
      const float2 Zm = r[p * LS + sw(k == 0 ? 0 : N - k)];
      float2 v;
      if ((l & 1) == 0) {  // (Z + conj(Zm)) / 2
        v.x = (Z.x + Zm.x) * 0.5f;
        v.y = (Z.y - Zm.y) * 0.5f;
      } else {             // (Z - conj(Zm)) / (2i)
        v.x = (Z.y + Zm.y) * 0.5f;
        v.y = (Zm.x - Z.x) * 0.5f;
      }
      o[e] = v;
    }
  }
};
// z pass, inverse (half-complex to real, times 1/N): A box -> packed full
// lines (Hermitian extension) -> TZ real rows of W
template <int N>
struct ZC2R {
  static constexpr int kRows = Tiles<float, FixedEngine<N>>::kZ;
  static constexpr int kLines = kRows / 2;
  static constexpr int kNh = N / 2 + 1;
  static constexpr int kSign = 1;
  static constexpr bool kLineFastest = true;
  static constexpr int kInBytes = kRows * kNh * 8, kOutBytes = kRows * N * 4;
  __device__ static int tiles(const PassDims& d) { return ZR2C<N>::tiles(d); }
  __device__ static TileBoxes box(const PassDims& d, int t) {
    const TileBoxes f = ZR2C<N>::box(d, t);
    return TileBoxes{{f.out[0], f.out[1], f.out[2]}, {f.in[0], f.in[1], f.in[2]}};
  }
  __device__ static float2 load(const void* in, int q, int k) {
    const float2* b = static_cast<const float2*>(in);  // b[kk][row]
    const bool cj = k >= kNh;
    const int kk = cj ? N - k : k;
    float2 Ae = b[kk * kRows + 2 * q];
    float2 Ao = b[kk * kRows + 2 * q + 1];
    if (cj) {
      Ae.y = -Ae.y;
      Ao.y = -Ao.y;
    }
    if (k == 0 || k == N / 2) {
      Ae.y = 0.f;
      Ao.y = 0.f;
    }
    return float2{Ae.x - Ao.y, Ae.y + Ao.x};
  }
  __device__ static void epilogue(const float2* r, void* stg, const PassDims& d, int tid,
                                  int nthr) {
    float* o = static_cast<float*>(stg);
    constexpr int LS = line_stride(N);
    for (int e = tid; e < kRows * N; e += nthr) {
      const int row = e / N, z = e - row * N;
      const float2 v = r[(row >> 1) * LS + sw(z)];
      o[e] = ((row & 1) ? v.y : v.x) * d.scale;
    }
  }
};

template <class P>
constexpr size_t pass_smem() {
  constexpr int N = P::N_;
  return kTmaStages * (size_t)round128(P::kInBytes) + (size_t)round128(P::kOutBytes) +
         sizeof(float2) * (2 * (size_t)P::kLines * line_stride(N) + N) +
         kTmaStages * sizeof(uint64_t) + 128;
}

template <class P>
__global__ void __launch_bounds__(kTmaThreads)
    k_pass_tma(const __grid_constant__ CUtensorMap in_map,
               const __grid_constant__ CUtensorMap out_map, const float2* __restrict__ twg,
               const PassDims d, IterCtrl* ctrl) {
  constexpr int N = P::N_;
  constexpr int S = kTmaStages;
  constexpr int kInStride = round128(P::kInBytes);
  using E = FixedEngine<N>;
  constexpr int LS = line_stride(N);
  if (ctrl && ctrl->done) return;
  extern __shared__ __align__(128) unsigned char tsm_raw[];
  // TMA boxes start on a 128-byte boundary (the size has 128 bytes of slack)
  unsigned char* const tsm = tsm_raw + ((128u - (smem_u32(tsm_raw) & 127u)) & 127u);
  unsigned char* const in0 = tsm;  // S input buffers of kInStride bytes
  unsigned char* const stg = in0 + S * kInStride;
  float2* const a = reinterpret_cast<float2*>(stg + round128(P::kOutBytes));
  float2* const b = a + P::kLines * LS;
  float2* const tw = b + P::kLines * LS;
  uint64_t* const bar = reinterpret_cast<uint64_t*>(tw + N);
  const int tiles = P::tiles(d);
  E::load_tw(tw, twg, N, threadIdx.x, blockDim.x);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < S; ++j) mbar_init(&bar[j], 1);
    mbar_init_fence();
  }
  __syncthreads();
  auto issue = [&](int t, int buf) {
    const TileBoxes bx = P::box(d, t);
    mbar_expect_tx(&bar[buf], (uint32_t)P::kInBytes);
    tma_load_3d(in0 + buf * kInStride, &in_map, &bar[buf], bx.in[0], bx.in[1], bx.in[2]);
  };
  // The block's k-th tile goes to buffer k mod S as that buffer's (k div S)-th
  // load, completing phase k div S of its mbarrier (waited for with parity
  // (k div S) & 1).  Tiles 0 .. S-2 are issued up front; each step issues
  // tile k+S-1 into the buffer of tile k-1, whose contents the first FFT
  // stage of tile k-1 read behind that tile's barriers.
  if (threadIdx.x == 0)
#pragma unroll
    for (int j = 0; j < S - 1; ++j)
      if ((int)blockIdx.x + j * (int)gridDim.x < tiles) issue(blockIdx.x + j * gridDim.x, j);
  bool failed = false;
  int k = 0, buf = 0, use = 0;  // buf = k mod S, use = k div S
  for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++k) {
    if (threadIdx.x == 0 && t + (S - 1) * (int)gridDim.x < tiles)
      issue(t + (S - 1) * gridDim.x, buf == 0 ? S - 1 : buf - 1);
    const bool ok = mbar_wait(&bar[buf], (uint32_t)(use & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    const void* src = in0 + buf * kInStride;
    const float2* r = E::template fft_loaded<P::kSign, P::kLineFastest>(
        [&](int l, int e) { return P::load(src, l, e); }, a, b, tw, P::kLines, LS, threadIdx.x,
        blockDim.x);
    // the staging box is free once the previous tile's store has read it
    if (threadIdx.x == 0) bulk_wait_read_all();
    __syncthreads();
    P::epilogue(r, stg, d, threadIdx.x, blockDim.x);
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      const TileBoxes bx = P::box(d, t);
      tma_store_3d(&out_map, stg, bx.out[0], bx.out[1], bx.out[2]);
      bulk_commit();
    }
    if (++buf == S) {
      buf = 0;
      ++use;
    }
  }
  if (threadIdx.x == 0) {
    bulk_wait_all();
    if (failed) {
      // the loads still in flight (tiles k .. k+S-1 of this block, those that
      // exist) land in this block's shared memory: wait for them (bounded)
      // before the block exits, then report
      for (int j = 0; j < S; ++j) {
        if ((long long)blockIdx.x + (long long)(k + j) * gridDim.x < tiles)
          mbar_wait(&bar[buf], (uint32_t)(use & 1));
        if (++buf == S) {
          buf = 0;
          ++use;
        }
      }
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

// A rank-3 map over 8-byte (one FP32 complex value) or 4-byte (FP32) elements.
bool map3(CUtensorMap* m, void* base, int elem_bytes, const uint64_t dims[3],
          const uint64_t strides[2], const uint32_t box[3]) {
  EncodeTiled enc = encoder();
  if (!enc) return false;
  const cuuint64_t d[3] = {dims[0], dims[1], dims[2]};
  const cuuint64_t s[2] = {strides[0], strides[1]};
  const cuuint32_t bx[3] = {box[0], box[1], box[2]};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
             3, base, d, s, bx, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// Tensor maps of the three layouts a pass reads or writes, boxes as the
// pass's policy uses them:
//   W[c][x][y][z] real      (z, y, c nx + x)   box (nz, TZ, 1)
//   A[c][x][kz][y] complex  (y, kz, c nx + x)  y pass: box (ny, 1, TY); z pass: box (TZ, nh, 1)
//   B[c][kz][ky][x] complex (x, ky, c nh + kz) box (TY, ny, 1)
struct Maps {
  CUtensorMap in, out;
};

template <int N>
struct Sized {
  static constexpr int N_ = N;
};

template <class P>
bool run_pass(const CUtensorMap& in_map, const CUtensorMap& out_map, const void* tw,
              const PassDims& d, int tiles, IterCtrl* ctrl, cudaStream_t st) {
  constexpr size_t smem = pass_smem<P>();
  static std::atomic<int> blocks{0};
  int nb = blocks.load();
  if (nb == 0) {
    cudaFuncSetAttribute(k_pass_tma<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pass_tma<P>, kTmaThreads, smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    nb = (per_sm < 1 ? 1 : per_sm) * sms;
    blocks.store(nb);
  }
  k_pass_tma<P><<<tiles < nb ? tiles : nb, kTmaThreads, smem, st>>>(
      in_map, out_map, reinterpret_cast<const float2*>(tw), d, ctrl);
  return true;
}

template <template <int> class Pol, int N>
struct Bound : Pol<N>, Sized<N> {};

enum class Kind { kYFwd, kYInv, kZR2C, kZC2R };

template <int N>
bool launch_kind(Kind kind, const Spectral<float>& sp, float* work, IterCtrl* ctrl,
                 cudaStream_t st, int ncomp) {
  const uint64_t c8 = 8, f4 = 4;
  const PassDims d{sp.nx, sp.ny, sp.nh, ncomp, (float)(1.0 / ((double)sp.nx * sp.ny * sp.nz))};
  CUtensorMap A, B, W;
  if (kind == Kind::kYFwd || kind == Kind::kYInv) {
    constexpr int TY = YFwd<N>::kLines;
    if (sp.ny != N || sp.nx % TY != 0) return false;
    const uint64_t da[3] = {(uint64_t)N, (uint64_t)sp.nh, (uint64_t)ncomp * sp.nx};
    const uint64_t sa[2] = {N * c8, (uint64_t)sp.nh * N * c8};
    const uint32_t ba[3] = {(uint32_t)N, 1u, (uint32_t)TY};
    const uint64_t db[3] = {(uint64_t)sp.nx, (uint64_t)N, (uint64_t)ncomp * sp.nh};
    const uint64_t sb[2] = {sp.nx * c8, (uint64_t)N * sp.nx * c8};
    const uint32_t bb[3] = {(uint32_t)TY, (uint32_t)N, 1u};
    if (!map3(&A, sp.X, 8, da, sa, ba) || !map3(&B, sp.X2, 8, db, sb, bb)) return false;
    const int tiles = ncomp * sp.nh * (sp.nx / TY);
    return kind == Kind::kYFwd
               ? run_pass<Bound<YFwd, N>>(A, B, sp.twy, d, tiles, ctrl, st)
               : run_pass<Bound<YInv, N>>(B, A, sp.twy, d, tiles, ctrl, st);
  }
  constexpr int TZ = ZR2C<N>::kRows;
  if (sp.nz != N || sp.ny % TZ != 0 || !work) return false;
  const uint64_t dw[3] = {(uint64_t)N, (uint64_t)sp.ny, (uint64_t)ncomp * sp.nx};
  const uint64_t sw_[2] = {N * f4, (uint64_t)sp.ny * N * f4};
  const uint32_t bw[3] = {(uint32_t)N, (uint32_t)TZ, 1u};
  const uint64_t da[3] = {(uint64_t)sp.ny, (uint64_t)sp.nh, (uint64_t)ncomp * sp.nx};
  const uint64_t sa[2] = {sp.ny * c8, (uint64_t)sp.nh * sp.ny * c8};
  const uint32_t ba[3] = {(uint32_t)TZ, (uint32_t)sp.nh, 1u};
  if (!map3(&W, work, 4, dw, sw_, bw) || !map3(&A, sp.X, 8, da, sa, ba)) return false;
  const int tiles = ncomp * sp.nx * (sp.ny / TZ);
  return kind == Kind::kZR2C ? run_pass<Bound<ZR2C, N>>(W, A, sp.twz, d, tiles, ctrl, st)
                             : run_pass<Bound<ZC2R, N>>(A, W, sp.twz, d, tiles, ctrl, st);
}

bool launch(Kind kind, const Spectral<float>& sp, float* work, const IterCtrl* ctrl,
            cudaStream_t st, int ncomp) {
  if (!g_tma_enabled.load()) return false;
  // the control block is device memory the loop's kernels update; a pass
  // only ORs a status bit into it
  IterCtrl* c = const_cast<IterCtrl*>(ctrl);
  const int n = (kind == Kind::kYFwd || kind == Kind::kYInv) ? sp.ny : sp.nz;
  switch (n) {
    case 64: return launch_kind<64>(kind, sp, work, c, st, ncomp);
    case 128: return launch_kind<128>(kind, sp, work, c, st, ncomp);
    case 256: return launch_kind<256>(kind, sp, work, c, st, ncomp);
    default: return false;
  }
}

}  // namespace
}  // namespace fft

// The TMA passes for FP32 spectra whose line length on the pass's axis is 64,
// 128 or 256 and whose other axis holds whole tiles; false (nothing launched)
// when a pass does not apply, is switched off, or the tensor-map encoder is
// unavailable.
bool launch_y_fwd_tma(const Spectral<float>& sp, const IterCtrl* ctrl, cudaStream_t st,
                      int ncomp) {
  return fft::launch(fft::Kind::kYFwd, sp, nullptr, ctrl, st, ncomp);
}
bool launch_y_inv_tma(const Spectral<float>& sp, const IterCtrl* ctrl, cudaStream_t st,
                      int ncomp) {
  return fft::launch(fft::Kind::kYInv, sp, nullptr, ctrl, st, ncomp);
}
bool launch_z_r2c_tma(const Spectral<float>& sp, const float* work, const IterCtrl* ctrl,
                      cudaStream_t st, int ncomp) {
  return fft::launch(fft::Kind::kZR2C, sp, const_cast<float*>(work), ctrl, st, ncomp);
}
bool launch_z_c2r_tma(const Spectral<float>& sp, float* work, const IterCtrl* ctrl,
                      cudaStream_t st, int ncomp) {
  return fft::launch(fft::Kind::kZC2R, sp, work, ctrl, st, ncomp);
}

int set_tma_passes(int enable) {
  if (enable < 0) return fft::g_tma_enabled.load();
  return fft::g_tma_enabled.exchange(enable ? 1 : 0);
}

}  // namespace vpfft
