// fft_passes.cuh -- the five line passes of the 3D real <-> half-complex
// transforms, templated on the line engine (fft_engine.cuh), and the table of
// kernel entry points of one engine (PassSet).
//
// Layouts (component c outermost, 5 components in the fixed-point loop):
//   W[c][x][y][z]   real field (P before the forward transform, d~ after)
//   A[c][x][kz][y]  after the z pass (kz in [0, nz/2])
//   B[c][kz][ky][x] after the y pass; the x pass works in place on B
//
//   pass_z_r2c   W -> A   pairs of real z-lines packed as one complex line
//   pass_y<-1>   A -> B
//   pass_x       B -> B   forward x FFT, [dhat = -Gbar(k) phat, inverse x FFT]
//   pass_y<+1>   B -> A
//   pass_z_c2r   A -> W   Hermitian extension, pairs unpacked, times 1/N
//
// Each block transforms a tile of consecutive lines of the flattened index of
// the two other axes (z pass: x ny + y; y pass: kz nx + x; x pass:
// kz ny + ky), so a tile may span several rows of a small grid.  Global reads
// and writes go in runs that are contiguous in the layout being read or
// written; the transpose between the two happens in the shared-memory tile.
// No thread-block cluster features are used.
#pragma once

#include <cuda_runtime.h>

#include "fft_engine.cuh"
#include "kernel_common.cuh"
#include "kernels.h"

namespace vpfft {
namespace fft {

// Lines per block and threads per block of an engine.  Fixed engines of
// length >= 64 hold about 2048 (FP32) or 1024 (FP64) complex values per
// ping-pong buffer; shorter lines take 512 so that a small single grid still
// spreads over many blocks.  The z and y passes run 256 (FP32) or 128 (FP64) threads
// per block, the x pass (two transforms and the Green operator) 128 threads,
// the settings measured fastest at 256^3.  The generic engine keeps 256
// threads and its short tiles.
// kEl != 0 selects a batched tile family: about kEl complex values per buffer
// (512, 1024 or 2048, at most the long tile), chosen by the batch's options or
// its autotuner.  A tile only groups lines: every line goes through the same
// arithmetic whatever the family, and the line transforms spell out their
// fused multiply-adds, so every family gives the same bits in both precisions.
template <typename S, class E, int kEl = 0>
struct Tiles {
  static constexpr bool kF32 = sizeof(S) == 4;
  static constexpr int kLong = kF32 ? 2048 : 1024;
  static constexpr int kElems = kEl ? (kEl < kLong ? kEl : kLong) : (E::kN >= 64 ? kLong : 512);
  static constexpr int kThreads = E::kN ? (kF32 ? 256 : 128) : 256;  // z and y passes
  static constexpr int kThreadsX = E::kN ? 128 : 256;                // x pass
  // x-pass blocks per SM the registers are capped for: FP32 at 6 (85
  // registers; measured 15 % faster than 4), FP64 at 4 (more would spill).
  // The batched x pass reads its Green constants from shared memory at each
  // use (GreenShared), which keeps it within the same caps without spills.
  static constexpr int kMinBlocksX = (E::kN && kF32) ? 6 : 512 / kThreadsX;
  static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  static constexpr int kZ = E::kN ? cmax(2, 2 * (kElems / E::kN)) : 16;  // real z-lines
  static constexpr int kY = E::kN ? cmax(1, kElems / E::kN) : (sizeof(S) == 4 ? 16 : 8);
  static constexpr int kX = E::kN ? cmax(1, kElems / (5 * E::kN)) : (sizeof(S) == 4 ? 4 : 2);
};
// Batched tile families of an engine: 512, 1024 (and 2048 in FP32) complex
// values per buffer for the fixed engines up to 96 points; one (the long
// tile) for longer lines and for the generic engine, whose tiles do not
// depend on it.
template <typename S, class E>
constexpr int batch_families() {
  return (E::kN == 0 || E::kN > 96) ? 1 : (sizeof(S) == 4 ? 3 : 2);
}
template <typename S, class E>
constexpr int batch_family_elems(int f) {
  return batch_families<S, E>() == 1 ? Tiles<S, E>::kLong : (512 << f);
}


// Copy of nrows rows of len elements: warp w takes rows w, w + nwarps, ...;
// lanes stride 32 along the row with kU independent loads in flight per lane
// before the matching stores.
constexpr int kU = 8;
template <typename V, typename G, typename P>
__device__ __forceinline__ void copy_rows(int nrows, int len, G get, P put) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int row = warp; row < nrows; row += nw) {
    for (int c0 = lane; c0 < len; c0 += 32 * kU) {
      V v[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int c = c0 + 32 * u;
        if (c < len) v[u] = get(row, c);
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int c = c0 + 32 * u;
        if (c < len) put(row, c, v[u]);
      }
    }
  }
}

// Copy of nrows x W elements, element i = (row i / W, column i % W), with
// consecutive threads on consecutive columns; kU loads in flight.
template <int W, typename V, typename G, typename P>
__device__ __forceinline__ void copy_short_rows(int nrows, G get, P put) {
  const int total = nrows * W, bd = blockDim.x;
  for (int base = threadIdx.x; base < total; base += kU * bd) {
    V v[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int i = base + u * bd;
      if (i < total) v[u] = get(i / W, i % W);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int i = base + u * bd;
      if (i < total) put(i / W, i % W, v[u]);
    }
  }
}

// ---------------------------------------------------------------- z, forward
// Tile bt of component c: real lines f = bt TZ ... (f = x ny + y).
template <typename S, class E, class TL>
__device__ __forceinline__ void pass_z_r2c_body(const S* __restrict__ W,
                                                typename CX<S>::T* __restrict__ A,
                                                const LinePlan& pl, const FastDiv& dny,
                                                const typename CX<S>::T* __restrict__ twg, int nx,
                                                int ny, int nh, int bt, int c) {
  using T = typename CX<S>::T;
  constexpr int TZ = TL::kZ;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nz = E::n(pl), ls = line_stride(nz);
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + nz;
  T* b = a + (TZ / 2) * ls;
  E::load_tw(tw, twg, nz, threadIdx.x, blockDim.x);
  const int nxy = nx * ny;
  const int f0 = bt * TZ;
  const int nf = min(TZ, nxy - f0);
  const int npair = (nf + 1) / 2;
  const S* src = W + ((long long)c * nxy + f0) * nz;
  // rows 2q and 2q+1 packed as line q: each lane reads both rows' element and
  // stores one complex value
  copy_rows<T>(
      npair, nz,
      [&](int q, int z) {
        const int l = 2 * q;
        return T{l < nf ? src[l * nz + z] : S(0), l + 1 < nf ? src[(l + 1) * nz + z] : S(0)};
      },
      [&](int q, int z, T v) { a[q * ls + sw(z)] = v; });
  __syncthreads();
  const T* r = E::template fft<-1>(a, b, tw, pl, npair, ls, threadIdx.x, blockDim.x);
  T* dst = A + (long long)c * nx * nh * ny;
  copy_short_rows<TZ, T>(
      nh,
      [&](int k, int l) {
        const int p = l >> 1;
        const T Z = r[p * ls + sw(k)];
        const T Zm = r[p * ls + sw(k == 0 ? 0 : nz - k)];
        T o;
        if ((l & 1) == 0) {  // (Z + conj(Zm)) / 2
          o.x = (Z.x + Zm.x) * S(0.5);
          o.y = (Z.y - Zm.y) * S(0.5);
        } else {             // (Z - conj(Zm)) / (2i)
          o.x = (Z.y + Zm.y) * S(0.5);
          o.y = (Zm.x - Z.x) * S(0.5);
        }
        return o;
      },
      [&](int k, int l, T v) {
        if (l < nf) {
          const int f = f0 + l;
          const int x = (int)fast_div((uint32_t)f, dny);
          dst[(x * nh + k) * ny + (f - x * ny)] = v;
        }
      });
}

// ---------------------------------------------------------------- z, inverse
template <typename S, class E, class TL>
__device__ __forceinline__ void pass_z_c2r_body(const typename CX<S>::T* __restrict__ A,
                                                S* __restrict__ W, const LinePlan& pl,
                                                const FastDiv& dny,
                                                const typename CX<S>::T* __restrict__ twg, int nx,
                                                int ny, int nh, S scale, int bt, int c) {
  using T = typename CX<S>::T;
  constexpr int TZ = TL::kZ;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nz = E::n(pl), ls = line_stride(nz);
  // a: (TZ/2) packed lines; b: the tile's half spectra first (TZ x (nh+1)),
  // then the FFT's ping-pong buffer -- sized max of the two (pass_smem)
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + nz;
  T* b = a + (TZ / 2) * ls;
  E::load_tw(tw, twg, nz, threadIdx.x, blockDim.x);
  const int nxy = nx * ny;
  const int f0 = bt * TZ;
  const int nf = min(TZ, nxy - f0);
  const int npair = (nf + 1) / 2;
  const T* src = A + (long long)c * nx * nh * ny;
  const int hs = nh + 1;
  copy_short_rows<TZ, T>(
      nh,
      [&](int k, int l) {
        if (l >= nf) return T{S(0), S(0)};
        const int f = f0 + l;
        const int x = (int)fast_div((uint32_t)f, dny);
        return src[(x * nh + k) * ny + (f - x * ny)];
      },
      [&](int k, int l, T v) { b[l * hs + k] = v; });
  __syncthreads();
  // packed full lines: Z = A_even + i A_odd, Hermitian extension for k >= nh
  for (int i = threadIdx.x; i < npair * nz; i += blockDim.x) {
    const int p = E::div_n(i, pl), k = i - p * nz;
    const bool cj = k >= nh;
    const int kk = cj ? nz - k : k;
    T Ae = b[(2 * p) * hs + kk];
    T Ao = b[(2 * p + 1) * hs + kk];
    if (cj) {
      Ae.y = -Ae.y;
      Ao.y = -Ao.y;
    }
    if (k == 0 || ((nz & 1) == 0 && k == nz / 2)) {
      Ae.y = S(0);
      Ao.y = S(0);
    }
    a[p * ls + sw(k)] = T{Ae.x - Ao.y, Ae.y + Ao.x};
  }
  __syncthreads();
  const T* r = E::template fft<1>(a, b, tw, pl, npair, ls, threadIdx.x, blockDim.x);
  S* dst = W + ((long long)c * nxy + f0) * nz;
  // line q holds rows 2q (real part) and 2q+1 (imaginary part)
  copy_rows<T>(
      npair, nz, [&](int q, int z) { return r[q * ls + sw(z)]; },
      [&](int q, int z, T v) {
        dst[2 * q * nz + z] = v.x * scale;
        if (2 * q + 1 < nf) dst[(2 * q + 1) * nz + z] = v.y * scale;
      });
}

// ---------------------------------------------------------------- y passes
// Lines g = kz nx + x of component c.  Forward: A[c][x][kz][y] ->
// B[c][kz][ky][x]; inverse: B -> A.
template <int SIGN, typename S, class E, class TL>
__device__ __forceinline__ void pass_y_body(const typename CX<S>::T* __restrict__ in,
                                            typename CX<S>::T* __restrict__ out,
                                            const LinePlan& pl, const FastDiv& dnx,
                                            const typename CX<S>::T* __restrict__ twg, int nx,
                                            int nh, int bt, int c) {
  using T = typename CX<S>::T;
  constexpr int TY = TL::kY;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ny = E::n(pl), ls = line_stride(ny);
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + ny;
  T* b = a + TY * ls;
  E::load_tw(tw, twg, ny, threadIdx.x, blockDim.x);
  const int g0 = bt * TY;
  const int ng = min(TY, nh * nx - g0);
  // component base (offsets inside a component are < 2^31 for dimensions <= 512)
  const long long cb = (long long)c * nx * nh * ny;
  const T* inc = in + cb;
  T* outc = out + cb;
  // A line (x, kz) starts at (x nh + kz) ny; B element (kz, ky, x) is at (kz ny + ky) nx + x
  auto a_row = [&](int l) {
    const int g = g0 + l;
    const int kz = (int)fast_div((uint32_t)g, dnx);
    return ((g - kz * nx) * nh + kz) * ny;
  };
  auto b_at = [&](int ky, int l) {
    const int g = g0 + l;
    const int kz = (int)fast_div((uint32_t)g, dnx);
    return (kz * ny + ky) * nx + (g - kz * nx);
  };
  if (SIGN < 0) {
    copy_rows<T>(
        TY, ny, [&](int l, int y) { return l < ng ? inc[a_row(l) + y] : T{S(0), S(0)}; },
        [&](int l, int y, T v) { a[l * ls + sw(y)] = v; });
  } else {
    copy_short_rows<TY, T>(
        ny, [&](int y, int l) { return l < ng ? inc[b_at(y, l)] : T{S(0), S(0)}; },
        [&](int y, int l, T v) { a[l * ls + sw(y)] = v; });
  }
  __syncthreads();
  const T* r = E::template fft<SIGN>(a, b, tw, pl, TY, ls, threadIdx.x, blockDim.x);
  if (SIGN < 0) {
    copy_short_rows<TY, T>(
        ny, [&](int y, int l) { return r[l * ls + sw(y)]; },
        [&](int y, int l, T v) {
          if (l < ng) outc[b_at(y, l)] = v;
        });
  } else {
    copy_rows<T>(
        ng, ny, [&](int l, int y) { return r[l * ls + sw(y)]; },
        [&](int l, int y, T v) { outc[a_row(l) + y] = v; });
  }
}

// ---------------------------------------------------------------- x pass
// In place on B[c][kz][ky][x], lines f = kz ny + ky of all ncomp components:
// MODE 0 forward, 1 inverse, 2 forward + Green operator computed per wave
// vector + inverse, 3 forward + Green operator read from a stored table +
// inverse.  The table (gtab, MODE 3) holds the kGreenStored values of every
// wave vector of the half spectrum, value j of wave vector (f, x) at
// gtab[j nh ny nx + f nx + x] (consecutive x contiguous: coalesced); MODE 2
// and MODE 3 perform the same operations on the same values.
template <int MODE, typename S, class E, class TL, class G>
__device__ __forceinline__ void pass_x_body(typename CX<S>::T* __restrict__ B, const LinePlan& pl,
                                            const FastDiv& dny,
                                            const typename CX<S>::T* __restrict__ twg,
                                            const G& gp,
                                            const S* __restrict__ gtab, int ny, int nh, int ncomp,
                                            int bt) {
  using T = typename CX<S>::T;
  constexpr int TK = TL::kX;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nx = E::n(pl), ls = line_stride(nx);
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + nx;
  T* b = a + ncomp * TK * ls;
  E::load_tw(tw, twg, nx, threadIdx.x, blockDim.x);
  const int f0 = bt * TK;
  const int nfk = min(TK, nh * ny - f0);
  // component stride and the block's offset: < 2^31 for dimensions <= 512
  const int cs = nh * ny * nx;
  T* Bb = B + (long long)f0 * nx;
  const int nl = ncomp * TK;
  copy_rows<T>(
      nl, nx,
      [&](int L, int xx) {
        const int c = L / TK, kl = L - c * TK;
        return kl < nfk ? Bb[c * cs + kl * nx + xx] : T{S(0), S(0)};
      },
      [&](int L, int xx, T v) { a[L * ls + sw(xx)] = v; });
  __syncthreads();
  T* r = a;
  T* o = b;
  if (MODE != 1) {
    r = E::template fft<-1>(a, b, tw, pl, nl, ls, threadIdx.x, blockDim.x);
    o = (r == a) ? b : a;
  }
  if constexpr (MODE == 2) {
    for (int i = threadIdx.x; i < TK * nx; i += blockDim.x) {
      const int kl = E::div_n(i, pl), xx = i - kl * nx;
      if (kl >= nfk) continue;
      const int f = f0 + kl;
      const int kz = (int)fast_div((uint32_t)f, dny);
      S pre[5], pim[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const T z = r[(c * TK + kl) * ls + sw(xx)];
        pre[c] = z.x;
        pim[c] = z.y;
      }
      green_apply<S>(gp, xx, f - kz * ny, kz, pre, pim);
#pragma unroll
      for (int c = 0; c < 5; ++c) r[(c * TK + kl) * ls + sw(xx)] = T{pre[c], pim[c]};
    }
    __syncthreads();
  }
  if constexpr (MODE == 3) {
    const long long M = (long long)nh * ny * nx;
    for (int i = threadIdx.x; i < TK * nx; i += blockDim.x) {
      const int kl = E::div_n(i, pl), xx = i - kl * nx;
      if (kl >= nfk) continue;
      const int f = f0 + kl;
      const int kz = (int)fast_div((uint32_t)f, dny);
      S pre[5], pim[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const T z = r[(c * TK + kl) * ls + sw(xx)];
        pre[c] = z.x;
        pim[c] = z.y;
      }
      green_apply_stored<S>(gp, xx, f - kz * ny, kz, gtab, M, (long long)f * nx + xx, pre, pim);
#pragma unroll
      for (int c = 0; c < 5; ++c) r[(c * TK + kl) * ls + sw(xx)] = T{pre[c], pim[c]};
    }
    __syncthreads();
  }
  if (MODE != 0) r = E::template fft<1>(r, o, tw, pl, nl, ls, threadIdx.x, blockDim.x);
  copy_rows<T>(
      nl, nx, [&](int L, int xx) { return r[L * ls + sw(xx)]; },
      [&](int L, int xx, T v) {
        const int c = L / TK, kl = L - c * TK;
        if (kl < nfk) Bb[c * cs + kl * nx + xx] = v;
      });
}

// ---------------------------------------------------------------- kernels
template <typename S, class E>
__global__ void __launch_bounds__(Tiles<S, E>::kThreads)
    k_pass_z_r2c(const S* __restrict__ W, typename CX<S>::T* __restrict__ A, LinePlan pl,
                 FastDiv dny, const typename CX<S>::T* __restrict__ twg, int nx, int ny, int nh,
                 const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_z_r2c_body<S, E, Tiles<S, E>>(W, A, pl, dny, twg, nx, ny, nh, blockIdx.x, blockIdx.y);
}
template <typename S, class E>
__global__ void __launch_bounds__(Tiles<S, E>::kThreads)
    k_pass_z_c2r(const typename CX<S>::T* __restrict__ A, S* __restrict__ W, LinePlan pl,
                 FastDiv dny, const typename CX<S>::T* __restrict__ twg, int nx, int ny, int nh,
                 S scale, const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_z_c2r_body<S, E, Tiles<S, E>>(A, W, pl, dny, twg, nx, ny, nh, scale, blockIdx.x,
                                     blockIdx.y);
}
template <int SIGN, typename S, class E>
__global__ void __launch_bounds__(Tiles<S, E>::kThreads)
    k_pass_y(const typename CX<S>::T* __restrict__ in, typename CX<S>::T* __restrict__ out,
             LinePlan pl, FastDiv dnx, const typename CX<S>::T* __restrict__ twg, int nx, int nh,
             const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_y_body<SIGN, S, E, Tiles<S, E>>(in, out, pl, dnx, twg, nx, nh, blockIdx.x, blockIdx.y);
}
template <int MODE, typename S, class E>
__global__ void __launch_bounds__(Tiles<S, E>::kThreadsX, Tiles<S, E>::kMinBlocksX)
    k_pass_x(typename CX<S>::T* __restrict__ B, LinePlan pl, FastDiv dny,
             const typename CX<S>::T* __restrict__ twg, GreenParams<S> gp,
             const S* __restrict__ gtab, int ny, int nh, int ncomp, const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_x_body<MODE, S, E, Tiles<S, E>>(B, pl, dny, twg, gp, gtab, ny, nh, ncomp, blockIdx.x);
}

// Batched passes of the fixed-point iteration (5 components): block -> slot,
// then the slot's tile from the local block index.  A block copies the slot's
// FFT fields (FftSlot, and the Green constants for the x pass) to shared
// memory; the runtime line plan of the generic engine is read in place.
template <typename S>
struct SlotFft {
  FftSlot<S> fs;
  GreenParams<S> gp;
};
template <typename S>
__device__ __forceinline__ const SlotDesc<S>* batch_pass_setup(const SlotDesc<S>* desc,
                                                               const BatchLaunch& bl, bool green,
                                                               SlotFft<S>* sm, int* lb) {
  const SlotDesc<S>* d = &desc[batch_slot(bl, blockIdx.x, lb)];
  if (d->ctrl->done) return nullptr;
  copy_struct(&sm->fs, &d->fs);
  if (green) copy_struct(&sm->gp, &d->gp);
  __syncthreads();
  return d;
}

template <typename S, class E, int kEl>
__global__ void __launch_bounds__(Tiles<S, E, kEl>::kThreads)
    k_pass_z_r2c_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  using T = typename CX<S>::T;
  using TL = Tiles<S, E, kEl>;
  __shared__ SlotFft<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, false, &sm, &lb);
  if (!d) return;
  const FftSlot<S>& fs = sm.fs;
  const int gt = (fs.nx * fs.ny + TL::kZ - 1) / TL::kZ;
  const int c = lb / gt;
  pass_z_r2c_body<S, E, TL>(fs.work, reinterpret_cast<T*>(fs.X), d->sp.pz, fs.dny,
                            reinterpret_cast<const T*>(fs.twz), fs.nx, fs.ny, fs.nh, lb - c * gt,
                            c);
}
template <typename S, class E, int kEl>
__global__ void __launch_bounds__(Tiles<S, E, kEl>::kThreads)
    k_pass_z_c2r_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  using T = typename CX<S>::T;
  using TL = Tiles<S, E, kEl>;
  __shared__ SlotFft<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, false, &sm, &lb);
  if (!d) return;
  const FftSlot<S>& fs = sm.fs;
  const int gt = (fs.nx * fs.ny + TL::kZ - 1) / TL::kZ;
  const int c = lb / gt;
  const S scale = S(1.0 / ((double)fs.nx * fs.ny * fs.nz));
  pass_z_c2r_body<S, E, TL>(reinterpret_cast<const T*>(fs.X), fs.work, d->sp.pz, fs.dny,
                            reinterpret_cast<const T*>(fs.twz), fs.nx, fs.ny, fs.nh, scale,
                            lb - c * gt, c);
}
template <int SIGN, typename S, class E, int kEl>
__global__ void __launch_bounds__(Tiles<S, E, kEl>::kThreads)
    k_pass_y_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  using T = typename CX<S>::T;
  using TL = Tiles<S, E, kEl>;
  __shared__ SlotFft<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, false, &sm, &lb);
  if (!d) return;
  const FftSlot<S>& fs = sm.fs;
  const int gt = (fs.nh * fs.nx + TL::kY - 1) / TL::kY;
  const int c = lb / gt;
  const T* in = reinterpret_cast<const T*>(SIGN < 0 ? fs.X : fs.X2);
  T* out = reinterpret_cast<T*>(SIGN < 0 ? fs.X2 : fs.X);
  pass_y_body<SIGN, S, E, TL>(in, out, d->sp.py, fs.dnx, reinterpret_cast<const T*>(fs.twy),
                              fs.nx, fs.nh, lb - c * gt, c);
}
template <typename S, class E, int kEl>
__global__ void __launch_bounds__(Tiles<S, E, kEl>::kThreadsX, Tiles<S, E, kEl>::kMinBlocksX)
    k_pass_x_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  using T = typename CX<S>::T;
  using TL = Tiles<S, E, kEl>;
  __shared__ SlotFft<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, true, &sm, &lb);
  if (!d) return;
  const FftSlot<S>& fs = sm.fs;
  pass_x_body<2, S, E, TL>(reinterpret_cast<T*>(fs.X2), d->sp.px, fs.dny,
                           reinterpret_cast<const T*>(fs.twx), GreenShared<S>(&sm.gp), nullptr,
                           fs.ny, fs.nh, 5, lb);
}

// ---------------------------------------------------------------- entry table
// The batched passes of one tile family.
template <typename S>
struct BatchPasses {
  int tz, ty, tk;  // real z-lines, y-lines and ky-lines (per component) per block
  void (*z_r2c)(const SlotDesc<S>*, const BatchLaunch);
  void (*z_c2r)(const SlotDesc<S>*, const BatchLaunch);
  void (*y_fwd)(const SlotDesc<S>*, const BatchLaunch);
  void (*y_inv)(const SlotDesc<S>*, const BatchLaunch);
  void (*x_green)(const SlotDesc<S>*, const BatchLaunch);
};
template <typename S>
struct PassSet {
  using T = typename CX<S>::T;
  int threads, threads_x;  // z and y passes, x pass
  int tz, ty, tk;     // real z-lines, y-lines and ky-lines (per component) per block
  void (*z_r2c)(const S*, T*, LinePlan, FastDiv, const T*, int, int, int, const IterCtrl*);
  void (*z_c2r)(const T*, S*, LinePlan, FastDiv, const T*, int, int, int, S, const IterCtrl*);
  void (*y_fwd)(const T*, T*, LinePlan, FastDiv, const T*, int, int, const IterCtrl*);
  void (*y_inv)(const T*, T*, LinePlan, FastDiv, const T*, int, int, const IterCtrl*);
  void (*x_fwd)(T*, LinePlan, FastDiv, const T*, GreenParams<S>, const S*, int, int, int,
                const IterCtrl*);
  void (*x_inv)(T*, LinePlan, FastDiv, const T*, GreenParams<S>, const S*, int, int, int,
                const IterCtrl*);
  void (*x_table)(T*, LinePlan, FastDiv, const T*, GreenParams<S>, const S*, int, int, int,
                  const IterCtrl*);
  void (*x_green)(T*, LinePlan, FastDiv, const T*, GreenParams<S>, const S*, int, int, int,
                  const IterCtrl*);
  int nfam;                // batched tile families; the last is the long tile
  BatchPasses<S> fam[3];
};

// Dynamic shared memory limit = the opt-in maximum minus the kernel's static part.
template <typename K>
inline void optin_rest(K kern, int total) {
  cudaFuncAttributes a{};
  if (cudaFuncGetAttributes(&a, (const void*)kern) != cudaSuccess) return;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       total - (int)a.sharedSizeBytes);
}

template <typename S, class E, int kEl>
BatchPasses<S> make_batch_passes(int smem) {
  using TL = Tiles<S, E, kEl>;
  static_assert(TL::kThreads == Tiles<S, E>::kThreads &&
                    TL::kThreadsX == Tiles<S, E>::kThreadsX,
                "batched and single kernels share the thread counts");
  BatchPasses<S> q;
  q.tz = TL::kZ;
  q.ty = TL::kY;
  q.tk = TL::kX;
  q.z_r2c = k_pass_z_r2c_batch<S, E, kEl>;
  q.z_c2r = k_pass_z_c2r_batch<S, E, kEl>;
  q.y_fwd = k_pass_y_batch<-1, S, E, kEl>;
  q.y_inv = k_pass_y_batch<1, S, E, kEl>;
  q.x_green = k_pass_x_batch<S, E, kEl>;
  // the batched kernels hold the slot's descriptor in static shared memory
  optin_rest(q.z_r2c, smem);
  optin_rest(q.z_c2r, smem);
  optin_rest(q.y_fwd, smem);
  optin_rest(q.y_inv, smem);
  optin_rest(q.x_green, smem);
  return q;
}

template <typename S, class E>
PassSet<S> make_pass_set() {
  using Ti = Tiles<S, E>;
  PassSet<S> p;
  p.threads = Ti::kThreads;
  p.threads_x = Ti::kThreadsX;
  p.tz = Ti::kZ;
  p.ty = Ti::kY;
  p.tk = Ti::kX;
  p.z_r2c = k_pass_z_r2c<S, E>;
  p.z_c2r = k_pass_z_c2r<S, E>;
  p.y_fwd = k_pass_y<-1, S, E>;
  p.y_inv = k_pass_y<1, S, E>;
  p.x_fwd = k_pass_x<0, S, E>;
  p.x_inv = k_pass_x<1, S, E>;
  p.x_green = k_pass_x<2, S, E>;
  p.x_table = k_pass_x<3, S, E>;
  const int s = 227 * 1024;
  optin_rest(p.z_r2c, s);
  optin_rest(p.z_c2r, s);
  optin_rest(p.y_fwd, s);
  optin_rest(p.y_inv, s);
  optin_rest(p.x_fwd, s);
  optin_rest(p.x_inv, s);
  optin_rest(p.x_green, s);
  optin_rest(p.x_table, s);
  constexpr int nf = batch_families<S, E>();
  p.nfam = nf;
  p.fam[0] = make_batch_passes<S, E, batch_family_elems<S, E>(0)>(s);
  if constexpr (nf > 1) p.fam[1] = make_batch_passes<S, E, batch_family_elems<S, E>(1)>(s);
  if constexpr (nf > 2) p.fam[2] = make_batch_passes<S, E, batch_family_elems<S, E>(2)>(s);
  return p;
}

// Entry tables of the fixed engines (fft_fixed_*.cu): nullptr for a length
// without one.
template <typename S>
const PassSet<S>* fixed_pass_set_small(int n);  // 16, 32, 48, 64, 96
template <typename S>
const PassSet<S>* fixed_pass_set_large(int n);  // 128, 192, 256, 384, 512

}  // namespace fft
}  // namespace vpfft
