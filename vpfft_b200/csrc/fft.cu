// fft.cu -- the 3D real <-> half-complex transforms of the fixed-point loop,
// with the Green operator fused into the x pass.
//
// The transform is done as five line passes, each of which reads its lines in
// contiguous runs of at least 128 bytes and writes them in the layout the next
// pass reads contiguously (the transpose happens in the shared-memory tile):
//
//   W[c][x][y][z]   real field (P before the forward transform, d~ after)
//   A[c][x][kz][y]  after the z pass (kz in [0, nz/2])
//   B[c][kz][ky][x] after the y pass; the x pass works in place on B
//
//   pass_z_r2c   W -> A   pairs of real z-lines packed as one complex line
//   pass_y<-1>   A -> B
//   pass_x_green B -> B   forward x FFT, dhat = -Gbar(k) phat, inverse x FFT
//   pass_y<+1>   B -> A
//   pass_z_c2r   A -> W   Hermitian extension, pairs unpacked, times 1/N
//
// Inside a tile every line is transformed by a shared-memory Stockham FFT
// (radices 4, 2, 3, 5).  Line strides in shared memory are padded by one
// element so that the transposing reads and writes are (nearly) bank-conflict
// free.  No multicast or cluster features are used.
#include <cuda_runtime.h>

#include "kernel_common.cuh"
#include "kernels.h"

namespace vpfft {

namespace {

template <typename R>
struct CX;
template <>
struct CX<float> {
  using T = float2;
};
template <>
struct CX<double> {
  using T = double2;
};

template <typename T>
__device__ __forceinline__ T add(T a, T b) {
  return T{a.x + b.x, a.y + b.y};
}
template <typename T>
__device__ __forceinline__ T sub(T a, T b) {
  return T{a.x - b.x, a.y - b.y};
}
template <typename T, typename R>
__device__ __forceinline__ T scl(T a, R s) {
  return T{a.x * s, a.y * s};
}
template <int SIGN, typename T>
__device__ __forceinline__ T tw_mul(T v, T w) {
  if (SIGN < 0) return T{v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x};
  return T{v.x * w.x + v.y * w.y, v.y * w.x - v.x * w.y};
}
template <int SIGN, typename T>
__device__ __forceinline__ T mul_si(T z) {
  if (SIGN < 0) return T{z.y, -z.x};
  return T{-z.y, z.x};
}

// Shared-memory layout of a staged line: element i at sw(i) = i + i/16 (one
// pad slot per 16 elements), line stride line_stride(n) (odd, so lines are
// staggered across banks).  The pad spreads the stores of the early Stockham
// stages (span 1 and 4: stride-4 across threads) over all banks.
__host__ __device__ __forceinline__ int line_stride(int n) { return n + (n >> 4) + 1; }
__device__ __forceinline__ int sw(int i) { return i + (i >> 4); }

// In-register DFTs of size R (forward SIGN = -1: W = exp(-2 pi i / R)), input
// and output in natural order.
template <int SIGN, typename T>
__device__ __forceinline__ void dft4(T& a0, T& a1, T& a2, T& a3) {
  const T u0 = add(a0, a2), u1 = sub(a0, a2), u2 = add(a1, a3);
  const T u3 = mul_si<SIGN>(sub(a1, a3));
  a0 = add(u0, u2);
  a1 = add(u1, u3);
  a2 = sub(u0, u2);
  a3 = sub(u1, u3);
}

// exp(-i theta) = (cos theta, -sin theta), the convention of the twiddle
// tables: tw_mul<SIGN> conjugates it for the inverse transform.
template <int SIGN, typename T, typename R>
__device__ __forceinline__ T wconst(R c, R s) {
  return T{c, -s};
}

template <int RADIX, int SIGN, typename T>
__device__ __forceinline__ void dft(T (&v)[RADIX]) {
  using R = decltype(T{}.x);
  if constexpr (RADIX == 2) {
    const T t = v[0];
    v[0] = add(t, v[1]);
    v[1] = sub(t, v[1]);
  } else if constexpr (RADIX == 3) {
    const T t1 = add(v[1], v[2]);
    const T t2 = sub(v[0], scl(t1, R(0.5)));
    const T t3 = mul_si<SIGN>(scl(sub(v[1], v[2]), R(0.86602540378443864676)));
    v[0] = add(v[0], t1);
    v[1] = add(t2, t3);
    v[2] = sub(t2, t3);
  } else if constexpr (RADIX == 4) {
    dft4<SIGN>(v[0], v[1], v[2], v[3]);
  } else if constexpr (RADIX == 5) {
    const R c1 = R(0.30901699437494742410), c2 = R(-0.80901699437494742410);
    const R s1 = R(0.95105651629515357212), s2 = R(0.58778525229247312917);
    const T a1 = add(v[1], v[4]), a2 = add(v[2], v[3]), b1 = sub(v[1], v[4]),
            b2 = sub(v[2], v[3]);
    const T p1 = add(v[0], add(scl(a1, c1), scl(a2, c2)));
    const T p2 = add(v[0], add(scl(a1, c2), scl(a2, c1)));
    const T q1 = mul_si<SIGN>(add(scl(b1, s1), scl(b2, s2)));
    const T q2 = mul_si<SIGN>(sub(scl(b1, s2), scl(b2, s1)));
    v[0] = add(v[0], add(a1, a2));
    v[1] = add(p1, q1);
    v[4] = sub(p1, q1);
    v[2] = add(p2, q2);
    v[3] = sub(p2, q2);
  } else if constexpr (RADIX == 16) {
    // 16 = 4 x 4: Y[n1][k1] = DFT4 over n2 of v[n1 + 4 n2], times W16^(n1 k1);
    // X[k1 + 4 k2] = DFT4 over n1 of Y[n1][k1]
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) dft4<SIGN>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
    // now v[n1 + 4 k1] = Y[n1][k1]
    const R c = R(0.92387953251128675613), s = R(0.38268343236508977173);
    const R h = R(0.70710678118654752440);
    v[5] = tw_mul<SIGN>(v[5], wconst<SIGN, T>(c, s));     // n1 1, k1 1: W^1
    v[9] = tw_mul<SIGN>(v[9], wconst<SIGN, T>(h, h));     // n1 1, k1 2: W^2
    v[13] = tw_mul<SIGN>(v[13], wconst<SIGN, T>(s, c));   // n1 1, k1 3: W^3
    v[6] = tw_mul<SIGN>(v[6], wconst<SIGN, T>(h, h));     // n1 2, k1 1: W^2
    v[10] = mul_si<SIGN>(v[10]);                          // n1 2, k1 2: W^4
    v[14] = tw_mul<SIGN>(v[14], wconst<SIGN, T>(-h, h));  // n1 2, k1 3: W^6
    v[7] = tw_mul<SIGN>(v[7], wconst<SIGN, T>(s, c));     // n1 3, k1 1: W^3
    v[11] = tw_mul<SIGN>(v[11], wconst<SIGN, T>(-h, h));  // n1 3, k1 2: W^6
    v[15] = tw_mul<SIGN>(v[15], wconst<SIGN, T>(-c, -s)); // n1 3, k1 3: W^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
      dft4<SIGN>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // now v[4 k1 + k2] = X[k1 + 4 k2]: transpose 4 x 4 into natural order
    T x[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) x[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = x[r];
  }
}

// One Stockham stage of radix R over nlines lines: butterfly j of a line
// reads in[j + r nb] (nb = n / R), multiplies by tw[r e] (e = (j mod Ns) n /
// (Ns R)), transforms in registers and writes out[(j - j mod Ns) R + j mod Ns + r Ns].
template <int RADIX, int SIGN, typename T>
__device__ __forceinline__ void stockham_stage(const T* a, T* b, const T* tw, int n, int Ns,
                                               int nlines, int ls, const FastDiv& dnb,
                                               const FastDiv& dns) {
  const int nb = n / RADIX;
  const int total = nb * nlines;
  const int tws = n / (Ns * RADIX);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = (int)fast_div((uint32_t)t, dnb);
    const int j = t - line * nb;
    const T* in = a + line * ls;
    T* out = b + line * ls;
    const int jm = j - (int)fast_div((uint32_t)j, dns) * Ns;
    const int e = jm * tws;
    const int od = (j - jm) * RADIX + jm;
    T v[RADIX];
#pragma unroll
    for (int r = 0; r < RADIX; ++r) v[r] = in[sw(j + r * nb)];
    if (e) {
#pragma unroll
      for (int r = 1; r < RADIX; ++r) v[r] = tw_mul<SIGN>(v[r], tw[r * e]);
    }
    dft<RADIX, SIGN>(v);
#pragma unroll
    for (int r = 0; r < RADIX; ++r) out[sw(od + r * Ns)] = v[r];
  }
}

// Stockham autosort FFT of nlines lines (line stride ls) of length pl.n in
// shared memory; a and b are ping-pong buffers, the result buffer is returned.
// B16: whether the plan may contain a radix-16 stage (kernels without it keep
// a smaller register footprint for lines that never use one).
template <int SIGN, bool B16, typename T>
__device__ T* line_fft(T* a, T* b, const T* tw, const LinePlan& pl, int nlines, int ls) {
  const int n = pl.n;
  int Ns = 1;
  for (int st = 0; st < pl.nrad; ++st) {
    const int Rr = pl.rad[st];
    const FastDiv dnb = pl.by_nb[st], dns = pl.by_ns[st];
    switch (Rr) {
      case 16:
        if constexpr (B16) stockham_stage<16, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns);
        break;
      case 4: stockham_stage<4, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns); break;
      case 2: stockham_stage<2, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns); break;
      case 3: stockham_stage<3, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns); break;
      default: stockham_stage<5, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns); break;
    }
    __syncthreads();
    T* tmp = a;
    a = b;
    b = tmp;
    Ns *= Rr;
  }
  return a;
}

template <typename T>
__device__ __forceinline__ void load_twiddles(T* tw, const T* twg, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
}

// Copy of nrows rows of len elements: warp w takes rows w, w + nwarps, ...;
// lanes stride 32 along the row with kU independent loads in flight per lane
// before the matching stores (global rows are contiguous: one coalesced
// request per 32 elements, and enough bytes in flight to cover DRAM latency).
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

// Copy of a tile whose contiguous global rows are only W (compile-time)
// elements long: element i is (row i / W, column i % W); kU loads in flight.
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

}  // namespace

// Tile sizes: lines per block chosen so that global rows are >= 128 bytes.
template <typename R>
struct FftTiles {
  static constexpr int kZ = 16;                        // real z-lines (y tile) per block
  static constexpr int kY = sizeof(R) == 4 ? 16 : 8;   // y-lines (x tile) per block
  static constexpr int kX = sizeof(R) == 4 ? 4 : 2;    // ky tile of the x pass (x 5 components)
};
constexpr int kFftThreads = 256;

// ---------------------------------------------------------------- z, forward
template <typename S, bool B16>
__device__ __forceinline__ void pass_z_r2c_body(const S* __restrict__ W,
                                                typename CX<S>::T* __restrict__ A,
                                                const LinePlan& pl,
                                                const typename CX<S>::T* __restrict__ twg, int nx,
                                                int ny, int nh, int bx, int by, int bz) {
  using T = typename CX<S>::T;
  constexpr int TY = FftTiles<S>::kZ;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nz = pl.n, ls = line_stride(nz);
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + nz;
  T* b = a + (TY / 2) * ls;
  load_twiddles(tw, twg, nz);
  const int y0 = bx * TY, x = by, c = bz;
  const int ty = min(TY, ny - y0);
  const int npair = (ty + 1) / 2;
  const S* src = W + ((long long)(c * nx + x) * ny + y0) * nz;
  copy_rows<S>(
      2 * npair, nz,
      [&](int l, int z) { return l < ty ? src[l * nz + z] : S(0); },
      [&](int l, int z, S v) { reinterpret_cast<S*>(&a[(l >> 1) * ls + sw(z)])[l & 1] = v; });
  __syncthreads();
  const T* r = line_fft<-1, B16>(a, b, tw, pl, npair, ls);
  T* dst = A + ((long long)(c * nx + x) * nh) * ny + y0;
  copy_short_rows<TY, T>(
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
        if (l < ty) dst[k * ny + l] = v;
      });
}

// ---------------------------------------------------------------- z, inverse
template <typename S, bool B16>
__device__ __forceinline__ void pass_z_c2r_body(const typename CX<S>::T* __restrict__ A,
                                                S* __restrict__ W, const LinePlan& pl,
                                                const typename CX<S>::T* __restrict__ twg, int nx,
                                                int ny, int nh, S scale, int bx, int by, int bz) {
  using T = typename CX<S>::T;
  constexpr int TY = FftTiles<S>::kZ;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nz = pl.n, ls = line_stride(nz);
  // a: (TY/2) packed lines; b: the tile's half spectra first (TY x (nh+1)),
  // then the FFT's ping-pong buffer -- sized max of the two (see pass_smem)
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + nz;
  T* b = a + (TY / 2) * ls;
  load_twiddles(tw, twg, nz);
  const int y0 = bx * TY, x = by, c = bz;
  const int ty = min(TY, ny - y0);
  const int npair = (ty + 1) / 2;
  // half spectra of the tile into b: h[l][k]
  const T* src = A + ((long long)(c * nx + x) * nh) * ny + y0;
  const int hs = nh + 1;
  copy_short_rows<TY, T>(
      nh, [&](int k, int l) { return l < ty ? src[k * ny + l] : T{S(0), S(0)}; },
      [&](int k, int l, T v) { b[l * hs + k] = v; });
  __syncthreads();
  // packed full lines: Z = A_even + i A_odd, Hermitian extension for k >= nh
  for (int i = threadIdx.x; i < npair * nz; i += blockDim.x) {
    const int p = (int)fast_div((uint32_t)i, pl.by_n), k = i - p * nz;
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
  const T* r = line_fft<1, B16>(a, b, tw, pl, npair, ls);
  S* dst = W + ((long long)(c * nx + x) * ny + y0) * nz;
  copy_rows<S>(
      ty, nz,
      [&](int l, int z) {
        const T Z = r[(l >> 1) * ls + sw(z)];
        return ((l & 1) ? Z.y : Z.x) * scale;
      },
      [&](int l, int z, S v) { dst[l * nz + z] = v; });
}

// ---------------------------------------------------------------- y passes
// Forward: A[c][x][kz][y] -> B[c][kz][ky][x]; inverse: B -> A.
template <int SIGN, bool B16, typename R>
__device__ __forceinline__ void pass_y_body(const typename CX<R>::T* __restrict__ in,
                                            typename CX<R>::T* __restrict__ out,
                                            const LinePlan& pl,
                                            const typename CX<R>::T* __restrict__ twg, int nx,
                                            int nh, int bx, int by, int bz) {
  using T = typename CX<R>::T;
  constexpr int TX = FftTiles<R>::kY;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ny = pl.n, ls = line_stride(ny);
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + ny;
  T* b = a + TX * ls;
  load_twiddles(tw, twg, ny);
  const int x0 = bx * TX, kz = by, c = bz;
  const int tx = min(TX, nx - x0);
  // A line (c, x, kz) starts at ((c*nx + x)*nh + kz)*ny; B row (c, kz, ky) at ((c*nh + kz)*ny + ky)*nx
  // (offsets below are < 2^31 for dimensions <= 512: 32-bit index arithmetic)
  const long long a_base = ((long long)(c * nx + x0) * nh + kz) * ny;
  const int a_xs = nh * ny;
  const long long b_base = ((long long)(c * nh + kz) * ny) * nx + x0;
  const T* in_a = in + a_base;
  const T* in_b = in + b_base;
  T* out_a = out + a_base;
  T* out_b = out + b_base;
  if (SIGN < 0) {
    copy_rows<T>(
        TX, ny, [&](int xl, int y) { return xl < tx ? in_a[xl * a_xs + y] : T{R(0), R(0)}; },
        [&](int xl, int y, T v) { a[xl * ls + sw(y)] = v; });
  } else {
    copy_short_rows<TX, T>(
        ny, [&](int y, int xl) { return xl < tx ? in_b[y * nx + xl] : T{R(0), R(0)}; },
        [&](int y, int xl, T v) { a[xl * ls + sw(y)] = v; });
  }
  __syncthreads();
  const T* r = line_fft<SIGN, B16>(a, b, tw, pl, TX, ls);
  if (SIGN < 0) {
    copy_short_rows<TX, T>(
        ny, [&](int y, int xl) { return r[xl * ls + sw(y)]; },
        [&](int y, int xl, T v) {
          if (xl < tx) out_b[y * nx + xl] = v;
        });
  } else {
    copy_rows<T>(
        tx, ny, [&](int xl, int y) { return r[xl * ls + sw(y)]; },
        [&](int xl, int y, T v) { out_a[xl * a_xs + y] = v; });
  }
}

// ---------------------------------------------------------------- x pass
// In place on B[c][kz][ky][x]: MODE 0 forward, 1 inverse, 2 forward + Green + inverse.
template <int MODE, bool B16, typename R>
__device__ __forceinline__ void pass_x_body(typename CX<R>::T* __restrict__ B, const LinePlan& pl,
                                            const typename CX<R>::T* __restrict__ twg,
                                            const GreenParams<R>& gp, int ny, int nh, int ncomp,
                                            int bx, int by) {
  using T = typename CX<R>::T;
  constexpr int TK = FftTiles<R>::kX;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nx = pl.n, ls = line_stride(nx);
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + nx;
  T* b = a + ncomp * TK * ls;
  load_twiddles(tw, twg, nx);
  const int ky0 = bx * TK, kz = by;
  const int tk = min(TK, ny - ky0);
  // component stride and the block's offset: < 2^31 for dimensions <= 512
  const int cs = nh * ny * nx;
  T* Bb = B + ((long long)kz * ny + ky0) * nx;
  const int nl = ncomp * TK;
  copy_rows<T>(
      nl, nx,
      [&](int L, int xx) {
        const int c = L / TK, kl = L - c * TK;
        return kl < tk ? Bb[c * cs + kl * nx + xx] : T{R(0), R(0)};
      },
      [&](int L, int xx, T v) { a[L * ls + sw(xx)] = v; });
  __syncthreads();
  T* r = a;
  T* o = b;
  if (MODE != 1) {
    r = line_fft<-1, B16>(a, b, tw, pl, nl, ls);
    o = (r == a) ? b : a;
  }
  if (MODE == 2) {
    for (int i = threadIdx.x; i < TK * nx; i += blockDim.x) {
      const int kl = (int)fast_div((uint32_t)i, pl.by_n), xx = i - kl * nx;
      if (kl >= tk) continue;
      R pre[5], pim[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const T z = r[(c * TK + kl) * ls + sw(xx)];
        pre[c] = z.x;
        pim[c] = z.y;
      }
      green_apply<R>(gp, xx, ky0 + kl, kz, pre, pim);
#pragma unroll
      for (int c = 0; c < 5; ++c) r[(c * TK + kl) * ls + sw(xx)] = T{pre[c], pim[c]};
    }
    __syncthreads();
  }
  if (MODE != 0) r = line_fft<1, B16>(r, o, tw, pl, nl, ls);
  copy_rows<T>(
      nl, nx, [&](int L, int xx) { return r[L * ls + sw(xx)]; },
      [&](int L, int xx, T v) {
        const int c = L / TK, kl = L - c * TK;
        if (kl < tk) Bb[c * cs + kl * nx + xx] = v;
      });
}

// ---------------------------------------------------------------- kernels
template <typename S, bool B16>
__global__ void __launch_bounds__(kFftThreads)
    k_pass_z_r2c(const S* __restrict__ W, typename CX<S>::T* __restrict__ A, LinePlan pl,
                 const typename CX<S>::T* __restrict__ twg, int nx, int ny, int nh,
                 const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_z_r2c_body<S, B16>(W, A, pl, twg, nx, ny, nh, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <typename S, bool B16>
__global__ void __launch_bounds__(kFftThreads)
    k_pass_z_c2r(const typename CX<S>::T* __restrict__ A, S* __restrict__ W, LinePlan pl,
                 const typename CX<S>::T* __restrict__ twg, int nx, int ny, int nh, S scale,
                 const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_z_c2r_body<S, B16>(A, W, pl, twg, nx, ny, nh, scale, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int SIGN, bool B16, typename R>
__global__ void __launch_bounds__(kFftThreads)
    k_pass_y(const typename CX<R>::T* __restrict__ in, typename CX<R>::T* __restrict__ out,
             LinePlan pl, const typename CX<R>::T* __restrict__ twg, int nx, int nh,
             const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_y_body<SIGN, B16, R>(in, out, pl, twg, nx, nh, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int MODE, bool B16, typename R>
__global__ void __launch_bounds__(kFftThreads, 2)
    k_pass_x(typename CX<R>::T* __restrict__ B, LinePlan pl,
             const typename CX<R>::T* __restrict__ twg, GreenParams<R> gp, int ny, int nh,
             int ncomp, const IterCtrl* ctrl) {
  if (ctrl && ctrl->done) return;
  pass_x_body<MODE, B16, R>(B, pl, twg, gp, ny, nh, ncomp, blockIdx.x, blockIdx.y);
}

// Batched passes of the fixed-point iteration (5 components): block -> slot,
// then the slot's tile from the local block index.
template <typename S>
struct SlotSpectral {
  Spectral<S> sp;
  GreenParams<S> gp;
};
template <typename S>
__device__ __forceinline__ const SlotDesc<S>* batch_pass_setup(const SlotDesc<S>* desc,
                                                               const BatchLaunch& bl, bool green,
                                                               SlotSpectral<S>* sm, int* lb) {
  const SlotDesc<S>* d = &desc[batch_slot(bl, blockIdx.x, lb)];
  if (d->ctrl->done) return nullptr;
  copy_struct(&sm->sp, &d->sp);
  if (green) copy_struct(&sm->gp, &d->gp);
  __syncthreads();
  return d;
}

template <typename S, bool B16>
__global__ void __launch_bounds__(kFftThreads)
    k_pass_z_r2c_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  __shared__ SlotSpectral<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, false, &sm, &lb);
  if (!d) return;
  const Spectral<S>& sp = sm.sp;
  const int gx = (sp.ny + FftTiles<S>::kZ - 1) / FftTiles<S>::kZ;
  const int t = lb / gx;
  pass_z_r2c_body<S, B16>(d->f.work, reinterpret_cast<typename CX<S>::T*>(sp.X), sp.pz,
                     reinterpret_cast<const typename CX<S>::T*>(sp.twz), sp.nx, sp.ny, sp.nh,
                     lb - t * gx, t % sp.nx, t / sp.nx);
}
template <typename S, bool B16>
__global__ void __launch_bounds__(kFftThreads)
    k_pass_z_c2r_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  __shared__ SlotSpectral<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, false, &sm, &lb);
  if (!d) return;
  const Spectral<S>& sp = sm.sp;
  const int gx = (sp.ny + FftTiles<S>::kZ - 1) / FftTiles<S>::kZ;
  const int t = lb / gx;
  const S scale = S(1.0 / ((double)sp.nx * sp.ny * sp.nz));
  pass_z_c2r_body<S, B16>(reinterpret_cast<const typename CX<S>::T*>(sp.X), d->f.work, sp.pz,
                     reinterpret_cast<const typename CX<S>::T*>(sp.twz), sp.nx, sp.ny, sp.nh,
                     scale, lb - t * gx, t % sp.nx, t / sp.nx);
}
template <int SIGN, bool B16, typename S>
__global__ void __launch_bounds__(kFftThreads)
    k_pass_y_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  using T = typename CX<S>::T;
  __shared__ SlotSpectral<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, false, &sm, &lb);
  if (!d) return;
  const Spectral<S>& sp = sm.sp;
  const int gx = (sp.nx + FftTiles<S>::kY - 1) / FftTiles<S>::kY;
  const int t = lb / gx;
  const T* in = reinterpret_cast<const T*>(SIGN < 0 ? sp.X : sp.X2);
  T* out = reinterpret_cast<T*>(SIGN < 0 ? sp.X2 : sp.X);
  pass_y_body<SIGN, B16, S>(in, out, sp.py, reinterpret_cast<const T*>(sp.twy), sp.nx, sp.nh,
                       lb - t * gx, t % sp.nh, t / sp.nh);
}
template <typename S, bool B16>
__global__ void __launch_bounds__(kFftThreads, 2)
    k_pass_x_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  using T = typename CX<S>::T;
  __shared__ SlotSpectral<S> sm;
  int lb;
  const SlotDesc<S>* d = batch_pass_setup(desc, bl, true, &sm, &lb);
  if (!d) return;
  const Spectral<S>& sp = sm.sp;
  const int gx = (sp.ny + FftTiles<S>::kX - 1) / FftTiles<S>::kX;
  pass_x_body<2, B16, S>(reinterpret_cast<T*>(sp.X2), sp.px, reinterpret_cast<const T*>(sp.twx),
                    sm.gp, sp.ny, sp.nh, 5, lb % gx, lb / gx);
}

// ---------------------------------------------------------------- launchers
namespace {
template <typename R>
struct PassSmem {
  size_t z_r2c, z_c2r, y, x;
};
template <typename R>
PassSmem<R> pass_smem(const Spectral<R>& sp, int ncomp) {
  using T = typename CX<R>::T;
  PassSmem<R> s;
  const int TY = FftTiles<R>::kZ, TX = FftTiles<R>::kY, TK = FftTiles<R>::kX;
  const int lz = line_stride(sp.nz);
  s.z_r2c = sizeof(T) * (sp.nz + 2 * (size_t)(TY / 2) * lz);
  const size_t bsz = std::max((size_t)(TY / 2) * lz, (size_t)TY * (sp.nh + 1));
  s.z_c2r = sizeof(T) * (sp.nz + (size_t)(TY / 2) * lz + bsz);
  s.y = sizeof(T) * (sp.ny + 2 * (size_t)TX * line_stride(sp.ny));
  s.x = sizeof(T) * (sp.nx + 2 * (size_t)ncomp * TK * line_stride(sp.nx));
  return s;
}
// Dynamic shared memory limit = the opt-in maximum minus the kernel's static part.
template <typename K>
void optin_rest(K kern, int total) {
  cudaFuncAttributes a{};
  if (cudaFuncGetAttributes(&a, kern) != cudaSuccess) return;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       total - (int)a.sharedSizeBytes);
}
template <typename R, bool B16>
void pass_optin_variant(int s) {
  cudaFuncSetAttribute(k_pass_z_r2c<R, B16>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_pass_z_c2r<R, B16>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_pass_y<-1, B16, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_pass_y<1, B16, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_pass_x<0, B16, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_pass_x<1, B16, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_pass_x<2, B16, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  // the batched kernels hold the slot's descriptor in static shared memory
  optin_rest(k_pass_z_r2c_batch<R, B16>, s);
  optin_rest(k_pass_z_c2r_batch<R, B16>, s);
  optin_rest(k_pass_y_batch<-1, B16, R>, s);
  optin_rest(k_pass_y_batch<1, B16, R>, s);
  optin_rest(k_pass_x_batch<R, B16>, s);
}
template <typename R>
void pass_optin() {
  static bool done = false;  // attributes are per function and device-independent here
  if (done) return;
  const int s = 227 * 1024;
  pass_optin_variant<R, false>(s);
  pass_optin_variant<R, true>(s);
  done = true;
}
}  // namespace

static bool has16(const LinePlan& p) {
  for (int st = 0; st < p.nrad; ++st)
    if (p.rad[st] == 16) return true;
  return false;
}

template <typename S>
int launch_spectral_iteration(const Spectral<S>& sp, const GreenParams<S>& gp, S* work,
                              const IterCtrl* ctrl, cudaStream_t st, int ncomp,
                              cudaEvent_t* ev) {
  using T = typename CX<S>::T;
  pass_optin<S>();
  const PassSmem<S> sm = pass_smem(sp, ncomp);
  T* A = reinterpret_cast<T*>(sp.X);
  T* B = reinterpret_cast<T*>(sp.X2);
  const T* twx = reinterpret_cast<const T*>(sp.twx);
  const T* twy = reinterpret_cast<const T*>(sp.twy);
  const T* twz = reinterpret_cast<const T*>(sp.twz);
  const dim3 gz((sp.ny + FftTiles<S>::kZ - 1) / FftTiles<S>::kZ, sp.nx, ncomp);
  const dim3 gy((sp.nx + FftTiles<S>::kY - 1) / FftTiles<S>::kY, sp.nh, ncomp);
  const dim3 gx((sp.ny + FftTiles<S>::kX - 1) / FftTiles<S>::kX, sp.nh);
  if (ev) cudaEventRecord(ev[0], st);
  const bool bz = has16(sp.pz), by = has16(sp.py), bx = has16(sp.px);
  (bz ? k_pass_z_r2c<S, true> : k_pass_z_r2c<S, false>)<<<gz, kFftThreads, sm.z_r2c, st>>>(
      work, A, sp.pz, twz, sp.nx, sp.ny, sp.nh, ctrl);
  if (ev) cudaEventRecord(ev[1], st);
  (by ? k_pass_y<-1, true, S> : k_pass_y<-1, false, S>)<<<gy, kFftThreads, sm.y, st>>>(
      A, B, sp.py, twy, sp.nx, sp.nh, ctrl);
  if (ev) cudaEventRecord(ev[2], st);
  (bx ? k_pass_x<2, true, S> : k_pass_x<2, false, S>)<<<gx, kFftThreads, sm.x, st>>>(
      B, sp.px, twx, gp, sp.ny, sp.nh, ncomp, ctrl);
  if (ev) cudaEventRecord(ev[3], st);
  (by ? k_pass_y<1, true, S> : k_pass_y<1, false, S>)<<<gy, kFftThreads, sm.y, st>>>(
      B, A, sp.py, twy, sp.nx, sp.nh, ctrl);
  if (ev) cudaEventRecord(ev[4], st);
  const S scale = S(1.0 / ((double)sp.nx * sp.ny * sp.nz));
  (bz ? k_pass_z_c2r<S, true> : k_pass_z_c2r<S, false>)<<<gz, kFftThreads, sm.z_c2r, st>>>(
      A, work, sp.pz, twz, sp.nx, sp.ny, sp.nh, scale, ctrl);
  if (ev) cudaEventRecord(ev[5], st);
  return 5;
}

template <typename S>
int launch_fft3d(const Spectral<S>& sp, S* real, int ncomp, int mode, cudaStream_t st) {
  using T = typename CX<S>::T;
  pass_optin<S>();
  const PassSmem<S> sm = pass_smem(sp, ncomp);
  T* A = reinterpret_cast<T*>(sp.X);
  T* B = reinterpret_cast<T*>(sp.X2);
  const T* twx = reinterpret_cast<const T*>(sp.twx);
  const T* twy = reinterpret_cast<const T*>(sp.twy);
  const T* twz = reinterpret_cast<const T*>(sp.twz);
  const dim3 gz((sp.ny + FftTiles<S>::kZ - 1) / FftTiles<S>::kZ, sp.nx, ncomp);
  const dim3 gy((sp.nx + FftTiles<S>::kY - 1) / FftTiles<S>::kY, sp.nh, ncomp);
  const dim3 gx((sp.ny + FftTiles<S>::kX - 1) / FftTiles<S>::kX, sp.nh);
  GreenParams<S> gp{};
  if (mode == 0) {
    const bool bz = has16(sp.pz), by = has16(sp.py), bx = has16(sp.px);
    (bz ? k_pass_z_r2c<S, true> : k_pass_z_r2c<S, false>)<<<gz, kFftThreads, sm.z_r2c, st>>>(
        real, A, sp.pz, twz, sp.nx, sp.ny, sp.nh,
                                                       nullptr);
    (by ? k_pass_y<-1, true, S> : k_pass_y<-1, false, S>)<<<gy, kFftThreads, sm.y, st>>>(
        A, B, sp.py, twy, sp.nx, sp.nh, nullptr);
    (bx ? k_pass_x<0, true, S> : k_pass_x<0, false, S>)<<<gx, kFftThreads, sm.x, st>>>(
        B, sp.px, twx, gp, sp.ny, sp.nh, ncomp, nullptr);
  } else {
    const bool bz = has16(sp.pz), by = has16(sp.py), bx = has16(sp.px);
    (bx ? k_pass_x<1, true, S> : k_pass_x<1, false, S>)<<<gx, kFftThreads, sm.x, st>>>(
        B, sp.px, twx, gp, sp.ny, sp.nh, ncomp, nullptr);
    (by ? k_pass_y<1, true, S> : k_pass_y<1, false, S>)<<<gy, kFftThreads, sm.y, st>>>(
        B, A, sp.py, twy, sp.nx, sp.nh, nullptr);
    const S scale = S(1.0 / ((double)sp.nx * sp.ny * sp.nz));
    (bz ? k_pass_z_c2r<S, true> : k_pass_z_c2r<S, false>)<<<gz, kFftThreads, sm.z_c2r, st>>>(
        A, real, sp.pz, twz, sp.nx, sp.ny, sp.nh,
                                                       scale, nullptr);
  }
  return 3;
}

template <typename S>
SpectralShape spectral_shape(const Spectral<S>& sp, int ncomp) {
  const PassSmem<S> sm = pass_smem(sp, ncomp);
  SpectralShape r;
  r.blocks_z = ((sp.ny + FftTiles<S>::kZ - 1) / FftTiles<S>::kZ) * sp.nx * ncomp;
  r.blocks_y = ((sp.nx + FftTiles<S>::kY - 1) / FftTiles<S>::kY) * sp.nh * ncomp;
  r.blocks_x = ((sp.ny + FftTiles<S>::kX - 1) / FftTiles<S>::kX) * sp.nh;
  r.smem_z_r2c = sm.z_r2c;
  r.smem_z_c2r = sm.z_c2r;
  r.smem_y = sm.y;
  r.smem_x = sm.x;
  r.r16_z = has16(sp.pz);
  r.r16_y = has16(sp.py);
  r.r16_x = has16(sp.px);
  return r;
}

template <typename S>
int launch_spectral_batch(const SlotDesc<S>* d, const BatchLaunch& bl_z, const BatchLaunch& bl_y,
                          const BatchLaunch& bl_x, const SpectralShape& sm, cudaStream_t st) {
  if (bl_z.blocks <= 0) return 0;
  pass_optin<S>();
  const bool bz = sm.r16_z, by = sm.r16_y, bx = sm.r16_x;
  (bz ? k_pass_z_r2c_batch<S, true> : k_pass_z_r2c_batch<S, false>)<<<bl_z.blocks, kFftThreads,
                                                                     sm.smem_z_r2c, st>>>(d, bl_z);
  (by ? k_pass_y_batch<-1, true, S> : k_pass_y_batch<-1, false, S>)<<<bl_y.blocks, kFftThreads,
                                                                       sm.smem_y, st>>>(d, bl_y);
  (bx ? k_pass_x_batch<S, true> : k_pass_x_batch<S, false>)<<<bl_x.blocks, kFftThreads,
                                                              sm.smem_x, st>>>(d, bl_x);
  (by ? k_pass_y_batch<1, true, S> : k_pass_y_batch<1, false, S>)<<<bl_y.blocks, kFftThreads,
                                                                     sm.smem_y, st>>>(d, bl_y);
  (bz ? k_pass_z_c2r_batch<S, true> : k_pass_z_c2r_batch<S, false>)<<<bl_z.blocks, kFftThreads,
                                                                     sm.smem_z_c2r, st>>>(d, bl_z);
  return 5;
}

template SpectralShape spectral_shape<double>(const Spectral<double>&, int);
template SpectralShape spectral_shape<float>(const Spectral<float>&, int);
template int launch_spectral_batch<double>(const SlotDesc<double>*, const BatchLaunch&,
                                           const BatchLaunch&, const BatchLaunch&,
                                           const SpectralShape&, cudaStream_t);
template int launch_spectral_batch<float>(const SlotDesc<float>*, const BatchLaunch&,
                                          const BatchLaunch&, const BatchLaunch&,
                                          const SpectralShape&, cudaStream_t);
template int launch_spectral_iteration<double>(const Spectral<double>&, const GreenParams<double>&,
                                               double*, const IterCtrl*, cudaStream_t, int,
                                               cudaEvent_t*);
template int launch_spectral_iteration<float>(const Spectral<float>&, const GreenParams<float>&,
                                              float*, const IterCtrl*, cudaStream_t, int,
                                              cudaEvent_t*);
template int launch_fft3d<double>(const Spectral<double>&, double*, int, int, cudaStream_t);
template int launch_fft3d<float>(const Spectral<float>&, float*, int, int, cudaStream_t);

}  // namespace vpfft
