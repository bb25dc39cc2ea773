// fft_engine.cuh -- line FFT engines for lines staged in shared memory.
//
// A "line" is one 1D complex transform of length n held in shared memory with
// the padded layout sw(i) = i + i/16 (one pad slot per 16 elements) and line
// stride line_stride(n).  Two engines transform nlines such lines with a
// Stockham autosort FFT (ping-pong between buffers a and b, the result buffer
// is returned):
//
//   GenericEngine<B16>  any n = 2^a 3^b 5^c; the radix plan (4, 2, 3, 5, and
//                       one radix-16 stage when B16) is a runtime LinePlan.
//   FixedEngine<N>      the lengths of the common grid edges (16 ... 512); the
//                       plan is a compile-time list of radices led by a
//                       radix-16 stage, so every index, twiddle stride and
//                       padded offset is a compile-time constant and each
//                       thread holds a whole radix-16 butterfly in registers.
//
// Both engines start from the twiddle table exp(-2 pi i i / n) (i in [0, n)),
// which load_tw stages in shared memory (the fixed engine as per-stage tables
// read without bank conflicts), and give the unnormalised DFT with exponent
// sign SIGN.  Everything here is __host__ __device__ so that a host build can
// run a block's work sequentially (thread 0 of a 1-thread block) and check it
// against a direct DFT.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "kernels.h"

#define VPFFT_HD __host__ __device__ __forceinline__

namespace vpfft {
namespace fft {

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
VPFFT_HD T add(T a, T b) {
  return T{a.x + b.x, a.y + b.y};
}
template <typename T>
VPFFT_HD T sub(T a, T b) {
  return T{a.x - b.x, a.y - b.y};
}
// FP32 complex add and subtract as one paired instruction each on sm_100
// (a - b as fma(b, -1, a): one rounding, the same value as a - b).
template <>
VPFFT_HD float2 add(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __fadd2_rn(a, b);
#else
  return float2{a.x + b.x, a.y + b.y};
#endif
}
template <>
VPFFT_HD float2 sub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
  return float2{a.x - b.x, a.y - b.y};
#endif
}
template <typename T, typename R>
VPFFT_HD T scl(T a, R s) {
  return T{a.x * s, a.y * s};
}
// v * w for SIGN < 0, v * conj(w) for SIGN > 0 (w from the table: exp(-i theta))
// (products and sums spelled out with fmad, see device_math.cuh)
template <int SIGN, typename T>
VPFFT_HD T tw_mul(T v, T w) {
  if (SIGN < 0) return T{fmad(v.x, w.x, -(v.y * w.y)), fmad(v.x, w.y, v.y * w.x)};
  return T{fmad(v.x, w.x, v.y * w.y), fmad(v.y, w.x, -(v.x * w.y))};
}
// z * (SIGN i)
template <int SIGN, typename T>
VPFFT_HD T mul_si(T z) {
  if (SIGN < 0) return T{z.y, -z.x};
  return T{-z.y, z.x};
}

// Padded shared-memory line layout: element i at sw(i), lines line_stride(n)
// apart (odd, so consecutive lines start in different banks).
VPFFT_HD constexpr int line_stride(int n) { return n + (n >> 4) + 1; }
VPFFT_HD constexpr int sw(int i) { return i + (i >> 4); }

VPFFT_HD void block_sync() {
#ifdef __CUDA_ARCH__
  __syncthreads();
#endif
}

template <int I, int N, typename F>
VPFFT_HD void static_for(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

// cos(2 pi m / 48), m in [0, 12] (first quadrant; the rest by symmetry).
VPFFT_HD constexpr double cos48q(int m) {
  constexpr double c[13] = {1.0,
                            0.99144486137381041114,
                            0.96592582628906828675,
                            0.92387953251128675613,
                            0.86602540378443864676,
                            0.79335334029123516458,
                            0.70710678118654752440,
                            0.60876142900872063942,
                            0.5,
                            0.38268343236508977173,
                            0.25881904510252076235,
                            0.13052619222005159155,
                            0.0};
  return c[m];
}
// cos and sin of 2 pi m / 48 for any m in [0, 48)
VPFFT_HD constexpr double cos48(int m) {
  return m <= 12 ? cos48q(m) : m <= 24 ? -cos48q(24 - m) : m <= 36 ? -cos48q(m - 24) : cos48q(48 - m);
}
VPFFT_HD constexpr double sin48(int m) { return cos48((m + 36) % 48); }

// v * W_R^M with W_R = exp(SIGN 2 pi i / R), compile-time R (a divisor of 48)
// and M; quarter turns are exact.
template <int SIGN, int R, int M, typename T>
VPFFT_HD T twc(T v) {
  static_assert(48 % R == 0, "internal twiddles need R | 48");
  using F = decltype(T{}.x);
  constexpr int m = ((M % R) * (48 / R)) % 48;
  if constexpr (m == 0) {
    return v;
  } else if constexpr (m == 12) {
    return mul_si<SIGN>(v);
  } else if constexpr (m == 24) {
    return T{-v.x, -v.y};
  } else if constexpr (m == 36) {
    return mul_si<-SIGN>(v);
  } else {
    constexpr F c = F(cos48(m));
    constexpr F s = F(SIGN < 0 ? -sin48(m) : sin48(m));
    return T{fmad(v.x, c, -(v.y * s)), fmad(v.x, s, v.y * c)};
  }
}

// ------------------------------------------------------------- codelets
// In-register DFT of size R, natural order in and out:
// X[k] = sum_n x[n] exp(SIGN 2 pi i n k / R).
template <int R, int SIGN, typename T>
VPFFT_HD void dft(T (&v)[R]);

template <int SIGN, typename T>
VPFFT_HD void dft4(T& a0, T& a1, T& a2, T& a3) {
  const T u0 = add(a0, a2), u1 = sub(a0, a2), u2 = add(a1, a3);
  const T u3 = mul_si<SIGN>(sub(a1, a3));
  a0 = add(u0, u2);
  a1 = add(u1, u3);
  a2 = sub(u0, u2);
  a3 = sub(u1, u3);
}

// R = R1 R2 by one Cooley-Tukey split: n = n1 + R1 n2, k = k2 + R2 k1;
// DFT_R2 over n2 for each n1, internal twiddles W_R^(n1 k2), DFT_R1 over n1
// for each k2.
template <int R1, int R2, int SIGN, typename T>
VPFFT_HD void dft_split(T (&v)[R1 * R2]) {
  constexpr int R = R1 * R2;
  static_for<0, R1>([&](auto n1c) {
    constexpr int n1 = decltype(n1c)::value;
    T u[R2];
    static_for<0, R2>([&](auto n2c) { u[decltype(n2c)::value] = v[n1 + R1 * decltype(n2c)::value]; });
    dft<R2, SIGN>(u);
    static_for<0, R2>([&](auto k2c) {
      constexpr int k2 = decltype(k2c)::value;
      v[n1 + R1 * k2] = twc<SIGN, R, n1 * k2>(u[k2]);
    });
  });
  T out[R];
  static_for<0, R2>([&](auto k2c) {
    constexpr int k2 = decltype(k2c)::value;
    T u[R1];
    static_for<0, R1>([&](auto n1c) { u[decltype(n1c)::value] = v[decltype(n1c)::value + R1 * k2]; });
    dft<R1, SIGN>(u);
    static_for<0, R1>([&](auto k1c) { out[k2 + R2 * decltype(k1c)::value] = u[decltype(k1c)::value]; });
  });
  static_for<0, R>([&](auto ic) { v[decltype(ic)::value] = out[decltype(ic)::value]; });
}

template <int R, int SIGN, typename T>
VPFFT_HD void dft(T (&v)[R]) {
  using F = decltype(T{}.x);
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    const T t = v[0];
    v[0] = add(t, v[1]);
    v[1] = sub(t, v[1]);
  } else if constexpr (R == 3) {
    const T t1 = add(v[1], v[2]);
    const T t2 = sub(v[0], scl(t1, F(0.5)));
    const T t3 = mul_si<SIGN>(scl(sub(v[1], v[2]), F(0.86602540378443864676)));
    v[0] = add(v[0], t1);
    v[1] = add(t2, t3);
    v[2] = sub(t2, t3);
  } else if constexpr (R == 4) {
    dft4<SIGN>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 5) {
    const F c1 = F(0.30901699437494742410), c2 = F(-0.80901699437494742410);
    const F s1 = F(0.95105651629515357212), s2 = F(0.58778525229247312917);
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
  } else if constexpr (R == 6) {
    dft_split<3, 2, SIGN>(v);
  } else if constexpr (R == 8) {
    dft_split<4, 2, SIGN>(v);
  } else if constexpr (R == 12) {
    dft_split<4, 3, SIGN>(v);
  } else if constexpr (R == 16) {
    dft_split<4, 4, SIGN>(v);
  } else {
    static_assert(R == 16, "no codelet for this radix");
  }
}

// ------------------------------------------------------------- generic engine
// One Stockham stage of radix RADIX over nlines lines: butterfly j of a line
// reads in[j + r nb] (nb = n / RADIX), multiplies by tw[r e] (e = (j mod Ns)
// n / (Ns RADIX)), transforms in registers and writes
// out[(j - j mod Ns) RADIX + j mod Ns + r Ns].  Threads tid, tid + nthr, ...
template <int RADIX, int SIGN, typename T>
VPFFT_HD void stockham_stage(const T* a, T* b, const T* tw, int n, int Ns, int nlines, int ls,
                             const FastDiv& dnb, const FastDiv& dns, int tid, int nthr) {
  const int nb = n / RADIX;
  const int total = nb * nlines;
  const int tws = n / (Ns * RADIX);
  for (int t = tid; t < total; t += nthr) {
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

template <bool B16>
struct GenericEngine {
  static constexpr int kN = 0;
  VPFFT_HD static int n(const LinePlan& p) { return p.n; }
  // shared-memory twiddles: the table itself (n entries)
  template <typename T>
  VPFFT_HD static void load_tw(T* tw, const T* twg, int n, int tid, int nthr) {
    for (int i = tid; i < n; i += nthr) tw[i] = twg[i];
  }
  VPFFT_HD static int div_n(int i, const LinePlan& p) { return (int)fast_div((uint32_t)i, p.by_n); }
  // B16: whether the plan may contain a radix-16 stage (kernels without it
  // keep a smaller register footprint for lines that never use one).
  template <int SIGN, typename T>
  VPFFT_HD static T* fft(T* a, T* b, const T* tw, const LinePlan& pl, int nlines, int ls, int tid,
                         int nthr) {
    const int n = pl.n;
    int Ns = 1;
    for (int st = 0; st < pl.nrad; ++st) {
      const int Rr = pl.rad[st];
      const FastDiv dnb = pl.by_nb[st], dns = pl.by_ns[st];
      switch (Rr) {
        case 16:
          if constexpr (B16)
            stockham_stage<16, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns, tid, nthr);
          break;
        case 4: stockham_stage<4, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns, tid, nthr); break;
        case 2: stockham_stage<2, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns, tid, nthr); break;
        case 3: stockham_stage<3, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns, tid, nthr); break;
        default: stockham_stage<5, SIGN>(a, b, tw, n, Ns, nlines, ls, dnb, dns, tid, nthr); break;
      }
      block_sync();
      T* tmp = a;
      a = b;
      b = tmp;
      Ns *= Rr;
    }
    return a;
  }
};

// ------------------------------------------------------------- fixed engine
template <int... Rs>
struct Radices {};

// Compile-time plans: a radix-16 stage first (span 1: contiguous 16-element
// groups, conflict-free with the padded layout), then the remaining factor.
template <int N>
struct FixedPlan;
template <> struct FixedPlan<16> { using type = Radices<16>; };
template <> struct FixedPlan<32> { using type = Radices<16, 2>; };
template <> struct FixedPlan<48> { using type = Radices<16, 3>; };
template <> struct FixedPlan<64> { using type = Radices<16, 4>; };
template <> struct FixedPlan<96> { using type = Radices<16, 6>; };
template <> struct FixedPlan<128> { using type = Radices<16, 8>; };
template <> struct FixedPlan<192> { using type = Radices<16, 12>; };
template <> struct FixedPlan<256> { using type = Radices<16, 16>; };
template <> struct FixedPlan<384> { using type = Radices<16, 12, 2>; };
template <> struct FixedPlan<512> { using type = Radices<16, 16, 2>; };

// The same stage with every size a compile-time constant.  tws: the stage's
// own twiddles, tws[(r - 1) NS + j mod NS] = W_N^(r (j mod NS) N / (NS RADIX)),
// so that the threads of a warp (consecutive j) read consecutive entries.
template <int N, int RADIX, int NS, int SIGN, typename T>
VPFFT_HD void fixed_stage(const T* a, T* b, const T* tws, int nlines, int ls, int tid, int nthr) {
  constexpr int NB = N / RADIX;
  static_assert(N % (NS * RADIX) == 0, "plan does not divide N");
  const int total = NB * nlines;
  for (int t = tid; t < total; t += nthr) {
    const int line = t / NB;
    const int j = t - line * NB;
    const int jm = j % NS;
    const int od = (j - jm) * RADIX + jm;
    const T* in = a + line * ls;
    T* out = b + line * ls;
    T v[RADIX];
    static_for<0, RADIX>([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      v[r] = in[sw(j + r * NB)];
    });
    if constexpr (NS > 1) {
      static_for<1, RADIX>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        v[r] = tw_mul<SIGN>(v[r], tws[(r - 1) * NS + jm]);
      });
    }
    dft<RADIX, SIGN>(v);
    static_for<0, RADIX>([&](auto rc) {
      constexpr int r = decltype(rc)::value;
      out[sw(od + r * NS)] = v[r];
    });
  }
}

// Offset of the next stage's twiddles: stages with a span NS > 1 keep
// (R - 1) NS entries (at most N in all).
template <int NS, int R>
constexpr int stage_tw_size() {
  return NS > 1 ? (R - 1) * NS : 0;
}

template <int N, int SIGN, int NS, int OFF, typename T>
VPFFT_HD T* fixed_stages(T* a, T*, const T*, int, int, int, int, Radices<>) {
  return a;
}
template <int N, int SIGN, int NS, int OFF, typename T, int R, int... Rest>
VPFFT_HD T* fixed_stages(T* a, T* b, const T* tw, int nlines, int ls, int tid, int nthr,
                         Radices<R, Rest...>) {
  fixed_stage<N, R, NS, SIGN>(a, b, tw + OFF, nlines, ls, tid, nthr);
  block_sync();
  return fixed_stages<N, SIGN, NS * R, OFF + stage_tw_size<NS, R>()>(b, a, tw, nlines, ls, tid,
                                                                    nthr, Radices<Rest...>{});
}

// The stage twiddle tables from the table twg[i] = exp(-2 pi i i / N).
template <int N, int NS, int OFF, typename T>
VPFFT_HD void fixed_tw_build(T*, const T*, int, int, Radices<>) {}
template <int N, int NS, int OFF, typename T, int R, int... Rest>
VPFFT_HD void fixed_tw_build(T* tw, const T* twg, int tid, int nthr, Radices<R, Rest...>) {
  if constexpr (NS > 1) {
    constexpr int TWS = N / (NS * R);
    for (int i = tid; i < (R - 1) * NS; i += nthr) {
      const int r = i / NS + 1, jm = i - (r - 1) * NS;
      tw[OFF + i] = twg[r * jm * TWS];
    }
  }
  fixed_tw_build<N, NS * R, OFF + stage_tw_size<NS, R>()>(tw, twg, tid, nthr,
                                                          Radices<Rest...>{});
}

template <int N>
struct FixedEngine {
  static constexpr int kN = N;
  VPFFT_HD static constexpr int n(const LinePlan&) { return N; }
  VPFFT_HD static int div_n(int i, const LinePlan&) { return i / N; }
  // shared-memory twiddles: the per-stage tables (at most N entries)
  template <typename T>
  VPFFT_HD static void load_tw(T* tw, const T* twg, int, int tid, int nthr) {
    fixed_tw_build<N, 1, 0>(tw, twg, tid, nthr, typename FixedPlan<N>::type{});
  }
  template <int SIGN, typename T>
  VPFFT_HD static T* fft(T* a, T* b, const T* tw, const LinePlan&, int nlines, int ls, int tid,
                         int nthr) {
    return fixed_stages<N, SIGN, 1, 0>(a, b, tw, nlines, ls, tid, nthr,
                                       typename FixedPlan<N>::type{});
  }
  // The same transform of lines staged in any layout: the first stage reads
  // element i of line l as load(l, i) and writes padded lines to a, the rest
  // ping-pong a / b.  kLineFastest: consecutive threads take consecutive
  // lines of one butterfly index (for layouts where the lines are adjacent in
  // memory, e.g. the columns of a tile), else consecutive butterflies of one
  // line.  The arithmetic is the first stage's, so the result is the same bit
  // for bit as fft() on the same values.
  template <int SIGN, bool kLineFastest, typename T, class Load>
  VPFFT_HD static T* fft_loaded(Load load, T* a, T* b, const T* tw, int nlines, int ls, int tid,
                                int nthr) {
    return first_loaded<SIGN, kLineFastest>(load, a, b, tw, nlines, ls, tid, nthr,
                                            typename FixedPlan<N>::type{});
  }

 private:
  template <int SIGN, bool kLineFastest, typename T, class Load, int R, int... Rest>
  VPFFT_HD static T* first_loaded(Load load, T* a, T* b, const T* tw, int nlines, int ls,
                                  int tid, int nthr, Radices<R, Rest...>) {
    // first stage: span 1, no twiddles; butterfly j of line l reads elements
    // j + r N/R and writes j R + r
    constexpr int NB = N / R;
    for (int t = tid; t < NB * nlines; t += nthr) {
      const int line = kLineFastest ? t % nlines : t / NB;
      const int j = kLineFastest ? t / nlines : t - line * NB;
      T v[R];
      static_for<0, R>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        v[r] = load(line, j + r * NB);
      });
      dft<R, SIGN>(v);
      T* out = a + line * ls;
      static_for<0, R>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        out[sw(j * R + r)] = v[r];
      });
    }
    block_sync();
    return fixed_stages<N, SIGN, R, stage_tw_size<1, R>()>(a, b, tw, nlines, ls, tid, nthr,
                                                           Radices<Rest...>{});
  }
};

}  // namespace fft
}  // namespace vpfft
