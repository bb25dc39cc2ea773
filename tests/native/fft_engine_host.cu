// Host check of the line FFT engines (vpfft_b200/csrc/fft_engine.cuh): each
// engine's block program runs sequentially (thread 0 of a 1-thread block) on
// padded lines and is compared with a direct DFT in long double.  Prints one
// line per case and exits non-zero on a failure.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../vpfft_b200/csrc/fft_engine.cuh"

using namespace vpfft;
using namespace vpfft::fft;

template <typename S>
std::vector<typename CX<S>::T> table(int n) {
  std::vector<typename CX<S>::T> t(n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < n; ++i) {
    const long double th = 2 * pi * i / n;
    t[i].x = (S)cosl(th);
    t[i].y = (S)(-sinl(th));
  }
  return t;
}

// max |X - X_ref| / max |X_ref| over nl lines
template <typename S, typename Run>
double check(int n, int nl, int sign, Run run) {
  using T = typename CX<S>::T;
  const int ls = line_stride(n);
  std::vector<T> a(nl * ls), b(nl * ls);
  std::vector<long double> xr(nl * n), xi(nl * n);
  std::mt19937_64 rng(1234 + n);
  std::uniform_real_distribution<double> u(-1, 1);
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) {
      T v{(S)u(rng), (S)u(rng)};
      a[l * ls + sw(i)] = v;
      xr[l * n + i] = v.x;
      xi[l * n + i] = v.y;
    }
  std::vector<T> tw = table<S>(n);
  T* r = run(a.data(), b.data(), tw.data(), nl, ls);
  const long double pi = 3.141592653589793238462643383279502884L;
  long double err = 0, mag = 0;
  for (int l = 0; l < nl; ++l)
    for (int k = 0; k < n; ++k) {
      long double sr = 0, si = 0;
      for (int j = 0; j < n; ++j) {
        const long double th = sign * 2 * pi * (long double)((long long)j * k % n) / n;
        sr += xr[l * n + j] * cosl(th) - xi[l * n + j] * sinl(th);
        si += xr[l * n + j] * sinl(th) + xi[l * n + j] * cosl(th);
      }
      const T g = r[l * ls + sw(k)];
      err = fmaxl(err, hypotl(g.x - sr, g.y - si));
      mag = fmaxl(mag, hypotl(sr, si));
    }
  return (double)(err / mag);
}

int failures = 0;

template <typename S, int N>
void fixed_case() {
  using T = typename CX<S>::T;
  for (int sign = -1; sign <= 1; sign += 2) {
    const double e = check<S>(N, 3, sign, [&](T* a, T* b, const T* tw, int nl, int ls) {
      std::vector<T> st(N);  // the per-stage tables built from the plain table
      FixedEngine<N>::load_tw(st.data(), tw, N, 0, 1);
      return sign < 0 ? FixedEngine<N>::template fft<-1>(a, b, st.data(), LinePlan{}, nl, ls, 0, 1)
                      : FixedEngine<N>::template fft<1>(a, b, st.data(), LinePlan{}, nl, ls, 0, 1);
    });
    const double tol = sizeof(S) == 4 ? 2e-6 : 1e-14;
    const bool ok = e < tol;
    failures += !ok;
    std::printf("fixed   %-6s n=%4d sign=%+d rel.err %.3e %s\n", sizeof(S) == 4 ? "float" : "double",
                N, sign, e, ok ? "ok" : "FAIL");
  }
}

template <typename S, bool B16>
void generic_case(int n, std::vector<int> rad) {
  using T = typename CX<S>::T;
  LinePlan p{};
  p.n = n;
  p.nrad = (int)rad.size();
  p.by_n = make_fast_div((uint32_t)n);
  int ns = 1;
  for (int st = 0; st < p.nrad; ++st) {
    p.rad[st] = rad[st];
    p.by_nb[st] = make_fast_div((uint32_t)(n / rad[st]));
    p.by_ns[st] = make_fast_div((uint32_t)ns);
    ns *= rad[st];
  }
  for (int sign = -1; sign <= 1; sign += 2) {
    const double e = check<S>(n, 3, sign, [&](T* a, T* b, const T* tw, int nl, int ls) {
      return sign < 0 ? GenericEngine<B16>::template fft<-1>(a, b, tw, p, nl, ls, 0, 1)
                      : GenericEngine<B16>::template fft<1>(a, b, tw, p, nl, ls, 0, 1);
    });
    const double tol = sizeof(S) == 4 ? 2e-6 : 1e-14;
    const bool ok = e < tol;
    failures += !ok;
    std::printf("generic %-6s n=%4d sign=%+d rel.err %.3e %s\n", sizeof(S) == 4 ? "float" : "double",
                n, sign, e, ok ? "ok" : "FAIL");
  }
}

template <typename S>
void all() {
  fixed_case<S, 16>();
  fixed_case<S, 32>();
  fixed_case<S, 48>();
  fixed_case<S, 64>();
  fixed_case<S, 96>();
  fixed_case<S, 128>();
  fixed_case<S, 192>();
  fixed_case<S, 256>();
  fixed_case<S, 384>();
  fixed_case<S, 512>();
  generic_case<S, false>(15, {3, 5});
  generic_case<S, false>(12, {4, 3});
  generic_case<S, false>(10, {2, 5});
  generic_case<S, true>(256, {4, 4, 16});
  generic_case<S, true>(512, {4, 4, 16, 2});
  generic_case<S, false>(96, {4, 4, 2, 3});
}

int main() {
  all<float>();
  all<double>();
  std::printf("%s\n", failures ? "FAILED" : "ALL OK");
  return failures ? 1 : 0;
}
