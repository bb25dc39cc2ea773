// fft_fixed_small.cu -- entry tables of the compile-time line engines for
// edges 16, 32, 48, 64 and 96 (a separate unit so the two halves of the
// fixed engines compile in parallel).
#include "fft_passes.cuh"

namespace vpfft {
namespace fft {

namespace {
template <typename S, int N>
const PassSet<S>* fixed_set() {
  static const PassSet<S> s = make_pass_set<S, FixedEngine<N>>();
  return &s;
}
template <typename S>
const PassSet<S>* small_set(int n) {
  switch (n) {
    case 16: return fixed_set<S, 16>();
    case 32: return fixed_set<S, 32>();
    case 48: return fixed_set<S, 48>();
    case 64: return fixed_set<S, 64>();
    case 96: return fixed_set<S, 96>();
    default: return nullptr;
  }
}
}  // namespace

template <>
const PassSet<float>* fixed_pass_set_small<float>(int n) {
  return small_set<float>(n);
}
template <>
const PassSet<double>* fixed_pass_set_small<double>(int n) {
  return small_set<double>(n);
}

}  // namespace fft
}  // namespace vpfft
