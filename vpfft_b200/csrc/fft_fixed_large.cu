// fft_fixed_large.cu -- entry tables of the compile-time line engines for
// edges 128, 192, 256, 384 and 512 (a separate unit so the two halves of the
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
const PassSet<S>* large_set(int n) {
  switch (n) {
    case 128: return fixed_set<S, 128>();
    case 192: return fixed_set<S, 192>();
    case 256: return fixed_set<S, 256>();
    case 384: return fixed_set<S, 384>();
    case 512: return fixed_set<S, 512>();
    default: return nullptr;
  }
}
}  // namespace

template <>
const PassSet<float>* fixed_pass_set_large<float>(int n) {
  return large_set<float>(n);
}
template <>
const PassSet<double>* fixed_pass_set_large<double>(int n) {
  return large_set<double>(n);
}

}  // namespace fft
}  // namespace vpfft
