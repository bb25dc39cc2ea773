// fft.cu -- launchers of the 3D real <-> half-complex transforms of the
// fixed-point loop (five line passes, the Green operator fused into the x
// pass; fft_passes.cuh), single grid and batched.
//
// Each axis picks its line engine by its length: a compile-time engine for the
// common edges (16, 32, 48, 64, 96, 128, 192, 256, 384, 512; fft_fixed_*.cu),
// otherwise the runtime-plan Stockham engine (radices 4, 2, 3, 5 and a
// radix-16 stage for long power-of-4 runs).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "fft_passes.cuh"

namespace vpfft {

using namespace fft;

namespace {

bool has16(const LinePlan& p) {
  for (int st = 0; st < p.nrad; ++st)
    if (p.rad[st] == 16) return true;
  return false;
}

template <typename S>
const PassSet<S>& generic_set(bool b16) {
  static const PassSet<S> g0 = make_pass_set<S, GenericEngine<false>>();
  static const PassSet<S> g1 = make_pass_set<S, GenericEngine<true>>();
  return b16 ? g1 : g0;
}

template <typename S>
const PassSet<S>& pass_set(const LinePlan& p) {
  if (const PassSet<S>* f = fixed_pass_set_small<S>(p.n)) return *f;
  if (const PassSet<S>* f = fixed_pass_set_large<S>(p.n)) return *f;
  return generic_set<S>(has16(p));
}

int cdiv(int a, int b) { return (a + b - 1) / b; }

// The TMA y passes where they apply (FP32; see fft_tma.cu).
bool y_fwd_tma(const Spectral<float>& sp, const IterCtrl* ctrl, cudaStream_t st, int ncomp) {
  return launch_y_fwd_tma(sp, ctrl, st, ncomp);
}
bool y_fwd_tma(const Spectral<double>&, const IterCtrl*, cudaStream_t, int) { return false; }
bool y_inv_tma(const Spectral<float>& sp, const IterCtrl* ctrl, cudaStream_t st, int ncomp) {
  return launch_y_inv_tma(sp, ctrl, st, ncomp);
}
bool y_inv_tma(const Spectral<double>&, const IterCtrl*, cudaStream_t, int) { return false; }
bool z_r2c_tma(const Spectral<float>& sp, const float* w, const IterCtrl* ctrl, cudaStream_t st,
               int ncomp) {
  return launch_z_r2c_tma(sp, w, ctrl, st, ncomp);
}
bool z_r2c_tma(const Spectral<double>&, const double*, const IterCtrl*, cudaStream_t, int) {
  return false;
}
bool z_c2r_tma(const Spectral<float>& sp, float* w, const IterCtrl* ctrl, cudaStream_t st,
               int ncomp) {
  return launch_z_c2r_tma(sp, w, ctrl, st, ncomp);
}
bool z_c2r_tma(const Spectral<double>&, double*, const IterCtrl*, cudaStream_t, int) {
  return false;
}

template <typename S>
struct PassSmem {
  size_t z_r2c, z_c2r, y, x;
};
// Dynamic shared memory of the passes for tiles tz (real z-lines), ty
// (y-lines) and tk (ky-lines per component).
template <typename S>
PassSmem<S> pass_smem(const Spectral<S>& sp, int tz, int ty, int tk, int ncomp) {
  using T = typename CX<S>::T;
  PassSmem<S> s;
  const size_t lz = line_stride(sp.nz);
  const size_t zl = (size_t)(tz / 2) * lz;  // packed z-lines of a tile
  s.z_r2c = sizeof(T) * (sp.nz + 2 * zl);
  s.z_c2r = sizeof(T) * (sp.nz + zl + std::max(zl, (size_t)tz * (sp.nh + 1)));
  s.y = sizeof(T) * (sp.ny + 2 * (size_t)ty * line_stride(sp.ny));
  s.x = sizeof(T) * (sp.nx + 2 * (size_t)ncomp * tk * line_stride(sp.nx));
  return s;
}

}  // namespace

template <typename S>
int launch_spectral_iteration(const Spectral<S>& sp, const GreenParams<S>& gp, S* work,
                              const IterCtrl* ctrl, cudaStream_t st, int ncomp,
                              cudaEvent_t* ev, const S* gtab) {
  using T = typename CX<S>::T;
  const PassSet<S>& Z = pass_set<S>(sp.pz);
  const PassSet<S>& Y = pass_set<S>(sp.py);
  const PassSet<S>& X = pass_set<S>(sp.px);
  const PassSmem<S> sm = pass_smem(sp, Z.tz, Y.ty, X.tk, ncomp);
  T* A = reinterpret_cast<T*>(sp.X);
  T* B = reinterpret_cast<T*>(sp.X2);
  const T* twx = reinterpret_cast<const T*>(sp.twx);
  const T* twy = reinterpret_cast<const T*>(sp.twy);
  const T* twz = reinterpret_cast<const T*>(sp.twz);
  const dim3 gz(cdiv(sp.nx * sp.ny, Z.tz), ncomp);
  const dim3 gy(cdiv(sp.nh * sp.nx, Y.ty), ncomp);
  const dim3 gx(cdiv(sp.nh * sp.ny, X.tk));
  const S scale = S(1.0 / ((double)sp.nx * sp.ny * sp.nz));
  if (ev) cudaEventRecord(ev[0], st);
  if (!z_r2c_tma(sp, work, ctrl, st, ncomp))
    Z.z_r2c<<<gz, Z.threads, sm.z_r2c, st>>>(work, A, sp.pz, sp.py.by_n, twz, sp.nx, sp.ny, sp.nh,
                                             ctrl);
  if (ev) cudaEventRecord(ev[1], st);
  if (!y_fwd_tma(sp, ctrl, st, ncomp))
    Y.y_fwd<<<gy, Y.threads, sm.y, st>>>(A, B, sp.py, sp.px.by_n, twy, sp.nx, sp.nh, ctrl);
  if (ev) cudaEventRecord(ev[2], st);
  (gtab ? X.x_table : X.x_green)<<<gx, X.threads_x, sm.x, st>>>(B, sp.px, sp.py.by_n, twx, gp,
                                                               gtab, sp.ny, sp.nh, ncomp, ctrl);
  if (ev) cudaEventRecord(ev[3], st);
  if (!y_inv_tma(sp, ctrl, st, ncomp))
    Y.y_inv<<<gy, Y.threads, sm.y, st>>>(B, A, sp.py, sp.px.by_n, twy, sp.nx, sp.nh, ctrl);
  if (ev) cudaEventRecord(ev[4], st);
  if (!z_c2r_tma(sp, work, ctrl, st, ncomp))
    Z.z_c2r<<<gz, Z.threads, sm.z_c2r, st>>>(A, work, sp.pz, sp.py.by_n, twz, sp.nx, sp.ny, sp.nh,
                                             scale, ctrl);
  if (ev) cudaEventRecord(ev[5], st);
  return 5;
}

// The stored Green operator: for every wave vector of the half spectrum the
// kGreenStored values of green_core (C = (V L0 V^T)^-1 row-major, then
// 1/(k.C k); zeros where the operator has no Gamma part), value j of
// (f = kz ny + ky, x) at tab[j M + f nx + x].  The x pass then finishes the
// operator with the arithmetic of the computed path, so both give the same bits.
template <typename S>
__global__ void k_green_table(const GreenParams<S> gp, S* __restrict__ tab, int nh) {
  const long long M = (long long)nh * gp.ny * gp.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % gp.nx);
    const long long f = i / gp.nx;
    const int ky = (int)(f % gp.ny), kz = (int)(f / gp.ny);
    GreenPoint<S> q;
    S C[3][3] = {}, ikak = S(0);
    if (green_geometry(gp, x, ky, kz, q) && q.wg != S(0)) green_core(gp, q, C, ikak);
#pragma unroll
    for (int j = 0; j < 9; ++j) tab[j * M + i] = C[j / 3][j % 3];
    tab[9 * M + i] = ikak;
  }
}

template <typename S>
int launch_green_table(const GreenParams<S>& gp, S* tab, int nh, cudaStream_t st) {
  const long long M = (long long)nh * gp.ny * gp.nx;
  const int blocks = (int)std::min<long long>((M + 255) / 256, 148LL * 16);
  k_green_table<S><<<blocks, 256, 0, st>>>(gp, tab, nh);
  return 1;
}

template <typename S>
int launch_x_pass(const Spectral<S>& sp, const GreenParams<S>& gp, const S* gtab, void* buf,
                  int ncomp, cudaStream_t st) {
  using T = typename CX<S>::T;
  const PassSet<S>& Z = pass_set<S>(sp.pz);
  const PassSet<S>& Y = pass_set<S>(sp.py);
  const PassSet<S>& X = pass_set<S>(sp.px);
  const PassSmem<S> sm = pass_smem(sp, Z.tz, Y.ty, X.tk, ncomp);
  const dim3 gx(cdiv(sp.nh * sp.ny, X.tk));
  (gtab ? X.x_table : X.x_green)<<<gx, X.threads_x, sm.x, st>>>(
      reinterpret_cast<T*>(buf), sp.px, sp.py.by_n, reinterpret_cast<const T*>(sp.twx), gp, gtab,
      sp.ny, sp.nh, ncomp, nullptr);
  return 1;
}

template <typename S>
int launch_fft3d(const Spectral<S>& sp, S* real, int ncomp, int mode, cudaStream_t st) {
  using T = typename CX<S>::T;
  const PassSet<S>& Z = pass_set<S>(sp.pz);
  const PassSet<S>& Y = pass_set<S>(sp.py);
  const PassSet<S>& X = pass_set<S>(sp.px);
  const PassSmem<S> sm = pass_smem(sp, Z.tz, Y.ty, X.tk, ncomp);
  T* A = reinterpret_cast<T*>(sp.X);
  T* B = reinterpret_cast<T*>(sp.X2);
  const T* twx = reinterpret_cast<const T*>(sp.twx);
  const T* twy = reinterpret_cast<const T*>(sp.twy);
  const T* twz = reinterpret_cast<const T*>(sp.twz);
  const dim3 gz(cdiv(sp.nx * sp.ny, Z.tz), ncomp);
  const dim3 gy(cdiv(sp.nh * sp.nx, Y.ty), ncomp);
  const dim3 gx(cdiv(sp.nh * sp.ny, X.tk));
  GreenParams<S> gp{};
  if (mode == 0) {
    if (!z_r2c_tma(sp, real, nullptr, st, ncomp))
      Z.z_r2c<<<gz, Z.threads, sm.z_r2c, st>>>(real, A, sp.pz, sp.py.by_n, twz, sp.nx, sp.ny,
                                               sp.nh, nullptr);
    if (!y_fwd_tma(sp, nullptr, st, ncomp))
      Y.y_fwd<<<gy, Y.threads, sm.y, st>>>(A, B, sp.py, sp.px.by_n, twy, sp.nx, sp.nh, nullptr);
    X.x_fwd<<<gx, X.threads_x, sm.x, st>>>(B, sp.px, sp.py.by_n, twx, gp, nullptr, sp.ny, sp.nh,
                                         ncomp,
                                         nullptr);
  } else {
    X.x_inv<<<gx, X.threads_x, sm.x, st>>>(B, sp.px, sp.py.by_n, twx, gp, nullptr, sp.ny, sp.nh,
                                         ncomp,
                                         nullptr);
    if (!y_inv_tma(sp, nullptr, st, ncomp))
      Y.y_inv<<<gy, Y.threads, sm.y, st>>>(B, A, sp.py, sp.px.by_n, twy, sp.nx, sp.nh, nullptr);
    const S scale = S(1.0 / ((double)sp.nx * sp.ny * sp.nz));
    if (!z_c2r_tma(sp, real, nullptr, st, ncomp))
      Z.z_c2r<<<gz, Z.threads, sm.z_c2r, st>>>(A, real, sp.pz, sp.py.by_n, twz, sp.nx, sp.ny,
                                               sp.nh, scale, nullptr);
  }
  return 3;
}

template <typename S>
SpectralShape spectral_shape(const Spectral<S>& sp, int ncomp, int fam) {
  const PassSet<S>& Z = pass_set<S>(sp.pz);
  const PassSet<S>& Y = pass_set<S>(sp.py);
  const PassSet<S>& X = pass_set<S>(sp.px);
  // each axis takes the requested family, or its longest tile
  auto pick = [fam](const PassSet<S>& P) { return (fam < 0 || fam >= P.nfam) ? P.nfam - 1 : fam; };
  SpectralShape r;
  r.fam_z = pick(Z);
  r.fam_y = pick(Y);
  r.fam_x = pick(X);
  const BatchPasses<S>& bz = Z.fam[r.fam_z];
  const BatchPasses<S>& by = Y.fam[r.fam_y];
  const BatchPasses<S>& bx = X.fam[r.fam_x];
  const PassSmem<S> sm = pass_smem(sp, bz.tz, by.ty, bx.tk, ncomp);
  r.blocks_z = cdiv(sp.nx * sp.ny, bz.tz) * ncomp;
  r.blocks_y = cdiv(sp.nh * sp.nx, by.ty) * ncomp;
  r.blocks_x = cdiv(sp.nh * sp.ny, bx.tk);
  r.smem_z_r2c = sm.z_r2c;
  r.smem_z_c2r = sm.z_c2r;
  r.smem_y = sm.y;
  r.smem_x = sm.x;
  r.set_z = &Z;
  r.set_y = &Y;
  r.set_x = &X;
  r.families = std::max(Z.nfam, std::max(Y.nfam, X.nfam));
  return r;
}

template <typename S>
int launch_spectral_chain(const SlotDesc<S>* d, const PassChain& c, cudaStream_t st) {
  if (c.z.blocks <= 0) return 0;
  const BatchPasses<S>& Z = static_cast<const PassSet<S>*>(c.set_z)->fam[c.fam_z];
  const BatchPasses<S>& Y = static_cast<const PassSet<S>*>(c.set_y)->fam[c.fam_y];
  const BatchPasses<S>& X = static_cast<const PassSet<S>*>(c.set_x)->fam[c.fam_x];
  const int tzy = static_cast<const PassSet<S>*>(c.set_z)->threads;
  const int tyy = static_cast<const PassSet<S>*>(c.set_y)->threads;
  const int txx = static_cast<const PassSet<S>*>(c.set_x)->threads_x;
  Z.z_r2c<<<c.z.blocks, tzy, c.smem_z_r2c, st>>>(d, c.z);
  Y.y_fwd<<<c.y.blocks, tyy, c.smem_y, st>>>(d, c.y);
  X.x_green<<<c.x.blocks, txx, c.smem_x, st>>>(d, c.x);
  Y.y_inv<<<c.y.blocks, tyy, c.smem_y, st>>>(d, c.y);
  Z.z_c2r<<<c.z.blocks, tzy, c.smem_z_c2r, st>>>(d, c.z);
  return 5;
}

template SpectralShape spectral_shape<double>(const Spectral<double>&, int, int);
template SpectralShape spectral_shape<float>(const Spectral<float>&, int, int);
template int launch_spectral_chain<double>(const SlotDesc<double>*, const PassChain&,
                                           cudaStream_t);
template int launch_spectral_chain<float>(const SlotDesc<float>*, const PassChain&, cudaStream_t);
template int launch_spectral_iteration<double>(const Spectral<double>&, const GreenParams<double>&,
                                               double*, const IterCtrl*, cudaStream_t, int,
                                               cudaEvent_t*, const double*);
template int launch_spectral_iteration<float>(const Spectral<float>&, const GreenParams<float>&,
                                              float*, const IterCtrl*, cudaStream_t, int,
                                              cudaEvent_t*, const float*);
template int launch_green_table<double>(const GreenParams<double>&, double*, int, cudaStream_t);
template int launch_green_table<float>(const GreenParams<float>&, float*, int, cudaStream_t);
template int launch_x_pass<double>(const Spectral<double>&, const GreenParams<double>&,
                                   const double*, void*, int, cudaStream_t);
template int launch_x_pass<float>(const Spectral<float>&, const GreenParams<float>&, const float*,
                                  void*, int, cudaStream_t);
template int launch_fft3d<double>(const Spectral<double>&, double*, int, int, cudaStream_t);
template int launch_fft3d<float>(const Spectral<float>&, float*, int, int, cudaStream_t);

}  // namespace vpfft
