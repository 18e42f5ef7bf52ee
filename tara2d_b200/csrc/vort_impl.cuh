// Right-hand side of the incompressible vorticity models (reference:
// src/derive2csh.f95:3-149, unscreened; src/derive2css.f95:6-136, screened)
// as three kernels:
//
//   k_col_inv        y-inverse of psi, i*ky*psi, W and i*ky*W, with
//                    psi = omega/(k^2 + lambda) (zero at k = 0) and W = omega
//                    (unscreened) or k^2 psi (screened); the kx multipliers
//                    are applied on the rows
//   k_row_vort       per grid row: four c2r along x (ux = c2r(i ky psi),
//                    uy = c2r(-i kx psi), d omega/dx = c2r(i kx W),
//                    d omega/dy = c2r(i ky W)), the products, and one r2c of
//                    ux d omega/dx + uy d omega/dy.  The reference's two r2c
//                    and their sum (src/derive2csh.f95:119-134) are merged by
//                    linearity; both terms share the same 2/3 mask.
//   k_col_fwd_vort   y-forward, dealiasing, then
//                    d omega/dt = -(alpha NL + nu k^2 W) and the stepper
//                    update (alpha = 1 in the unscreened model).
#pragma once
#include "models.h"

namespace tara {

template <class T> struct RowVortArgs {
  Tables<T> tb;
  const Cx<T>* H[4];  // y-inverse of psi, i ky psi, W, i ky W
  Cx<T>* X;           // x-transformed nonlinear term
  int rb;
};

// Phase 1: four c2r in four groups (each group's output array is its
// exchange buffer).  Phase 2: NL = ux d omega/dx + uy d omega/dy into array 0.
// Phase 3: one r2c, exchange buffer in array 1.
template <class T, int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(4 * (M / P))) k_row_vort(const RowVortArgs<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = 4, ARR = RF::SMEM_ELEMS;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* base = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * G * ARR;
  auto arr = [&](int q) { return base + q * ARR; };
  const int y = blockIdx.x * a.rb + th.row;
  const size_t ro = (size_t)y * tb.ld;
  const Cx<T>* Hpsi = a.H[0] + ro;
  const Cx<T>* Hpsiy = a.H[1] + ro;
  const Cx<T>* Hw = a.H[2] + ro;
  const Cx<T>* Hwy = a.H[3] + ro;
  const T* kx = tb.kx;
  Cx<T> v[P];
  // phase 1: c2r along x           (src/derive2csh.f95:60-97)
  {
    const int g = th.g;
    Cx<T>* dst = arr(g);
    row_c2r<RF>(dst, th.lane, v, tb, [&](int k) -> Cx<T> {
      switch (g) {
        case 0: return ldg(Hpsiy + k);                                   // ux = i ky psi
        case 1: { const Cx<T> z = ikmul(__ldg(kx + k), ldg(Hpsi + k));   // uy = -i kx psi
                  return cx<T>(-z.x, -z.y); }
        case 2: return ikmul(__ldg(kx + k), ldg(Hw + k));                // i kx W
        default: return ldg(Hwy + k);                                    // i ky W
      }
    }, sync);
    sync();
    fft_emit<RF>(th.lane, v, [&](int, int n, Cx<T> z) {
      dst[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb));
    });
  }
  __syncthreads();
  // phase 2: products               (:99-106)
  for (int m = th.g * NTR + th.lane; m < M; m += G * NTR) {
    const Cx<T> ux = arr(0)[m], uy = arr(1)[m], wx = arr(2)[m], wy = arr(3)[m];
    arr(0)[m] = cx<T>(mul_rn(ux.x, wx.x) + mul_rn(uy.x, wy.x), mul_rn(ux.y, wx.y) + mul_rn(uy.y, wy.y));
  }
  __syncthreads();
  // phase 3: r2c along x            (:108-134, merged by linearity)
  if (th.g == 0) {
    row_r2c_begin<RF>(th.lane, v, tb, [&](int n) { return arr(0)[n]; });
    Cx<T>* xo = a.X + ro;
    row_r2c_finish<RF>(arr(1), th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
  }
}

template <int Nx, class T>
static void launch_row_vort(const RowVortArgs<T>& a0, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  RowVortArgs<T> a = a0;
  const size_t per_row = (size_t)4 * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>);
  a.rb = 1;
  while (a.rb * 2 * 4 * NTR <= 128 && Ny % (a.rb * 2) == 0 && (a.rb * 2) * per_row <= 110 * 1024) a.rb *= 2;
  auto kern = k_row_vort<T, M, P>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, 4 * NTR * a.rb, smem, st>>>(a);
}

// ------------------------------------------------------------ forward y pass
template <class T> struct ColFwdVortArgs {
  Tables<T> tb;
  const Cx<T>* X;      // x-transformed nonlinear term
  const Cx<T>* w;      // omega (the RHS input), for the viscous term
  T nu, alpha, lam;
  int screened;
  StepArgs<T> step;
};

// d omega/dt = -(alpha * mask(NL) + nu (kx^2 + ky^2) W)
//   (src/derive2csh.f95:136-145, src/derive2css.f95:122-131)
template <class T, int L, int CB, int P>
__global__ void __launch_bounds__(CB * L / P, TARA_MINB(CB * L / P)) k_col_fwd_vort(const ColFwdVortArgs<T> a) {
  using F = FFTB<L, CB, P>;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  const int c0 = blockIdx.x * CB;
  const int Nh = a.tb.Nh, ld = a.tb.ld;
  Cx<T> v[P];
  fft_run<F, -1>(sm, threadIdx.x, v, TwGlobal<T>{a.tb.tw_col}, [&](int t, int i) -> Cx<T> {
    const int c = c0 + t;
    if (c >= Nh) return cx<T>(0, 0);
    return ldg(a.X + (size_t)i * ld + c);
  }, SyncBlock{});
  fft_emit<F>(threadIdx.x, v, [&](int t, int j, Cx<T> x) {
    const int c = c0 + t;
    if (c >= Nh) return;
    const size_t idx = (size_t)j * ld + c;
    const T kx = __ldg(a.tb.kx + c), ky = __ldg(a.tb.ky + j);
    const T k2 = ksq(kx, ky);
    const Cx<T> w = ldg(a.w + idx);
    Cx<T> W = w;
    if (a.screened) W = apply_psi_mul(MUL_WD, a.lam, kx, ky, c == 0 && j == 0, w);
    const bool masked = c >= __ldg(a.tb.cut + j);
    const Cx<T> nl = masked ? cx<T>(0, 0) : x;
    const T vk = mul_rn(a.nu, k2);
    const Cx<T> s = cx<T>(mul_rn(a.alpha, nl.x) + mul_rn(vk, W.x), mul_rn(a.alpha, nl.y) + mul_rn(vk, W.y));
    step_apply(a.step, 0, idx, cx<T>(-s.x, -s.y));
  });
}

template <int L, class T>
inline void col_fwd_vort_dispatch(const ColFwdVortArgs<T>& a, cudaStream_t st) {
  constexpr int CB = ColCfg<T, L>::CB, P = ColCfg<T, L>::P;
  auto kern = k_col_fwd_vort<T, L, CB, P>;
  const size_t smem = col_smem_bytes<T, L>();
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<(a.tb.Nh + CB - 1) / CB, CB * L / P, smem, st>>>(a);
}

template <class T>
int vort_rhs(const Grid<T>& g, VortWork<T>& w, const VortParamsT<T>& p, Cx<T>* const in[1],
             const StepArgs<T>& step, cudaStream_t st) {
  const T lam = p.screened ? p.lambda : (T)0;
  ColInvArgs<T> ci{};
  ci.tb = g.tb;
  const int mul[4] = {MUL_PSI, MUL_IKY_PSI, p.screened ? MUL_WD : MUL_ONE, p.screened ? MUL_IKY_WD : MUL_IKY};
  for (int q = 0; q < 4; q++) ci.job[q] = ColInvJob<T>{in[0], w.H[q], mul[q], lam};
  prof_mark(g.prof, st, KK_COL_INV);
  run_col_inv(ci, 4, st);

  if ((size_t)4 * (g.Nx / 2 + g.Nx / 32 + 1) * sizeof(Cx<T>) > 227 * 1024) {
    set_error("vorticity row pass does not fit in shared memory at this Nx and precision");
    return TARA_EUNSUPPORTED;
  }
  RowVortArgs<T> ra{};
  ra.tb = g.tb;
  for (int q = 0; q < 4; q++) ra.H[q] = w.H[q];
  ra.X = w.X[0];
  prof_mark(g.prof, st, KK_ROW_VORT);
  TARA_DISPATCH_LEN(g.Nx, launch_row_vort, ra, g.Ny, st)

  ColFwdVortArgs<T> cf{};
  cf.tb = g.tb;
  cf.X = w.X[0];
  cf.w = in[0];
  cf.nu = p.nu;
  cf.alpha = p.screened ? p.alpha : (T)1;
  cf.lam = lam;
  cf.screened = p.screened;
  cf.step = step;
  prof_mark(g.prof, st, KK_COL_FWD_VORT);
  TARA_DISPATCH_LEN(g.Ny, col_fwd_vort_dispatch, cf, st)
  prof_mark(g.prof, st, KK_END);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

}  // namespace tara
