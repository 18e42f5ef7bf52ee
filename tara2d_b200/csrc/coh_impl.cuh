// Right-hand side of 2D compressible isothermal hydro (reference:
// src/derive2coh.f95:6-265) as three kernels:
//
//   k_col_inv        y-inverse of n, ux, uy and of their i*ky / ky^2 multiples
//                    (8 half-real fields; the kx multipliers are applied later
//                    on the rows, where they commute with the y transform)
//   k_row_coh        per grid row: 11 c2r along x (n, ux, uy, dn/dx, dn/dy,
//                    dux/dx, dux/dy, duy/dx, duy/dy and the two viscous
//                    combinations mux*d2/dx2 + muy*d2/dy2), the real-space
//                    products, and one r2c per equation.  The reference's nine
//                    r2c and its final sum (src/derive2coh.f95:172-197, 251-252)
//                    are merged by linearity: r2c(NLx) + mux*r2c(Viscxx) +
//                    muy*r2c(Viscxy) + CS^2*r2c(Px) = r2c(NLx + (mux*Viscxx +
//                    muy*Viscxy) + CS^2*Px), all masked by the same 2/3 rule.
//   k_col_fwd_simple y-forward, dealiasing, sign, stepper update.
#pragma once
#include "models.h"

namespace tara {

template <class T> struct RowCohArgs {
  Tables<T> tb;
  const Cx<T>* H[8];
  Cx<T>* X[3];
  T mux, muy, cs2;
  int rb;
};

template <class T, int M, int P>
__global__ void __launch_bounds__(128) k_row_coh(const RowCohArgs<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  const int r = threadIdx.x / NTR, lane = threadIdx.x % NTR;
  const int y = blockIdx.x * a.rb + r;
  const Tables<T>& tb = a.tb;
  Cx<T>* xs = sm + (size_t)r * 7 * M;
  Cx<T>* rn = xs + M;       // real fields stored as pairs (x[2m], x[2m+1])
  Cx<T>* rux = xs + 2 * M;
  Cx<T>* ruy = xs + 3 * M;
  Cx<T>* fn = xs + 4 * M;
  Cx<T>* fx = xs + 5 * M;
  Cx<T>* fy = xs + 6 * M;
  const size_t ro = (size_t)y * tb.ld;
  const Cx<T>* Hn = a.H[0] + ro;
  const Cx<T>* Hny = a.H[1] + ro;
  const Cx<T>* Hux = a.H[2] + ro;
  const Cx<T>* Huxy = a.H[3] + ro;
  const Cx<T>* Huxyy = a.H[4] + ro;
  const Cx<T>* Huy = a.H[5] + ro;
  const Cx<T>* Huyy = a.H[6] + ro;
  const Cx<T>* Huyyy = a.H[7] + ro;
  const T* kx = tb.kx;
  const T mux = a.mux, muy = a.muy, cs2 = a.cs2;
  Cx<T> v[P];

  auto store = [&](Cx<T>* dst) {
    fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
      dst[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb));
    });
  };
  // n, ux, uy                                   (src/derive2coh.f95:92-99)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(Hn + k); });
  store(rn);
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(Hux + k); });
  store(rux);
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(Huy + k); });
  store(ruy);

  // dn/dx: NLn = ux*dn/dx + ..., Px = dn/dx / n   (:158, :162)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ikmul(__ldg(kx + k), ldg(Hn + k)); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> N = rn[n], U = rux[n];
    fn[n] = cx<T>(U.x * d0, U.y * d1);
    fx[n] = cx<T>(cs2 * (d0 / N.x), cs2 * (d1 / N.y));
  });
  // dn/dy                                        (:159, :162)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(Hny + k); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> N = rn[n], V = ruy[n], F = fn[n];
    fn[n] = cx<T>(F.x + V.x * d0, F.y + V.y * d1);
    fy[n] = cx<T>(cs2 * (d0 / N.x), cs2 * (d1 / N.y));
  });
  // dux/dx: NLn += n*dux/dx, NLx = ux*dux/dx     (:162, :164)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ikmul(__ldg(kx + k), ldg(Hux + k)); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> N = rn[n], U = rux[n], F = fn[n], G = fx[n];
    fn[n] = cx<T>(F.x + N.x * d0, F.y + N.y * d1);
    fx[n] = cx<T>(G.x + U.x * d0, G.y + U.y * d1);
  });
  // duy/dy: NLn += n*duy/dy, NLy = uy*duy/dy     (:162, :165)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(Huyy + k); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> N = rn[n], V = ruy[n], F = fn[n], G = fy[n];
    fn[n] = cx<T>(F.x + N.x * d0, F.y + N.y * d1);
    fy[n] = cx<T>(G.x + V.x * d0, G.y + V.y * d1);
  });
  // dux/dy: NLx += uy*dux/dy                     (:164)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(Huxy + k); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> V = ruy[n], G = fx[n];
    fx[n] = cx<T>(G.x + V.x * d0, G.y + V.y * d1);
  });
  // duy/dx: NLy += ux*duy/dx                     (:165)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ikmul(__ldg(kx + k), ldg(Huy + k)); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> U = rux[n], G = fy[n];
    fy[n] = cx<T>(G.x + U.x * d0, G.y + U.y * d1);
  });
  // viscous x: (mux*d2ux/dx2 + muy*d2ux/dy2)/n   (:153-154, :251)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) {
    const T k2 = __ldg(kx + k) * __ldg(kx + k);
    return rmul(mux, rmul(k2, ldg(Hux + k))) + rmul(muy, ldg(Huxyy + k));
  });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> N = rn[n], G = fx[n];
    fx[n] = cx<T>(G.x + d0 / N.x, G.y + d1 / N.y);
  });
  // viscous y                                    (:155-156, :252)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) {
    const T k2 = __ldg(kx + k) * __ldg(kx + k);
    return rmul(mux, rmul(k2, ldg(Huy + k))) + rmul(muy, ldg(Huyyy + k));
  });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
    const T d0 = normalise(z.x, tb), d1 = normalise(z.y, tb);
    const Cx<T> N = rn[n], G = fy[n];
    fy[n] = cx<T>(G.x + d0 / N.x, G.y + d1 / N.y);
  });
  __syncthreads();
  // three r2c along x                            (:172-197 merged)
  Cx<T>* Xn = a.X[0] + ro;
  Cx<T>* Xx = a.X[1] + ro;
  Cx<T>* Xy = a.X[2] + ro;
  row_r2c<RF>(xs, lane, NTR, v, tb, [&](int n) { return fn[n]; }, [&](int k, Cx<T> X) { st(Xn + k, X); });
  row_r2c<RF>(xs, lane, NTR, v, tb, [&](int n) { return fx[n]; }, [&](int k, Cx<T> X) { st(Xx + k, X); });
  row_r2c<RF>(xs, lane, NTR, v, tb, [&](int n) { return fy[n]; }, [&](int k, Cx<T> X) { st(Xy + k, X); });
}

template <int Nx, class T>
static void launch_row_coh(const RowCohArgs<T>& a0, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  RowCohArgs<T> a = a0;
  const size_t per_row = (size_t)7 * M * sizeof(Cx<T>);
  a.rb = rows_per_cta(NTR, Ny, per_row);
  auto kern = k_row_coh<T, M, P>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, NTR * a.rb, smem, st>>>(a);
}

template <class T>
int coh_rhs(const Grid<T>& g, CohWork<T>& w, const CohParamsT<T>& p, Cx<T>* const in[3],
            const StepArgs<T>& step, cudaStream_t st) {
  ColInvArgs<T> ci{};
  ci.tb = g.tb;
  const int src[8] = {0, 0, 1, 1, 1, 2, 2, 2};
  const int mul[8] = {MUL_ONE, MUL_IKY, MUL_ONE, MUL_IKY, MUL_KY2, MUL_ONE, MUL_IKY, MUL_KY2};
  for (int q = 0; q < 8; q++) ci.job[q] = ColInvJob<T>{in[src[q]], w.H[q], mul[q]};
  prof_mark(g.prof, st, KK_COL_INV);
  run_col_inv(ci, 8, st);

  if ((size_t)7 * (g.Nx / 2) * sizeof(Cx<T>) > 227 * 1024) {
    set_error("hydro row pass does not fit in shared memory at this Nx and precision");
    return TARA_EUNSUPPORTED;
  }
  RowCohArgs<T> ra{};
  ra.tb = g.tb;
  for (int q = 0; q < 8; q++) ra.H[q] = w.H[q];
  for (int q = 0; q < 3; q++) ra.X[q] = w.X[q];
  ra.mux = p.mux;
  ra.muy = p.muy;
  ra.cs2 = p.cs2;
  prof_mark(g.prof, st, KK_ROW_COH);
  TARA_DISPATCH_LEN(g.Nx, launch_row_coh, ra, g.Ny, st)

  ColFwdSimpleArgs<T> cf{};
  cf.tb = g.tb;
  for (int q = 0; q < 3; q++) { cf.X[q] = w.X[q]; cf.sign[q] = (T)-1; }
  cf.step = step;
  prof_mark(g.prof, st, KK_COL_FWD_SIMPLE);
  run_col_fwd_simple(cf, 3, st);
  prof_mark(g.prof, st, KK_END);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

}  // namespace tara
