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
  CflRow cfl;  // cfl.lam set: fold the rows' largest signal-speed rate into it
};

// One group per transform.  Phase 1: eleven c2r in eleven groups (each
// group's output array is its exchange buffer).  Phase 2: the products, in
// place.  Phase 3: three r2c, exchange buffers in the freed arrays 3..5.
// Rows y0 + (thread row) of the CTA; every thread of the CTA takes part
// (blockDim = rows * 11 * M/P), smem holds rows * 11 arrays.
template <class T, int M, int P>
__device__ __forceinline__ void row_coh_rows(const RowCohArgs<T>& a, int y0, Cx<T>* smem) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = 11, ARR = RF::SMEM_ELEMS;
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* base = smem + (size_t)th.row * G * ARR;
  // 0 n, 1 ux, 2 uy, 3 dn/dx, 4 dn/dy, 5 dux/dx, 6 dux/dy, 7 duy/dx, 8 duy/dy,
  // 9 mux d2ux/dx2 + muy d2ux/dy2, 10 mux d2uy/dx2 + muy d2uy/dy2   (pairs x[2m], x[2m+1])
  auto arr = [&](int q) { return base + q * ARR; };
  const int y = y0 + th.row;
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
  // phase 1: c2r along x                          (src/derive2coh.f95:92-151)
  {
    const int g = th.g;
    Cx<T>* dst = arr(g);
    row_c2r<RF>(dst, th.lane, v, tb, [&](int k) -> Cx<T> {
      const T k1 = __ldg(kx + k);
      switch (g) {
        case 0: return ldg(Hn + k);
        case 1: return ldg(Hux + k);
        case 2: return ldg(Huy + k);
        case 3: return ikmul(k1, ldg(Hn + k));
        case 4: return ldg(Hny + k);
        case 5: return ikmul(k1, ldg(Hux + k));
        case 6: return ldg(Huxy + k);
        case 7: return ikmul(k1, ldg(Huy + k));
        case 8: return ldg(Huyy + k);
        case 9: return rmul(mux, rmul(k1 * k1, ldg(Hux + k))) + rmul(muy, ldg(Huxyy + k));
        default: return rmul(mux, rmul(k1 * k1, ldg(Huy + k))) + rmul(muy, ldg(Huyyy + k));
      }
    }, sync);
    sync();
    fft_emit<RF>(th.lane, v, [&](int, int n, Cx<T> z) {
      dst[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb));
    });
  }
  __syncthreads();
  // phase 2: products                              (:153-165)
  //   NLn = ux dn/dx + uy dn/dy + n (dux/dx + duy/dy)
  //   Fx  = (ux dux/dx + uy dux/dy) + visc_x/n + CS^2 (dn/dx)/n   (+ same for y)
  // CFL control: largest (|ux| + CS)/dx + (|uy| + CS)/dy of the points, in FP64
  const bool cfl = a.cfl.lam != nullptr;
  const double cs = cfl ? sqrt(a.cfl.cs2) : 0.0;
  double cmax = 0.0;
  for (int m = th.g * NTR + th.lane; m < M; m += G * NTR) {
    T q[11][2];
#pragma unroll
    for (int f = 0; f < 11; f++) {
      const Cx<T> z = arr(f)[m];
      q[f][0] = z.x;
      q[f][1] = z.y;
    }
    T o[3][2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const T n = q[0][h], ux = q[1][h], uy = q[2][h];
      const T in = (T)1 / n;  // one reciprocal for the four divisions by n (last-bit differences)
      o[0][h] = ux * q[3][h] + uy * q[4][h] + n * (q[5][h] + q[8][h]);
      o[1][h] = (ux * q[5][h] + uy * q[6][h]) + q[9][h] * in + cs2 * (q[3][h] * in);
      o[2][h] = (ux * q[7][h] + uy * q[8][h]) + q[10][h] * in + cs2 * (q[4][h] * in);
    }
#pragma unroll
    for (int f = 0; f < 3; f++) arr(f)[m] = cx<T>(o[f][0], o[f][1]);
    if (cfl)
      for (int h = 0; h < 2; h++) cmax = nan_max(cmax, cfl_rate(q[1][h], q[2][h], cs, a.cfl.idx, a.cfl.idy));
  }
  if (cfl) cfl_fold(cmax, a.cfl.lam);
  __syncthreads();
  // phase 3: three r2c along x                     (:172-197, merged by linearity)
  if (th.g < 3) {
    const int g = th.g;
    row_r2c_begin<RF>(th.lane, v, tb, [&](int n) { return arr(g)[n]; });
    Cx<T>* xo = a.X[g] + ro;
    row_r2c_finish<RF>(arr(3 + g), th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
  }
}

template <class T, int M, int P>
// Two CTAs per SM where a row's CTA has at most 352 threads (their shared
// memory fits twice; left to itself the compiler uses ~156 registers at
// Nx = 1024 and only one CTA fits: 141 vs 152 us per launch); larger rows
// keep one CTA.
__global__ void __launch_bounds__(TARA_ROW_LB(11 * (M / P)), (11 * (M / P) <= 352 ? 2 : 1))
    k_row_coh(const RowCohArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  row_coh_rows<T, M, P>(a, blockIdx.x * a.rb, reinterpret_cast<Cx<T>*>(smraw));
}

template <int Nx, class T>
static void launch_row_coh(const RowCohArgs<T>& a0, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  RowCohArgs<T> a = a0;
  const size_t per_row = (size_t)11 * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>);
  a.rb = 1;
  while (a.rb * 2 * 11 * NTR <= 128 && Ny % (a.rb * 2) == 0 && (a.rb * 2) * per_row <= 110 * 1024) a.rb *= 2;
  auto kern = k_row_coh<T, M, P>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, 11 * NTR * a.rb, smem, st>>>(a);
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

  if ((size_t)11 * (g.Nx / 2 + g.Nx / 32 + 1) * sizeof(Cx<T>) > 227 * 1024 || 11 * (g.Nx / 2) / 16 > 1024) {
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
  if (p.cfl.dev) ra.cfl = CflRow{&p.cfl.dev->lam, p.cfl.idx, p.cfl.idy, p.cfl.cs2};
  prof_mark(g.prof, st, KK_ROW_COH);
  TARA_DISPATCH_LEN(g.Nx, launch_row_coh, ra, g.Ny, st)
  if (p.cfl.dev) {  // dt of this step, before the stepper update reads it
    prof_mark(g.prof, st, KK_CFL);
    TARA_TRY(launch_cfl_update(p.cfl, g.tb.status, st));
  }

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
