// Right-hand side of 2D compressible isothermal MHD in conservative form
// (reference: src/derive2com.f95:6-426) as five kernels:
//
//   k_col_inv      y-inverse of the six state fields (rho, rho ux, rho uy, E,
//                  Bx, By) [and of i ky Bx when curl B is corrected]
//   k_row_com1     per row: six c2r along x, u = rho u / rho, B^2, P = CS^2 rho,
//                  the momentum/induction fluxes and the part of the energy flux
//                  that needs no derivative; r2c of ux, uy, Mxx, Mxy, Myy,
//                  Mag, Ax, Ay (+ forcing)                      (:88-122, :180-213)
//   k_col_rt       d(uy)/dy: y-forward of X(uy), times i ky, y-inverse (:142-168)
//   k_row_com2     per row: d(ux)/dx from X(ux) (an x-only derivative: the y
//                  transforms of the reference cancel), d(uy)/dy, Bx, By, the
//                  curl-B terms of the energy flux and (div u)^2; adds their r2c
//                  to the energy fluxes                      (:183-209)
//   k_col_fwd_com  y-forward, i k multiplies, k^2 terms, dealiasing and the
//                  assembly of the six derivatives          (:262-419), fused with
//                  the stepper update.
//
// Mom_y_1 is Mom_x_2 (src/derive2com.f95:197, :199) and Mag_y is -Mag_x
// exactly (:212-213), so each is transformed once.  The reference also
// transforms i ky Bx and i kx By (:170-174) and then overwrites the results
// (:186-187); those two transforms are skipped unless fix_curlB is set.
#pragma once
#include "models.h"

namespace tara {

enum : int { XUX = 0, XUY, XMXX, XMXY, XMYY, XMAG, XEX, XEY, XEV, XFX, XFY };
enum : int { HRHO = 0, HMX, HMY, HE, HBX, HBY, HDUY, HIKYBX };

template <class T> struct RowCom1Args {
  Tables<T> tb;
  const Cx<T>* H[6];
  Cx<T>* X[11];
  T cs2, A, kf, dx, dy;
  int forcing, rb;
};

template <class T, int M, int P>
__global__ void __launch_bounds__(128) k_row_com1(const RowCom1Args<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  const int r = threadIdx.x / NTR, lane = threadIdx.x % NTR;
  const int y = blockIdx.x * a.rb + r;
  const Tables<T>& tb = a.tb;
  Cx<T>* xs = sm + (size_t)r * 9 * M;
  Cx<T>* f[8];  // rho, rho ux, rho uy, E, Bx, By, ux, uy (pairs)
#pragma unroll
  for (int q = 0; q < 8; q++) f[q] = xs + (q + 1) * M;
  const size_t ro = (size_t)y * tb.ld;
  Cx<T> v[P];
  // six c2r along x, normalised                (src/derive2com.f95:70-102)
#pragma unroll 1
  for (int q = 0; q < 6; q++) {
    const Cx<T>* h = a.H[q] + ro;
    row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(h + k); });
    Cx<T>* dst = f[q];
    fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
      dst[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb));
    });
  }
  // velocity                                    (:105-106)
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T>) {
    const Cx<T> rho = f[0][n], mx = f[1][n], my = f[2][n];
    f[6][n] = cx<T>(mx.x / rho.x, mx.y / rho.y);
    f[7][n] = cx<T>(my.x / rho.x, my.y / rho.y);
  });
  __syncthreads();
  const T cs2 = a.cs2;
  // fluxes of one grid point                    (:193-213)
  auto flux = [&](int which, int n, int half) -> T {
    const T rho = half ? f[0][n].y : f[0][n].x;
    const T mx = half ? f[1][n].y : f[1][n].x;
    const T my = half ? f[2][n].y : f[2][n].x;
    const T E = half ? f[3][n].y : f[3][n].x;
    const T bx = half ? f[4][n].y : f[4][n].x;
    const T by = half ? f[5][n].y : f[5][n].x;
    const T ux = half ? f[6][n].y : f[6][n].x;
    const T uy = half ? f[7][n].y : f[7][n].x;
    const T B2 = bx * bx + by * by;
    const T Pr = cs2 * rho;
    switch (which) {
      case XUX: return ux;
      case XUY: return uy;
      case XMXX: return mx * ux + Pr + B2 / (T)2 - bx * bx;
      case XMXY: return mx * uy - bx * by;
      case XMYY: return my * uy + Pr + B2 / (T)2 - by * by;
      case XMAG: return uy * bx - by * ux;
      case XEX: return (E + Pr + B2 / (T)2) * ux - ux * bx * bx - uy * bx * by;
      case XEY: return (E + Pr + B2 / (T)2) * uy - ux * bx * by - uy * by * by;
      default: return (T)0;
    }
  };
  const int nout = a.forcing ? 11 : 8;
#pragma unroll 1
  for (int q = 0; q < nout; q++) {
    if (q == XEV) continue;
    Cx<T>* xo = a.X[q] + ro;
    row_r2c<RF>(xs, lane, NTR, v, tb,
                [&](int n) -> Cx<T> {
                  if (q == XFX || q == XFY) {
                    // Fx = -rho A sin(kf y_j), Fy = rho A sin(kf x_i) on the grid
                    // x_i = (i-1) dx, y_j = (j-1) dy                      (:109-110)
                    const Cx<T> rho = f[0][n];
                    if (q == XFX) {
                      const T s = sin(a.kf * ((T)y * a.dy));
                      return cx<T>(-rho.x * a.A * s, -rho.y * a.A * s);
                    }
                    const T s0 = sin(a.kf * ((T)(2 * n) * a.dx));
                    const T s1 = sin(a.kf * ((T)(2 * n + 1) * a.dx));
                    return cx<T>(rho.x * a.A * s0, rho.y * a.A * s1);
                  }
                  return cx<T>(flux(q, n, 0), flux(q, n, 1));
                },
                [&](int k, Cx<T> X) { st(xo + k, X); });
  }
}

template <class T> struct RowCom2Args {
  Tables<T> tb;
  const Cx<T>* Xux;
  const Cx<T>* Hduy;
  const Cx<T>* Hbx;
  const Cx<T>* Hby;
  const Cx<T>* Hikybx;
  Cx<T>* Xex;
  Cx<T>* Xey;
  Cx<T>* Xev;
  T eta, inv_nx;
  int fix_curlB, rb;
};

template <class T, int M, int P>
__global__ void __launch_bounds__(128) k_row_com2(const RowCom2Args<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  const int r = threadIdx.x / NTR, lane = threadIdx.x % NTR;
  const int y = blockIdx.x * a.rb + r;
  const Tables<T>& tb = a.tb;
  Cx<T>* xs = sm + (size_t)r * 6 * M;
  Cx<T>* dux = xs + M;
  Cx<T>* duy = xs + 2 * M;
  Cx<T>* bx = xs + 3 * M;
  Cx<T>* by = xs + 4 * M;
  Cx<T>* curl = xs + 5 * M;
  const size_t ro = (size_t)y * tb.ld;
  const T* kx = tb.kx;
  Cx<T> v[P];
  // d_ux_dx = c2r(i kx ux_k)/(Nx Ny): on a row this is c2r_x(i kx X(ux))/Nx   (:164, :183)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ikmul(__ldg(kx + k), ldg(a.Xux + ro + k)); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) { dux[n] = cx<T>(z.x * a.inv_nx, z.y * a.inv_nx); });
  // d_uy_dy                                                                    (:167, :184)
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(a.Hduy + ro + k); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) { duy[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb)); });
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(a.Hbx + ro + k); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) { bx[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb)); });
  row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(a.Hby + ro + k); });
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) { by[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb)); });
  if (!a.fix_curlB) {
    // d_Bx_dy = d_ux_dx/(NxNy), d_By_dx = d_uy_dy/(NxNy), curl = d_By_dx - d_Bx_dy   (:186-190)
    fft_emit<RF>(lane, v, [&](int, int n, Cx<T>) {
      const Cx<T> p = dux[n], q = duy[n];
      curl[n] = cx<T>(q.x / tb.nn - p.x / tb.nn, q.y / tb.nn - p.y / tb.nn);
    });
  } else {
    row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ikmul(__ldg(kx + k), ldg(a.Hby + ro + k)); });
    fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) { curl[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb)); });
    row_c2r<RF>(xs, lane, v, tb, [&](int k) { return ldg(a.Hikybx + ro + k); });
    fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) {
      const Cx<T> c = curl[n];
      curl[n] = cx<T>(c.x - normalise(z.x, tb), c.y - normalise(z.y, tb));
    });
  }
  __syncthreads();
  const T eta = a.eta;
  // Energy_x -= eta By curl_B ; Energy_y += eta Bx curl_B ; E_Visc = (div u)^2   (:204-209)
  Cx<T>* xex = a.Xex + ro;
  Cx<T>* xey = a.Xey + ro;
  Cx<T>* xev = a.Xev + ro;
  row_r2c<RF>(xs, lane, NTR, v, tb,
              [&](int n) {
                const Cx<T> b = by[n], c = curl[n];
                return cx<T>(-(eta * b.x * c.x), -(eta * b.y * c.y));
              },
              [&](int k, Cx<T> X) { st(xex + k, ld(xex + k) + X); });
  row_r2c<RF>(xs, lane, NTR, v, tb,
              [&](int n) {
                const Cx<T> b = bx[n], c = curl[n];
                return cx<T>(eta * b.x * c.x, eta * b.y * c.y);
              },
              [&](int k, Cx<T> X) { st(xey + k, ld(xey + k) + X); });
  row_r2c<RF>(xs, lane, NTR, v, tb,
              [&](int n) {
                const Cx<T> p = dux[n], q = duy[n];
                const T d0 = p.x + q.x, d1 = p.y + q.y;
                return cx<T>(d0 * d0, d1 * d1);
              },
              [&](int k, Cx<T> X) { st(xev + k, X); });
}

template <class T> struct ColFwdComArgs {
  Tables<T> tb;
  const Cx<T>* X[11];
  const Cx<T>* in[6];  // stage input (the state the RHS is evaluated at)
  T mu, eta;
  int forcing;
  StepArgs<T> step;
};

template <class T, int L, int CB, int P>
__global__ void __launch_bounds__(CB * L / P) k_col_fwd_com(const ColFwdComArgs<T> a) {
  using F = FFTB<L, CB, P>;
  constexpr int RL = F::Pl::R[F::S - 1];
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  const int f = blockIdx.y;
  const int c0 = blockIdx.x * CB;
  const int Nh = a.tb.Nh, ld = a.tb.ld;
  const T* kx = a.tb.kx;
  const T* ky = a.tb.ky;
  const int tid = threadIdx.x;
  Cx<T> v[P], d[P];
  auto fft = [&](const Cx<T>* X) {
    __syncthreads();
    fft_run<F, -1>(sm, tid, v, TwGlobal<T>{a.tb.tw_col}, [&](int t, int i) -> Cx<T> {
      const int c = c0 + t;
      if (c >= Nh) return cx<T>(0, 0);
      return ldg(X + (size_t)i * ld + c);
    }, SyncBlock{});
  };
  // visit the outputs of the last stage: g(idx, c, j, masked)
  auto each = [&](auto&& g) {
#pragma unroll
    for (int q = 0; q < P / RL; q++)
#pragma unroll
      for (int r = 0; r < RL; r++) {
        int t, i;
        F::template out_pos<F::S - 1>(tid, q, r, t, i);
        const int c = min(c0 + t, Nh - 1);
        g(q * RL + r, c, i, c >= __ldg(a.tb.cut + i));
      }
  };
  const Cx<T> zero = cx<T>(0, 0);
  const T mu = a.mu, eta = a.eta;
  switch (f) {
    case 0:  // d_rho = -(i kx rho_ux_k + i ky rho_uy_k)                     (:402)
      each([&](int q, int c, int j, bool m) {
        const size_t o = (size_t)j * ld + c;
        const Cx<T> p = m ? zero : ikmul(__ldg(kx + c), ldg(a.in[1] + o));
        const Cx<T> s = m ? zero : ikmul(__ldg(ky + j), ldg(a.in[2] + o));
        d[q] = -(p + s);
      });
      break;
    case 1:  // -(i kx Mxx + i ky Mxy) - mu (kx^2 + ky^2) ux_k + Fx_k       (:405-406)
    case 2:  // -(i kx Mxy + i ky Myy) - mu (kx^2 + ky^2) uy_k + Fy_k       (:408-409)
      fft(a.X[f == 1 ? XMXX : XMXY]);
      each([&](int q, int c, int j, bool m) { d[q] = m ? zero : ikmul(__ldg(kx + c), v[q]); });
      fft(a.X[f == 1 ? XMXY : XMYY]);
      each([&](int q, int c, int j, bool m) { d[q] = -(d[q] + (m ? zero : ikmul(__ldg(ky + j), v[q]))); });
      fft(a.X[f == 1 ? XUX : XUY]);
      each([&](int q, int c, int j, bool m) {
        const T k1 = __ldg(kx + c), k2 = __ldg(ky + j);
        const Cx<T> p = m ? zero : rmul(k1 * k1, v[q]);
        const Cx<T> s = m ? zero : rmul(k2 * k2, v[q]);
        d[q] = d[q] - rmul(mu, p + s);
      });
      if (a.forcing) {
        fft(a.X[f == 1 ? XFX : XFY]);
        each([&](int q, int, int, bool) { d[q] = d[q] + v[q]; });
      }
      break;
    case 3:  // -(i kx Ex + i ky Ey) + mu E_Visc_k                          (:412-413)
      fft(a.X[XEX]);
      each([&](int q, int c, int j, bool m) { d[q] = m ? zero : ikmul(__ldg(kx + c), v[q]); });
      fft(a.X[XEY]);
      each([&](int q, int c, int j, bool m) { d[q] = -(d[q] + (m ? zero : ikmul(__ldg(ky + j), v[q]))); });
      fft(a.X[XEV]);
      each([&](int q, int c, int j, bool m) { d[q] = d[q] + rmul(mu, m ? zero : v[q]); });
      break;
    default:  // 4: -i ky Mag_x - eta k^2 Bx ; 5: -i kx Mag_y - eta k^2 By    (:416-417)
      fft(a.X[XMAG]);
      each([&](int q, int c, int j, bool m) {
        const size_t o = (size_t)j * ld + c;
        const T k1 = __ldg(kx + c), k2 = __ldg(ky + j);
        const Cx<T> B = ldg(a.in[f] + o);
        // Mag_y_k = -Mag_x_k exactly
        const Cx<T> nl = m ? zero : (f == 4 ? ikmul(k2, v[q]) : ikmul(k1, -v[q]));
        const Cx<T> p = m ? zero : rmul(k1 * k1, B);
        const Cx<T> s = m ? zero : rmul(k2 * k2, B);
        d[q] = -nl - rmul(eta, p + s);
      });
      break;
  }
#pragma unroll
  for (int q = 0; q < P / RL; q++)
#pragma unroll
    for (int r = 0; r < RL; r++) {
      int t, i;
      F::template out_pos<F::S - 1>(tid, q, r, t, i);
      const int c = c0 + t;
      if (c < Nh) step_apply(a.step, f, (size_t)i * ld + c, d[q * RL + r]);
    }
}

template <int L, class T>
inline void col_fwd_com_dispatch(const ColFwdComArgs<T>& a, cudaStream_t st) {
  constexpr int CB = ColCfg<T, L>::CB, P = ColCfg<T, L>::P;
  auto kern = k_col_fwd_com<T, L, CB, P>;
  const size_t smem = col_smem_bytes<T, L>();
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid((a.tb.Nh + CB - 1) / CB, 6);
  kern<<<grid, CB * L / P, smem, st>>>(a);
}

template <int Nx, class T>
static void launch_row_com1(const RowCom1Args<T>& a0, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  RowCom1Args<T> a = a0;
  const size_t per_row = (size_t)9 * M * sizeof(Cx<T>);
  a.rb = rows_per_cta(NTR, Ny, per_row);
  auto kern = k_row_com1<T, M, P>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, NTR * a.rb, smem, st>>>(a);
}
template <int Nx, class T>
static void launch_row_com2(const RowCom2Args<T>& a0, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  RowCom2Args<T> a = a0;
  const size_t per_row = (size_t)6 * M * sizeof(Cx<T>);
  a.rb = rows_per_cta(NTR, Ny, per_row);
  auto kern = k_row_com2<T, M, P>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, NTR * a.rb, smem, st>>>(a);
}

template <class T>
int com_rhs(const Grid<T>& g, ComWork<T>& w, const ComParamsT<T>& p, Cx<T>* const in[6],
            const StepArgs<T>& step, cudaStream_t st) {
  if ((size_t)9 * (g.Nx / 2) * sizeof(Cx<T>) > 227 * 1024) {
    set_error("MHD row pass does not fit in shared memory at this Nx and precision");
    return TARA_EUNSUPPORTED;
  }
  const int forcing = p.A != (T)0;
  ColInvArgs<T> ci{};
  ci.tb = g.tb;
  for (int q = 0; q < 6; q++) ci.job[q] = ColInvJob<T>{in[q], w.H[q], MUL_ONE};
  int nj = 6;
  if (p.fix_curlB) ci.job[nj++] = ColInvJob<T>{in[4], w.H[HIKYBX], MUL_IKY};
  prof_mark(g.prof, st, KK_COL_INV);
  run_col_inv(ci, nj, st);

  RowCom1Args<T> r1{};
  r1.tb = g.tb;
  for (int q = 0; q < 6; q++) r1.H[q] = w.H[q];
  for (int q = 0; q < 11; q++) r1.X[q] = w.X[q];
  r1.cs2 = p.cs2;
  r1.A = p.A;
  r1.kf = p.kf;
  r1.dx = (T)(g.Lx / g.Nx);
  r1.dy = (T)(g.Ly / g.Ny);
  r1.forcing = forcing;
  prof_mark(g.prof, st, KK_ROW_COM1);
  TARA_DISPATCH_LEN(g.Nx, launch_row_com1, r1, g.Ny, st)

  ColRtArgs<T> rt{};
  rt.tb = g.tb;
  rt.src = w.X[XUY];
  rt.dst = w.H[HDUY];
  rt.mul = MUL_IKY;
  prof_mark(g.prof, st, KK_COL_RT);
  run_col_rt(rt, st);

  RowCom2Args<T> r2{};
  r2.tb = g.tb;
  r2.Xux = w.X[XUX];
  r2.Hduy = w.H[HDUY];
  r2.Hbx = w.H[HBX];
  r2.Hby = w.H[HBY];
  r2.Hikybx = w.H[HIKYBX];
  r2.Xex = w.X[XEX];
  r2.Xey = w.X[XEY];
  r2.Xev = w.X[XEV];
  r2.eta = p.eta;
  r2.inv_nx = (T)(1.0 / g.Nx);
  r2.fix_curlB = p.fix_curlB;
  prof_mark(g.prof, st, KK_ROW_COM2);
  TARA_DISPATCH_LEN(g.Nx, launch_row_com2, r2, g.Ny, st)

  ColFwdComArgs<T> cf{};
  cf.tb = g.tb;
  for (int q = 0; q < 11; q++) cf.X[q] = w.X[q];
  for (int q = 0; q < 6; q++) cf.in[q] = in[q];
  cf.mu = p.mu;
  cf.eta = p.eta;
  cf.forcing = forcing;
  cf.step = step;
  prof_mark(g.prof, st, KK_COL_FWD_COM);
  TARA_DISPATCH_LEN(g.Ny, col_fwd_com_dispatch, cf, st)
  prof_mark(g.prof, st, KK_END);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

}  // namespace tara
