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
//                  the stepper update and, while stepping, with the y-inverse
//                  of the next RHS input (k_col_inv then runs only where a
//                  run starts).
//
// Mom_y_1 is Mom_x_2 (src/derive2com.f95:197, :199) and Mag_y is -Mag_x
// exactly (:212-213), so each is transformed once.  The reference also
// transforms i ky Bx and i kx By (:170-174) and then overwrites the results
// (:186-187); those two transforms are skipped unless fix_curlB is set.
#pragma once
#include "models.h"

namespace tara {

// XEX2/XEY2: the curl-B parts of the energy fluxes (second row pass), added
// to XEX/XEY as the column pass loads them
enum : int { XUX = 0, XUY, XMXX, XMXY, XMYY, XMAG, XEX, XEY, XEV, XFX, XFY, XEX2, XEY2 };
enum : int { HRHO = 0, HMX, HMY, HE, HBX, HBY, HDUY, HIKYBX };

// Rows per CTA so that a CTA has at least ~128 threads, within the shared
// memory budget and dividing Ny.
inline int row_cta_rows(int threads_per_row, size_t smem_per_row, int Ny, int max_threads = 1024) {
  int rb = 1;
  while (rb * 2 * threads_per_row <= 128 && rb * 2 * threads_per_row <= max_threads && Ny % (rb * 2) == 0 &&
         (rb * 2) * smem_per_row <= 110 * 1024)
    rb *= 2;
  return rb;
}

// ---------------------------------------------------------------- row pass 1
// One group per transform: phase 1 runs the six c2r of a row in six groups
// (each group's output array is also its exchange buffer), phase 2 forms the
// velocity, phase 3 runs the eight r2c in eight groups; once every group has
// gathered its inputs the eight field arrays become their exchange buffers.
// LOW (rows too long for eight arrays in shared memory): six arrays, the
// velocity is formed where it is used, and the last two r2c run after the
// first six have released their arrays.
template <class T> struct RowCom1Args {
  Tables<T> tb;
  const Cx<T>* H[6];
  Cx<T>* X[11];
  T cs2;
  int rb;
  CflRow cfl;  // cfl.lam set: fold the rows' largest signal-speed rate into it
};

// Rows y0 .. y0 + (blockDim.x / (8 M/P)) - 1 by the whole CTA (8 groups of
// M/P threads per row), in the CTA's dynamic shared memory.
template <class T, int M, int P, bool LOW>
__device__ __forceinline__ void row_com1_rows(const RowCom1Args<T>& a, int y0) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = 8, ARR = RF::SMEM_ELEMS, NA = LOW ? 6 : 8;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* base = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * NA * ARR;
  Cx<T>* f[8];  // rho, rho ux, rho uy, E, Bx, By, ux, uy (pairs x[2m], x[2m+1])
#pragma unroll
  for (int q = 0; q < 8; q++) f[q] = base + (q < NA ? q : q - NA) * ARR;
  const int y = y0 + th.row;
  const size_t ro = (size_t)y * tb.ld;
  Cx<T> v[P];
  // phase 1: six c2r along x, normalised         (src/derive2com.f95:70-102)
  if (th.g < 6) {
    const Cx<T>* h = a.H[th.g] + ro;
    Cx<T>* dst = f[th.g];
    row_c2r<RF>(dst, th.lane, v, tb, [&](int k) { return ldg(h + k); }, sync);
    sync();
    fft_emit<RF>(th.lane, v, [&](int, int n, Cx<T> z) {
      dst[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb));
    });
  }
  __syncthreads();
  if (a.cfl.lam) {
    // CFL control: largest (|ux| + cf)/dx + (|uy| + cf)/dy of the CTA's
    // points, cf = sqrt(CS^2 + |B|^2/rho) (fast magnetosonic speed), in FP64
    double m = 0.0;
    for (int n = th.g * NTR + th.lane; n < M; n += G * NTR) {
      const Cx<T> r = f[0][n], mx = f[1][n], my = f[2][n], bx = f[4][n], by = f[5][n];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const double rho = h ? r.y : r.x;
        const double ux = (h ? mx.y : mx.x) / rho, uy = (h ? my.y : my.x) / rho;
        const double b2 = h ? (double)bx.y * bx.y + (double)by.y * by.y : (double)bx.x * bx.x + (double)by.x * by.x;
        const double c = sqrt(a.cfl.cs2 + b2 / rho);
        m = nan_max(m, cfl_rate(ux, uy, c, a.cfl.idx, a.cfl.idy));
      }
    }
    cfl_fold(m, a.cfl.lam);
  }
  // flux q at one point                                                (:105-106, :193-213)
  const T cs2 = a.cs2;
  auto flux = [&](int qq, T rho, T mx, T my, T E, T bx, T by) -> T {
    // u = (rho u)/rho through one reciprocal (the reference divides twice;
    // the results differ in the last bit)
    const T ir = (T)1 / rho;
    const T ux = mx * ir, uy = my * ir;
    const T B2 = bx * bx + by * by;
    const T Pr = cs2 * rho;
    switch (qq) {
      case XUX: return ux;
      case XUY: return uy;
      case XMXX: return mx * ux + Pr + B2 / (T)2 - bx * bx;
      case XMXY: return mx * uy - bx * by;
      case XMYY: return my * uy + Pr + B2 / (T)2 - by * by;
      case XMAG: return uy * bx - by * ux;
      case XEX: return (E + Pr + B2 / (T)2) * ux - ux * bx * bx - uy * bx * by;
      default: return (E + Pr + B2 / (T)2) * uy - ux * bx * by - uy * by * by;  // XEY
    }
  };
  // phase 2 (eight arrays): all eight fluxes of every point, once, in place
  // (each point's six inputs are read before its eight outputs are written)
  if constexpr (!LOW) {
    for (int n = th.g * NTR + th.lane; n < M; n += G * NTR) {
      Cx<T> F[6];
#pragma unroll
      for (int k = 0; k < 6; k++) F[k] = f[k][n];
      T o[8][2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const T rho = h ? F[0].y : F[0].x, mx = h ? F[1].y : F[1].x, my = h ? F[2].y : F[2].x;
        const T E = h ? F[3].y : F[3].x, bx = h ? F[4].y : F[4].x, by = h ? F[5].y : F[5].x;
#pragma unroll
        for (int qq = 0; qq < 8; qq++) o[qq][h] = flux(qq, rho, mx, my, E, bx, by);
      }
#pragma unroll
      for (int qq = 0; qq < 8; qq++) f[qq][n] = cx<T>(o[qq][0], o[qq][1]);
    }
    __syncthreads();
  }
  // phase 3: flux th.g at the stage-0 points (six arrays: formed here), then r2c
  const int q = th.g;
  row_r2c_begin<RF>(th.lane, v, tb, [&](int n) -> Cx<T> {
    if constexpr (!LOW) {
      return f[q][n];
    } else {
      Cx<T> F[6];
#pragma unroll
      for (int k = 0; k < 6; k++) F[k] = f[k][n];
      T o[2];
#pragma unroll
      for (int h = 0; h < 2; h++)
        o[h] = flux(q, h ? F[0].y : F[0].x, h ? F[1].y : F[1].x, h ? F[2].y : F[2].x, h ? F[3].y : F[3].x,
                    h ? F[4].y : F[4].x, h ? F[5].y : F[5].x);
      return cx<T>(o[0], o[1]);
    }
  });
  __syncthreads();  // every group has its inputs: the field arrays are free
  Cx<T>* xo = a.X[q] + ro;
  if (q < NA) row_r2c_finish<RF>(f[q], th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
  if constexpr (LOW) {
    __syncthreads();  // arrays 0 and 1 are free again
    if (q >= NA) row_r2c_finish<RF>(f[q], th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
  }
}
template <class T, int M, int P, bool LOW>
__global__ void __launch_bounds__(TARA_ROW_LB(8 * (M / P))) k_row_com1(const RowCom1Args<T> a) {
  row_com1_rows<T, M, P, LOW>(a, blockIdx.x * a.rb);
}

// Forcing (only when A != 0):  Fx = -rho A sin(kf y_j), Fy = rho A sin(kf x_i)
// on the grid x_i = (i-1) dx, y_j = (j-1) dy                       (:109-110)
template <class T> struct RowForceArgs {
  Tables<T> tb;
  const Cx<T>* Hrho;
  Cx<T>* Xfx;
  Cx<T>* Xfy;
  T A, kf, dx, dy;
  int rb;
};
template <class T, int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(2 * (M / P))) k_row_force(const RowForceArgs<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = 2, ARR = RF::SMEM_ELEMS;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* rho = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * 3 * ARR;
  Cx<T>* xs = rho + (1 + th.g) * ARR;
  const int y = blockIdx.x * a.rb + th.row;
  const size_t ro = (size_t)y * tb.ld;
  Cx<T> v[P];
  if (th.g == 0) {
    row_c2r<RF>(xs, th.lane, v, tb, [&](int k) { return ldg(a.Hrho + ro + k); }, sync);
    fft_emit<RF>(th.lane, v, [&](int, int n, Cx<T> z) { rho[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb)); });
  }
  __syncthreads();
  const T sy = sin(a.kf * ((T)y * a.dy));
  row_r2c_begin<RF>(th.lane, v, tb, [&](int n) -> Cx<T> {
    const Cx<T> r = rho[n];
    if (th.g == 0) return cx<T>(-r.x * a.A * sy, -r.y * a.A * sy);
    return cx<T>(r.x * a.A * sin(a.kf * ((T)(2 * n) * a.dx)), r.y * a.A * sin(a.kf * ((T)(2 * n + 1) * a.dx)));
  });
  Cx<T>* xo = (th.g == 0 ? a.Xfx : a.Xfy) + ro;
  row_r2c_finish<RF>(xs, th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
}

// ---------------------------------------------------------------- row pass 2
// Groups: d(ux)/dx, d(uy)/dy, Bx, By [, dBy/dx, dBx/dy when corrected]; then
// curl B; then three r2c (energy-flux curl terms and E_Visc).
template <class T> struct RowCom2Args {
  Tables<T> tb;
  const Cx<T>* Xux;
  const Cx<T>* Hduy;
  const Cx<T>* Hbx;
  const Cx<T>* Hby;
  const Cx<T>* Hikybx;
  Cx<T>* Xex2;  // written, not updated: the column pass adds them to Ex, Ey
  Cx<T>* Xey2;
  Cx<T>* Xev;
  T eta, inv_nx;
  int rb;
};

// Rows y0 .. by the whole CTA (G groups of M/P threads per row).
template <class T, int M, int P, int FIX>
__device__ __forceinline__ void row_com2_rows(const RowCom2Args<T>& a, int y0) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = FIX ? 6 : 4, NA = FIX ? 6 : 5, ARR = RF::SMEM_ELEMS;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* base = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * NA * ARR;
  Cx<T>* dux = base;
  Cx<T>* duy = base + ARR;
  Cx<T>* bx = base + 2 * ARR;
  Cx<T>* by = base + 3 * ARR;
  Cx<T>* curl = base + 4 * ARR;
  Cx<T>* aux = base + (NA - 1) * ARR;  // dBx/dy when corrected
  const int y = y0 + th.row;
  const size_t ro = (size_t)y * tb.ld;
  const T* kx = tb.kx;
  Cx<T> v[P];
  // phase 1                                                              (:164-187)
  {
    const int g = th.g;
    Cx<T>* dst = g == 0 ? dux : g == 1 ? duy : g == 2 ? bx : g == 3 ? by : g == 4 ? curl : aux;
    row_c2r<RF>(dst, th.lane, v, tb, [&](int k) -> Cx<T> {
      switch (g) {
        case 0: return ikmul(__ldg(kx + k), ldg(a.Xux + ro + k));  // d_ux_dx: c2r_x(i kx X(ux))/Nx
        case 1: return ldg(a.Hduy + ro + k);
        case 2: return ldg(a.Hbx + ro + k);
        case 3: return ldg(a.Hby + ro + k);
        case 4: return ikmul(__ldg(kx + k), ldg(a.Hby + ro + k));  // d_By_dx (corrected)
        default: return ldg(a.Hikybx + ro + k);                     // d_Bx_dy (corrected)
      }
    }, sync);
    sync();
    const T sc = g == 0 ? a.inv_nx : (T)1;
    fft_emit<RF>(th.lane, v, [&](int, int n, Cx<T> z) {
      dst[n] = g == 0 ? cx<T>(z.x * sc, z.y * sc) : cx<T>(normalise(z.x, tb), normalise(z.y, tb));
    });
  }
  __syncthreads();
  // phase 2: curl B                                                      (:186-190)
  for (int n = th.g * NTR + th.lane; n < M; n += G * NTR) {
    if (!FIX) {
      // d_Bx_dy = d_ux_dx/(NxNy), d_By_dx = d_uy_dy/(NxNy)   (reference defect)
      // (/ NxNy: an exact multiply when NxNy is a power of two)
      const Cx<T> p = dux[n], q = duy[n];
      curl[n] = cx<T>(normalise(q.x, tb) - normalise(p.x, tb), normalise(q.y, tb) - normalise(p.y, tb));
    } else {
      const Cx<T> p = curl[n], q = aux[n];
      curl[n] = cx<T>(p.x - q.x, p.y - q.y);
    }
  }
  __syncthreads();
  // phase 3: Energy_x -= eta By curl, Energy_y += eta Bx curl, E_Visc = (div u)^2   (:204-209)
  const T eta = a.eta;
  if (th.g < 3) {
    const int g = th.g;
    row_r2c_begin<RF>(th.lane, v, tb, [&](int n) -> Cx<T> {
      if (g == 0) {
        const Cx<T> b = by[n], c = curl[n];
        return cx<T>(-(eta * b.x * c.x), -(eta * b.y * c.y));
      }
      if (g == 1) {
        const Cx<T> b = bx[n], c = curl[n];
        return cx<T>(eta * b.x * c.x, eta * b.y * c.y);
      }
      const Cx<T> p = dux[n], q = duy[n];
      const T d0 = p.x + q.x, d1 = p.y + q.y;
      return cx<T>(d0 * d0, d1 * d1);
    });
  }
  __syncthreads();  // inputs gathered: arrays 0..2 become exchange buffers
  if (th.g < 3) {
    const int g = th.g;
    Cx<T>* xo = (g == 0 ? a.Xex2 : g == 1 ? a.Xey2 : a.Xev) + ro;
    row_r2c_finish<RF>(base + g * ARR, th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
  }
}
template <class T, int M, int P, int FIX>
__global__ void __launch_bounds__(TARA_ROW_LB((FIX ? 6 : 4) * (M / P)),
                                  TARA_MINB(TARA_ROW_LB((FIX ? 6 : 4) * (M / P))))
k_row_com2(const RowCom2Args<T> a) {
  row_com2_rows<T, M, P, FIX>(a, blockIdx.x * a.rb);
}


template <class T> struct ColFwdComArgs {
  Tables<T> tb;
  const Cx<T>* X[13];
  const Cx<T>* in[6];  // stage input (the state the RHS is evaluated at)
  T mu, eta;
  int forcing;
  int closure;            // add the subgrid stress / EMF spectra of clos[]
  const Cx<T>* clos[4];   // tau_xx, tau_xy, tau_yy, EMF
  // fuse: also y-invert the next RHS input of field f into hnext[f] (and
  // i ky Bx into hikybx when set), the next RHS's column-inverse pass
  int fuse;
  Cx<T>* hnext[6];
  Cx<T>* hikybx;
  StepArgs<T> step;
};

// Whether the column-forward pass keeps the derivative it assembles in a
// second shared tile of CB*L values instead of registers.  Only CTAs of 512
// or more threads (128 registers per thread, one CTA per SM, so the tile
// costs no occupancy) where both tiles fit in 160 KB, and only where it was
// measured no slower (graph-replayed launches, same box): FP64 1024-point
// columns 118.7 against 118.6 us (spills 408/516 -> 64/72 bytes per thread,
// 288 against 307 MB of DRAM traffic per launch), FP32 2048 313 against 321
// us, FP32 4096 1650 against 1698 us.  FP64 2048-point columns were slower
// with it (594 against 561 us) and keep the derivative in registers.
template <class T, int L, int CB, int P> __host__ __device__ constexpr bool col_fwd_com_ds() {
  return CB * L / P >= 512 && 2 * (size_t)CB * L * sizeof(Cx<T>) <= 160 * 1024 &&
         (sizeof(T) == 8 ? L <= 1024 : L >= 2048);
}
// dynamic shared memory of the column-forward pass (elements)
template <class T, int L, int CB, int P> constexpr size_t col_fwd_com_smem_elems() {
  return (size_t)FFTB<L, CB, P>::SMEM_ELEMS + (col_fwd_com_ds<T, L, CB, P>() ? (size_t)CB * L : 0);
}

template <class T, int L, int CB, int P>
__global__ void __launch_bounds__(CB * L / P, TARA_MINB(CB * L / P)) k_col_fwd_com(const ColFwdComArgs<T> a) {
  using F = FFTB<L, CB, P>;
  constexpr int RL = F::Pl::R[F::S - 1];
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  const int f = blockIdx.y;
  const int c0 = blockIdx.x * CB;
#include "col_fwd_com_body.inc"
}

// The same pass as a device function: output field f, kx columns c0 .., by
// the CB*L/P threads of the calling CTA (persistent ensemble kernels).
template <class T, int L, int CB, int P>
__device__ __forceinline__ void col_fwd_com_tile(const ColFwdComArgs<T>& a, int f, int c0) {
  using F = FFTB<L, CB, P>;
  constexpr int RL = F::Pl::R[F::S - 1];
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
#include "col_fwd_com_body.inc"
}

template <int L, class T>
inline void col_fwd_com_dispatch(const ColFwdComArgs<T>& a, cudaStream_t st) {
  constexpr int CB = ColFwdComCfg<T, L>::CB, P = ColFwdComCfg<T, L>::P;
  auto kern = k_col_fwd_com<T, L, CB, P>;
  const size_t smem = col_fwd_com_smem_elems<T, L, CB, P>() * sizeof(Cx<T>);
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
  constexpr bool LOW = (size_t)8 * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>) > 200 * 1024;
  const size_t per_row = (size_t)(LOW ? 6 : 8) * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>);
  a.rb = row_cta_rows(8 * NTR, per_row, Ny);
  auto kern = k_row_com1<T, M, P, LOW>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, 8 * NTR * a.rb, smem, st>>>(a);
}
template <int Nx, class T>
static void launch_row_force(const RowForceArgs<T>& a0, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  RowForceArgs<T> a = a0;
  const size_t per_row = (size_t)3 * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>);
  a.rb = row_cta_rows(2 * NTR, per_row, Ny);
  auto kern = k_row_force<T, M, P>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, 2 * NTR * a.rb, smem, st>>>(a);
}
template <int FIX, int Nx, class T>
static void launch_row_com2_t(const RowCom2Args<T>& a0, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  constexpr int G = FIX ? 6 : 4, NA = FIX ? 6 : 5;
  RowCom2Args<T> a = a0;
  const size_t per_row = (size_t)NA * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>);
  a.rb = row_cta_rows(G * NTR, per_row, Ny);
  auto kern = k_row_com2<T, M, P, FIX>;
  const size_t smem = per_row * a.rb;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<Ny / a.rb, G * NTR * a.rb, smem, st>>>(a);
}
template <int Nx, class T>
static void launch_row_com2(const RowCom2Args<T>& a, int Ny, int fix, cudaStream_t st) {
  if (fix) launch_row_com2_t<1, Nx>(a, Ny, st);
  else launch_row_com2_t<0, Nx>(a, Ny, st);
}

template <class T>
int com_rhs(const Grid<T>& g, ComWork<T>& w, const ComParamsT<T>& p, Cx<T>* const in[6],
            const StepArgs<T>& step, cudaStream_t st) {
  if ((size_t)6 * (g.Nx / 2 + g.Nx / 32 + 1) * sizeof(Cx<T>) > 220 * 1024 || 8 * (g.Nx / 2) / 16 > 1024) {
    set_error("MHD row pass does not fit in shared memory at this Nx and precision");
    return TARA_EUNSUPPORTED;
  }
  const int forcing = p.A != (T)0;
  if (!p.skip_inv) {  // else w.H already holds the y-inverse of `in` (previous column pass)
    ColInvArgs<T> ci{};
    ci.tb = g.tb;
    for (int q = 0; q < 6; q++) ci.job[q] = ColInvJob<T>{in[q], w.H[q], MUL_ONE};
    int nj = 6;
    if (p.fix_curlB) ci.job[nj++] = ColInvJob<T>{in[4], w.H[HIKYBX], MUL_IKY};
    prof_mark(g.prof, st, KK_COL_INV);
    run_col_inv(ci, nj, st);
  }

  RowCom1Args<T> r1{};
  r1.tb = g.tb;
  for (int q = 0; q < 6; q++) r1.H[q] = w.H[q];
  for (int q = 0; q < 11; q++) r1.X[q] = w.X[q];
  r1.cs2 = p.cs2;
  if (p.cfl.dev) r1.cfl = CflRow{&p.cfl.dev->lam, p.cfl.idx, p.cfl.idy, p.cfl.cs2};
  prof_mark(g.prof, st, KK_ROW_COM1);
  TARA_DISPATCH_LEN(g.Nx, launch_row_com1, r1, g.Ny, st)
  if (p.cfl.dev) {  // dt of this step, before any stepper update reads it
    prof_mark(g.prof, st, KK_CFL);
    TARA_TRY(launch_cfl_update(p.cfl, g.tb.status, st));
  }
  if (forcing) {
    RowForceArgs<T> rf{};
    rf.tb = g.tb;
    rf.Hrho = w.H[HRHO];
    rf.Xfx = w.X[XFX];
    rf.Xfy = w.X[XFY];
    rf.A = p.A;
    rf.kf = p.kf;
    rf.dx = (T)(g.Lx / g.Nx);
    rf.dy = (T)(g.Ly / g.Ny);
    prof_mark(g.prof, st, KK_ROW_FORCE);
    TARA_DISPATCH_LEN(g.Nx, launch_row_force, rf, g.Ny, st)
  }

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
  r2.Xex2 = w.X[XEX2];
  r2.Xey2 = w.X[XEY2];
  r2.Xev = w.X[XEV];
  r2.eta = p.eta;
  r2.inv_nx = (T)(1.0 / g.Nx);
  prof_mark(g.prof, st, KK_ROW_COM2);
  TARA_DISPATCH_LEN(g.Nx, launch_row_com2, r2, g.Ny, p.fix_curlB, st)

  ColFwdComArgs<T> cf{};
  cf.tb = g.tb;
  for (int q = 0; q < 13; q++) cf.X[q] = w.X[q];
  for (int q = 0; q < 6; q++) cf.in[q] = in[q];
  cf.mu = p.mu;
  cf.eta = p.eta;
  cf.forcing = forcing;
  cf.closure = p.closure;
  for (int q = 0; q < 4; q++) cf.clos[q] = p.clos[q];
  cf.fuse = p.fuse_inv && step.mode != STEP_RHS;
  for (int q = 0; q < 6; q++) cf.hnext[q] = w.H[q];
  cf.hikybx = p.fix_curlB ? w.H[HIKYBX] : nullptr;
  cf.step = step;
  prof_mark(g.prof, st, KK_COL_FWD_COM);
  TARA_DISPATCH_LEN(g.Ny, col_fwd_com_dispatch, cf, st)
  prof_mark(g.prof, st, KK_END);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

}  // namespace tara
