// Model RHS launchers.  Each launches the kernels of one right-hand-side
// evaluation on `st` and hands every derivative value to the stepper
// epilogue described by StepArgs (write it out, AB2, Euler or an RK4 stage).
#pragma once
#include "plan.h"
#include "kernels.cuh"

namespace tara {

// ---- CFL control and state checks (guard.cu) ----
enum : int { CFL_OFF = TARA_CFL_OFF, CFL_CHECK = TARA_CFL_CHECK, CFL_ADAPT = TARA_CFL_ADAPT };
// CFL settings of one RHS evaluation: dev == nullptr, or a RHS that is not
// the first of its step, computes no rate.
struct CflCfg {
  CflDev* dev;
  int mode;
  double number;    // CFL number C: dt_cfl = C / max over the grid of the rate
  double dt;        // configured dt (the largest step)
  double idx, idy;  // 1/dx, 1/dy
  double cs2;       // squared sound speed
};
// dt of this step from the folded rate (one thread): writes dev->scale, ->dt,
// advances ->t, clears ->lam; TARA_ECFL / TARA_ENAN into *status.
int launch_cfl_update(const CflCfg& c, int* status, cudaStream_t st);
// TARA_ENAN into tb.status when a value of the nf fields is not finite.
template <class T>
int launch_finite_check(const Grid<T>& g, Cx<T>* const* f, int nf, cudaStream_t st);

// ---- compressible isothermal hydro, src/derive2coh.f95 ----
template <class T> struct CohParamsT {
  T mux, muy, cs2;
  CflCfg cfl;
};
template <class T> struct CohWork {
  FieldPool<T> H;  // 8 half-real fields: n, iky n, ux, iky ux, ky2 ux, uy, iky uy, ky2 uy
  FieldPool<T> X;  // 3 x-transformed rows: NLn, momentum-x, momentum-y
  int alloc(const Grid<T>& g, cudaStream_t st) {
    int s = H.alloc(g, 8, st);
    if (s) return s;
    return X.alloc(g, 3, st);
  }
  void release() { H.release(); X.release(); }
};
template <class T>
int coh_rhs(const Grid<T>& g, CohWork<T>& w, const CohParamsT<T>& p, Cx<T>* const in[3],
            const StepArgs<T>& step, cudaStream_t st);
constexpr int kCohLaunches = 3;

// ---- compressible MHD, src/derive2com.f95 ----
// closure != 0: the spectra of a subgrid stress (xx, xy, yy) and EMF in
// clos[] are added to the momentum and induction fluxes (learned closure).
// skip_inv: the half-real fields H already hold the y-inverse of the RHS
// input (written by the previous column-forward pass); fuse_inv: the
// column-forward pass writes H for the next RHS input (stepping modes).
template <class T> struct ComParamsT {
  T mu, eta, cs2, kf, A;
  int fix_curlB;
  int closure;
  const Cx<T>* clos[4];
  int skip_inv, fuse_inv;
  CflCfg cfl;
};
template <class T> struct ComWork {
  FieldPool<T> H;  // half-real: rho, rho_ux, rho_uy, E, Bx, By, d(uy)/dy, [iky Bx, ikx By]
  // x-transformed rows: ux, uy, Mxx, Mxy, Myy, Mag, Ex, Ey, EV, Fx, Fy, and the
  // curl-B parts of Ex, Ey
  FieldPool<T> X;
  int alloc(const Grid<T>& g, cudaStream_t st) {
    int s = H.alloc(g, 9, st);
    if (s) return s;
    return X.alloc(g, 13, st);
  }
  void release() { H.release(); X.release(); }
};
template <class T>
int com_rhs(const Grid<T>& g, ComWork<T>& w, const ComParamsT<T>& p, Cx<T>* const in[6],
            const StepArgs<T>& step, cudaStream_t st);
// per RHS evaluation while stepping: the column-inverse pass of the next RHS
// is fused into the column-forward pass (one more launch where a run starts)
constexpr int kComLaunches = 4;

// ---- incompressible (screened) vorticity, src/derive2csh.f95, src/derive2css.f95 ----
template <class T> struct VortParamsT { T nu, alpha, lambda; int screened; };
template <class T> struct VortWork {
  FieldPool<T> H;  // ux, uy, d omega/dx, d omega/dy (half-real)
  FieldPool<T> X;  // u.grad omega (x-transformed)
  int alloc(const Grid<T>& g, cudaStream_t st) {
    int s = H.alloc(g, 4, st);
    if (s) return s;
    return X.alloc(g, 1, st);
  }
  void release() { H.release(); X.release(); }
};
template <class T>
int vort_rhs(const Grid<T>& g, VortWork<T>& w, const VortParamsT<T>& p, Cx<T>* const in[1],
             const StepArgs<T>& step, cudaStream_t st);
constexpr int kVortLaunches = 3;

}  // namespace tara
