// Tracer particles of the incompressible vorticity driver
// (src/main2csh.f95:93-96, 187-268): after every step the velocity of the new
// state is formed in real space and every particle moves one forward-Euler
// step with the velocity interpolated bilinearly in its grid cell.
//
// Interpolation (reference :189-242): m = aint(xp/dx) + 1, n = aint(yp/dy) + 1,
// x(i) = (i-1) dx, h = 1/(dx dy),
//   v = u(m,n)(x1-xp)(y1-yp)h + u(m+1,n)(xp-x0)(y1-yp)h
//     + u(m,n+1)(x1-xp)(yp-y0)h + u(m+1,n+1)(xp-x0)(yp-y0)h
// with x0 = x(m), x1 = x(m+1) or Lx in the last column (y likewise), each
// product and sum rounded as written (no fused multiply-add).  In the last
// column / row the reference reads u(Nx+1,n) / u(m,Ny+1), past its (Nx,Ny)
// arrays; here the index wraps to column / row 1, the periodic neighbour.
// Move (:244-256): xp = xp + vxp dt; xp = xp - int(xp/Lx) Lx; if (xp <= 0)
// xp = xp + Lx (likewise y), so positions stay in (0, Lx] x (0, Ly].
#include "tracers.cuh"
#include "xform.cuh"

namespace tara {

namespace {

// velocity spectra from the vorticity: psi = omega/(k^2 + lam) (0 at k = 0),
// u_k = i ky psi, v_k = -i kx psi   (reference :122-148)
template <class T>
__global__ void k_velocity_spec(Tables<T> tb, const Cx<T>* __restrict__ w, T lam, Cx<T>* ux, Cx<T>* uy) {
  const size_t n = (size_t)tb.Ny * tb.Nh;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % tb.Nh), j = (int)(q / tb.Nh);
    const size_t o = (size_t)j * tb.ld + i;
    const T kx = tb.kx[i], ky = tb.ky[j];
    const Cx<T> psi = apply_psi_mul(MUL_PSI, lam, kx, ky, i == 0 && j == 0, w[o]);
    ux[o] = ikmul(ky, psi);
    uy[o] = -ikmul(kx, psi);
  }
}

struct TracerGeom {
  int Nx, Ny, np, move;
  double Lx, Ly, dx, dy, h, dt;
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// p into (0, L] as the move does; false for a non-finite or huge p
__device__ __forceinline__ bool wrap_into(double& p, double L) {
  if (p > 0.0 && p <= L) return true;
  const double q = p / L;
  if (!(fabs(q) < 1e9)) return false;
  p = sub(p, mul((double)(long long)q, L));
  if (p <= 0.0) p = add(p, L);
  return p > 0.0 && p <= L;
}
// one particle coordinate p in (0, L]: cell index (0-based, wrapped), near /
// far node coordinates
__device__ __forceinline__ void cell(double p, double d, double L, int N, int& i0, int& i1, double& p0,
                                     double& p1) {
  int m = (int)trunc(p / d) + 1;  // aint(p/d) + 1, 1-based; N + 1 only at p = L
  m = m < 1 ? 1 : (m > N + 1 ? N + 1 : m);
  p0 = (double)(m - 1) * d;              // x(m)
  p1 = m == N ? L : (double)m * d;       // x(m+1), Lx in the last column
  i0 = (m - 1) % N;
  i1 = m % N;
}

template <class T>
__global__ void k_tracers(TracerGeom g, const T* __restrict__ ux, const T* __restrict__ uy, double* xp, double* yp,
                          double* vxp, double* vyp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= g.np) return;
  double x = xp[k], y = yp[k];
  if (!wrap_into(x, g.Lx) || !wrap_into(y, g.Ly)) {  // not a position in the box
    vxp[k] = vyp[k] = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  int i0, i1, j0, j1;
  double x0, x1, y0, y1;
  cell(x, g.dx, g.Lx, g.Nx, i0, i1, x0, x1);
  cell(y, g.dy, g.Ly, g.Ny, j0, j1, y0, y1);
  const double ax = sub(x1, x), bx = sub(x, x0), ay = sub(y1, y), by = sub(y, y0);
  auto interp = [&](const T* u) {
    const double u00 = (double)u[(size_t)j0 * g.Nx + i0], u10 = (double)u[(size_t)j0 * g.Nx + i1];
    const double u01 = (double)u[(size_t)j1 * g.Nx + i0], u11 = (double)u[(size_t)j1 * g.Nx + i1];
    double v = mul(mul(mul(u00, ax), ay), g.h);
    v = add(v, mul(mul(mul(u10, bx), ay), g.h));
    v = add(v, mul(mul(mul(u01, ax), by), g.h));
    return add(v, mul(mul(mul(u11, bx), by), g.h));
  };
  const double vx = interp(ux), vy = interp(uy);
  vxp[k] = vx;
  vyp[k] = vy;
  if (!g.move) return;
  double xn = add(x, mul(vx, g.dt)), yn = add(y, mul(vy, g.dt));
  xn = sub(xn, mul((double)(int)(xn / g.Lx), g.Lx));
  if (xn <= 0.0) xn = add(xn, g.Lx);
  yn = sub(yn, mul((double)(int)(yn / g.Ly), g.Ly));
  if (yn <= 0.0) yn = add(yn, g.Ly);
  xp[k] = xn;
  yp[k] = yn;
}

}  // namespace

template <class T>
int tracer_velocity_real(const Grid<T>& g, const Cx<T>* omega, T lam, T* ux, T* uy, Cx<T>* const* work,
                         cudaStream_t st) {
  k_velocity_spec<T><<<592, 256, 0, st>>>(g.tb, omega, lam, work[0], work[1]);
  TARA_CUDA_TRY(cudaGetLastError());
  const Cx<T>* spec[2] = {work[0], work[1]};
  T* real[2] = {ux, uy};
  Cx<T>* w2[2] = {work[2], work[3]};
  return c2r_fields(g, 2, spec, real, w2, true, st);
}

template <class T>
int tracers_update(const Grid<T>& g, const T* ux, const T* uy, int np, double* xp, double* yp, double* vxp,
                   double* vyp, double dt, bool move, cudaStream_t st) {
  if (np <= 0) return TARA_OK;
  TracerGeom t{};
  t.Nx = g.Nx;
  t.Ny = g.Ny;
  t.np = np;
  t.move = move ? 1 : 0;
  t.Lx = g.Lx;
  t.Ly = g.Ly;
  t.dx = g.Lx / (double)g.Nx;
  t.dy = g.Ly / (double)g.Ny;
  t.h = 1.0 / (t.dx * t.dy);
  t.dt = dt;
  k_tracers<T><<<(np + 255) / 256, 256, 0, st>>>(t, ux, uy, xp, yp, vxp, vyp);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

template int tracer_velocity_real<double>(const Grid<double>&, const Cx<double>*, double, double*, double*,
                                          Cx<double>* const*, cudaStream_t);
template int tracer_velocity_real<float>(const Grid<float>&, const Cx<float>*, float, float*, float*,
                                         Cx<float>* const*, cudaStream_t);
template int tracers_update<double>(const Grid<double>&, const double*, const double*, int, double*, double*,
                                    double*, double*, double, bool, cudaStream_t);
template int tracers_update<float>(const Grid<float>&, const float*, const float*, int, double*, double*, double*,
                                   double*, double, bool, cudaStream_t);

}  // namespace tara
