/* CPU oracle: C restatement of the reference's RHS + time-step path.
 *
 * TEST INFRASTRUCTURE ONLY -- see tara_oracle.h for status and conventions.
 * Each routine cites the reference lines it follows.  Loop bodies keep the
 * reference's operation order so that rounding matches as closely as C allows
 * (compiled without FMA contraction, -ffp-contract=off).  The FFTs are the
 * reference's FFTW 3.3.9 with FFTW_ESTIMATE; the Fortran call
 * dfftw_plan_dft_c2r_2d(p,Nx,Ny,...) is fftw_plan_dft_c2r_2d(Ny,Nx,...) in C
 * (lib/fftw/api/f77funcs.h:206-210, 300-304).
 */
#include "tara_oracle.h"
#include <fftw3.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define IX(i, j, ld) ((size_t)(i) + (size_t)(ld) * (size_t)(j))

static int g_threads = 0;
void ora_set_threads(int n) { g_threads = n; }
int ora_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}
#define OMP_FOR _Pragma("omp parallel for num_threads(ora_get_threads()) schedule(static)")

static void *xmalloc(size_t n) {
  void *p = fftw_malloc(n ? n : 16);
  if (!p) abort();
  return p;
}
static ocplx *cnew(int Nh, int Ny) { return (ocplx *)xmalloc(sizeof(ocplx) * (size_t)Nh * Ny); }
static double *rnew(int Nx, int Ny) { return (double *)xmalloc(sizeof(double) * (size_t)Nx * Ny); }

/* c2r destroys its input (FFTW default for c2r), hence the *_dum copies in the
 * reference (src/derive2coh.f95:43-45); this helper copies internally. */
void ora_c2r_2d(int Nx, int Ny, const ocplx *in, double *out) {
  int Nh = Nx / 2 + 1;
  ocplx *tmp = cnew(Nh, Ny);
  memcpy(tmp, in, sizeof(ocplx) * (size_t)Nh * Ny);
  fftw_plan p = fftw_plan_dft_c2r_2d(Ny, Nx, (fftw_complex *)tmp, out, FFTW_ESTIMATE);
  fftw_execute(p);
  fftw_destroy_plan(p);
  fftw_free(tmp);
}
/* c2r that may destroy `in` (used where the reference passes a scratch array) */
static void c2r_destroy(int Nx, int Ny, ocplx *in, double *out) {
  fftw_plan p = fftw_plan_dft_c2r_2d(Ny, Nx, (fftw_complex *)in, out, FFTW_ESTIMATE);
  fftw_execute(p);
  fftw_destroy_plan(p);
}
void ora_r2c_2d(int Nx, int Ny, const double *in, ocplx *out) {
  /* r2c out-of-place preserves its input with FFTW_ESTIMATE */
  fftw_plan p = fftw_plan_dft_r2c_2d(Ny, Nx, (double *)in, (fftw_complex *)out, FFTW_ESTIMATE);
  fftw_execute(p);
  fftw_destroy_plan(p);
}

/* kx = 2*pi*(i-1)/Lx ; ky = 2*pi*(j-1)/Ly for j <= Ny/2, 2*pi*((j-1)-Ny)/Ly above
 * (src/derive2coh.f95:60-61, 74-75).  i, j are 0-based here. */
static inline double kx_of(int i, double pi, double Lx) { return 2.0 * pi * (double)i / Lx; }
static inline double ky_of(int j, int Ny, double pi, double Ly) {
  return (j < Ny / 2) ? 2.0 * pi * (double)j / Ly : 2.0 * pi * (double)(j - Ny) / Ly;
}
/* circular 2/3 rule: zero when sqrt(kx^2+ky^2) >= ((Nx+Ny)/2)/3 (src/derive2coh.f95:212) */
static inline int masked(double kx, double ky, int Nx, int Ny) {
  return sqrt(kx * kx + ky * ky) >= ((double)(Nx + Ny) / 2.0) / 3.0 + 0;
}
/* (0,1)*k*z evaluated as ((0,1)*k)*z with Fortran complex-multiply rules */
static inline ocplx ik_mul(double k, ocplx z) {
  double a = creal(z), b = cimag(z);
  return CMPLX(0.0 * a - k * b, 0.0 * b + k * a);
}
static inline ocplx rmul(double r, ocplx z) { return CMPLX(r * creal(z), r * cimag(z)); }

/* ======================================================================= */
/* derive2coh: src/derive2coh.f95:6-265                                     */
/* ======================================================================= */
void ora_derive2coh(int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                    const ocplx *nk, const ocplx *ukx, const ocplx *uky,
                    ocplx *dn_dt_new, ocplx *dux_dt_new, ocplx *duy_dt_new) {
  (void)time;
  const double Lx = P->Lx, Ly = P->Ly, mux = P->mux, muy = P->muy, CS = P->CS;
  const size_t nc = (size_t)Nh * Ny;
  enum { C_NKD, C_UXD, C_UYD, C_IKXN, C_IKYN, C_IKXUX, C_IKYUX, C_IKXUY, C_IKYUY,
         C_KX2UX, C_KY2UX, C_KX2UY, C_KY2UY,
         C_PKX, C_PKY, C_VXX, C_VXY, C_VYX, C_VYY, C_NLN, C_NLX, C_NLY, NC_ };
  enum { R_N, R_UX, R_UY, R_DNDX, R_DNDY, R_DUXDX, R_DUXDY, R_DUYDX, R_DUYDY,
         R_D2UXDX2, R_D2UXDY2, R_D2UYDX2, R_D2UYDY2,
         R_PX, R_PY, R_VXX, R_VXY, R_VYX, R_VYY, R_NLN, R_NLX, R_NLY, NR_ };
  ocplx *c[NC_];
  double *r[NR_];
  for (int q = 0; q < NC_; q++) c[q] = cnew(Nh, Ny);
  for (int q = 0; q < NR_; q++) r[q] = rnew(Nx, Ny);

  /* :32-50 backups for FFTW */
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      size_t k = IX(i, j, Nh);
      c[C_NKD][k] = nk[k];
      c[C_UXD][k] = ukx[k];
      c[C_UYD][k] = uky[k];
    }
  /* :54-90 spectral derivatives */
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      size_t k = IX(i, j, Nh);
      c[C_IKXN][k] = ik_mul(kx, nk[k]);
      c[C_IKYN][k] = ik_mul(ky, nk[k]);
      c[C_IKXUX][k] = ik_mul(kx, ukx[k]);
      c[C_IKYUX][k] = ik_mul(ky, ukx[k]);
      c[C_IKXUY][k] = ik_mul(kx, uky[k]);
      c[C_IKYUY][k] = ik_mul(ky, uky[k]);
      c[C_KX2UX][k] = rmul(kx * kx, ukx[k]);
      c[C_KY2UX][k] = rmul(ky * ky, ukx[k]);
      c[C_KX2UY][k] = rmul(kx * kx, uky[k]);
      c[C_KY2UY][k] = rmul(ky * ky, uky[k]);
    }
  /* :92-129 thirteen c2r */
  static const int c2r_src[13] = {C_NKD, C_UXD, C_UYD, C_IKXN, C_IKYN, C_IKXUX, C_IKYUX,
                                  C_IKXUY, C_IKYUY, C_KX2UX, C_KY2UX, C_KX2UY, C_KY2UY};
  for (int q = 0; q < 13; q++) c2r_destroy(Nx, Ny, c[c2r_src[q]], r[q]);

  /* :131-170 real space */
  const double NN = (double)Nx * (double)Ny;
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nx; i++) {
      size_t k = IX(i, j, Nx);
      for (int q = 0; q < 13; q++) r[q][k] = r[q][k] / NN;
      double n = r[R_N][k];
      r[R_VXX][k] = r[R_D2UXDX2][k] / n;
      r[R_VXY][k] = r[R_D2UXDY2][k] / n;
      r[R_VYX][k] = r[R_D2UYDX2][k] / n;
      r[R_VYY][k] = r[R_D2UYDY2][k] / n;
      r[R_PX][k] = r[R_DNDX][k] / n;
      r[R_PY][k] = r[R_DNDY][k] / n;
      r[R_NLN][k] = r[R_UX][k] * r[R_DNDX][k] + r[R_UY][k] * r[R_DNDY][k] +
                    n * (r[R_DUXDX][k] + r[R_DUYDY][k]);
      r[R_NLX][k] = r[R_UX][k] * r[R_DUXDX][k] + r[R_UY][k] * r[R_DUXDY][k];
      r[R_NLY][k] = r[R_UX][k] * r[R_DUYDX][k] + r[R_UY][k] * r[R_DUYDY][k];
    }
  /* :172-197 nine r2c */
  ora_r2c_2d(Nx, Ny, r[R_PX], c[C_PKX]);
  ora_r2c_2d(Nx, Ny, r[R_PY], c[C_PKY]);
  ora_r2c_2d(Nx, Ny, r[R_VXX], c[C_VXX]);
  ora_r2c_2d(Nx, Ny, r[R_VXY], c[C_VXY]);
  ora_r2c_2d(Nx, Ny, r[R_VYX], c[C_VYX]);
  ora_r2c_2d(Nx, Ny, r[R_VYY], c[C_VYY]);
  ora_r2c_2d(Nx, Ny, r[R_NLN], c[C_NLN]);
  ora_r2c_2d(Nx, Ny, r[R_NLX], c[C_NLX]);
  ora_r2c_2d(Nx, Ny, r[R_NLY], c[C_NLY]);

  /* :204-261 dealias, then assemble */
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      size_t k = IX(i, j, Nh);
      if (masked(kx, ky, Nx, Ny)) {
        c[C_NLN][k] = 0; c[C_NLX][k] = 0; c[C_NLY][k] = 0;
        c[C_PKX][k] = 0; c[C_PKY][k] = 0;
        c[C_VXX][k] = 0; c[C_VXY][k] = 0; c[C_VYX][k] = 0; c[C_VYY][k] = 0;
      }
      ocplx nlx = c[C_NLX][k] + (rmul(mux, c[C_VXX][k]) + rmul(muy, c[C_VXY][k])) + rmul(CS * CS, c[C_PKX][k]);
      ocplx nly = c[C_NLY][k] + (rmul(mux, c[C_VYX][k]) + rmul(muy, c[C_VYY][k])) + rmul(CS * CS, c[C_PKY][k]);
      dn_dt_new[k] = -c[C_NLN][k];
      dux_dt_new[k] = -nlx;
      duy_dt_new[k] = -nly;
    }
  for (int q = 0; q < NC_; q++) fftw_free(c[q]);
  for (int q = 0; q < NR_; q++) fftw_free(r[q]);
  (void)nc;
}

/* ab2coh: src/ab2coh.f95:19-27 */
void ora_ab2coh(int Nx, int Ny, int Nh, const ora_coh_params *P,
                const ocplx *nk, const ocplx *ukx, const ocplx *uky,
                ocplx *nk_new, ocplx *ukx_new, ocplx *uky_new,
                const ocplx *dn_dt_old, const ocplx *dux_dt_old, const ocplx *duy_dt_old,
                const ocplx *dn_dt_new, const ocplx *dux_dt_new, const ocplx *duy_dt_new) {
  (void)Nx;
  const double dt = P->dt;
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      size_t k = IX(i, j, Nh);
      nk_new[k] = nk[k] + rmul(dt, rmul(3.0 / 2.0, dn_dt_new[k]) - rmul(1.0 / 2.0, dn_dt_old[k]));
      ukx_new[k] = ukx[k] + rmul(dt, rmul(3.0 / 2.0, dux_dt_new[k]) - rmul(1.0 / 2.0, dux_dt_old[k]));
      uky_new[k] = uky[k] + rmul(dt, rmul(3.0 / 2.0, duy_dt_new[k]) - rmul(1.0 / 2.0, duy_dt_old[k]));
    }
}

/* euler2coh: src/euler2coh.f95:15-24 */
void ora_euler2coh(int Nx, int Ny, int Nh, const ora_coh_params *P,
                   const ocplx *nk, const ocplx *ukx, const ocplx *uky,
                   ocplx *nk_new, ocplx *ukx_new, ocplx *uky_new,
                   const ocplx *dn_dt, const ocplx *dux_dt, const ocplx *duy_dt) {
  (void)Nx;
  const double dt = P->dt;
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      size_t k = IX(i, j, Nh);
      nk_new[k] = nk[k] + rmul(dt, dn_dt[k]);
      ukx_new[k] = ukx[k] + rmul(dt, dux_dt[k]);
      uky_new[k] = uky[k] + rmul(dt, duy_dt[k]);
    }
}

/* pc_nk2coh / pc_ukx2coh / pc_uky2coh: src/pcnk2coh.f95:20-34 (and the ukx/uky
 * copies).  The corrector reads the unchanged argument derivative, so the
 * result is (predict + correct)*dt/2 with predict == correct; the derive2coh
 * call writes only subroutine-local arrays. */
void ora_pc2coh(int which, int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                const ocplx *nk, const ocplx *ukx, const ocplx *uky, ocplx *out,
                const ocplx *dn_dt, const ocplx *dux_dt, const ocplx *duy_dt) {
  const double dt = P->dt;
  const ocplx *f = which == 0 ? nk : which == 1 ? ukx : uky;
  const ocplx *d = which == 0 ? dn_dt : which == 1 ? dux_dt : duy_dt;
  ocplx *predict = cnew(Nh, Ny), *dum = cnew(Nh, Ny);
  ocplx *l0 = cnew(Nh, Ny), *l1 = cnew(Nh, Ny), *l2 = cnew(Nh, Ny);
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      size_t k = IX(i, j, Nh);
      predict[k] = d[k];
      dum[k] = f[k] + rmul(dt, predict[k]);
    }
  ora_derive2coh(Nx, Ny, Nh, pi, time + dt, P, which == 0 ? dum : nk, which == 1 ? dum : ukx,
                 which == 2 ? dum : uky, l0, l1, l2);
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      size_t k = IX(i, j, Nh);
      ocplx correct = d[k];
      ocplx s = predict[k] + correct;
      out[k] = f[k] + CMPLX(creal(s) * dt / 2.0, cimag(s) * dt / 2.0);
    }
  fftw_free(predict); fftw_free(dum); fftw_free(l0); fftw_free(l1); fftw_free(l2);
}

/* rk4_nk2coh / rk4_ukx2coh / rk4_uky2coh: src/rk4nk2coh.f95:21-56.  Every
 * stage reads the unchanged argument derivative (k1 = k2 = k3 = k4); the three
 * derive2coh calls write only subroutine-local arrays. */
void ora_rk42coh(int which, int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                 const ocplx *nk, const ocplx *ukx, const ocplx *uky, ocplx *out,
                 const ocplx *dn_dt, const ocplx *dux_dt, const ocplx *duy_dt) {
  const double dt = P->dt;
  const ocplx *f = which == 0 ? nk : which == 1 ? ukx : uky;
  const ocplx *d = which == 0 ? dn_dt : which == 1 ? dux_dt : duy_dt;
  ocplx *k1 = cnew(Nh, Ny), *k2 = cnew(Nh, Ny), *k3 = cnew(Nh, Ny), *dum = cnew(Nh, Ny);
  ocplx *l0 = cnew(Nh, Ny), *l1 = cnew(Nh, Ny), *l2 = cnew(Nh, Ny);
  ocplx *ks[3] = {k1, k2, k3};
  for (int s = 0; s < 3; s++) {
    for (int j = 0; j < Ny; j++)
      for (int i = 0; i < Nh; i++) {
        size_t k = IX(i, j, Nh);
        ks[s][k] = d[k];
        ocplx t = ks[s][k];
        dum[k] = f[k] + CMPLX(creal(t) * dt / 2.0, cimag(t) * dt / 2.0);
      }
    ora_derive2coh(Nx, Ny, Nh, pi, time + dt / 2.0, P, which == 0 ? dum : nk, which == 1 ? dum : ukx,
                   which == 2 ? dum : uky, l0, l1, l2);
  }
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      size_t k = IX(i, j, Nh);
      ocplx k4 = d[k];
      ocplx s = k1[k] + rmul(2.0, k2[k]) + rmul(2.0, k3[k]) + k4;
      out[k] = f[k] + rmul(dt / 6.0, s);
    }
  fftw_free(k1); fftw_free(k2); fftw_free(k3); fftw_free(dum);
  fftw_free(l0); fftw_free(l1); fftw_free(l2);
}

/* Classical RK4 of the coupled hydro system (new; no reference counterpart). */
void ora_rk4coh(int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                ocplx *nk, ocplx *ukx, ocplx *uky) {
  const double dt = P->dt;
  const size_t nc = (size_t)Nh * Ny;
  ocplx *u[3] = {nk, ukx, uky};
  ocplx *us[3], *acc[3], *k[3];
  for (int f = 0; f < 3; f++) { us[f] = cnew(Nh, Ny); acc[f] = cnew(Nh, Ny); k[f] = cnew(Nh, Ny); }
  static const double cstage[4] = {0.5, 0.5, 1.0, 0.0};
  static const double wstage[4] = {1.0, 2.0, 2.0, 1.0};
  for (int f = 0; f < 3; f++) memcpy(us[f], u[f], nc * sizeof(ocplx));
  for (int s = 0; s < 4; s++) {
    ora_derive2coh(Nx, Ny, Nh, pi, time + (s == 0 ? 0.0 : cstage[s - 1] * dt), P, us[0], us[1], us[2],
                   k[0], k[1], k[2]);
    for (int f = 0; f < 3; f++)
      for (size_t q = 0; q < nc; q++) {
        ocplx kk = k[f][q];
        if (s == 0) acc[f][q] = u[f][q] + rmul(dt / 6.0, kk);
        else acc[f][q] = acc[f][q] + rmul(wstage[s] * dt / 6.0, kk);
        if (s < 3) us[f][q] = u[f][q] + rmul(cstage[s] * dt, kk);
      }
  }
  for (int f = 0; f < 3; f++) {
    memcpy(u[f], acc[f], nc * sizeof(ocplx));
    fftw_free(us[f]); fftw_free(acc[f]); fftw_free(k[f]);
  }
}

/* ======================================================================= */
/* derive2com: src/derive2com.f95:6-426                                     */
/* ======================================================================= */
void ora_derive2com(int Nx, int Ny, int Nh, double pi, double time, const ora_com_params *P,
                    const ocplx *rho_k, const ocplx *rho_ux_k, const ocplx *rho_uy_k,
                    const ocplx *E_k, const ocplx *Bx_k, const ocplx *By_k,
                    ocplx *d_rho, ocplx *d_rho_ux, ocplx *d_rho_uy,
                    ocplx *d_E, ocplx *d_Bx, ocplx *d_By) {
  (void)time;
  const double Lx = P->Lx, Ly = P->Ly, mu = P->mu, CS = P->CS, eta = P->eta, kf = P->kf, A = P->A;
  enum { rho, rho_ux, rho_uy, E, Bx, By, ux, uy, Fx, Fy, B2, d_ux_dx, d_uy_dy, d_Bx_dy, d_By_dx,
         curl_B, Pr, Mx1, Mx2, My1, My2, Ex, Ey, EV, Magx, Magy, NR_ };
  enum { ux_k, uy_k, Fx_k, Fy_k, ikx_ux, iky_uy, iky_Bx, ikx_By, Mx1k, Mx2k, My1k, My2k, Exk, Eyk,
         EVk, Magxk, Magyk, dum, NC_ };
  double *r[NR_];
  ocplx *c[NC_];
  for (int q = 0; q < NR_; q++) r[q] = rnew(Nx, Ny);
  for (int q = 0; q < NC_; q++) c[q] = cnew(Nh, Ny);
  const size_t nc = (size_t)Nh * Ny;
  const double NN = (double)Nx * (double)Ny;

  /* :52-86 backups + six c2r */
  const ocplx *st[6] = {rho_k, rho_ux_k, rho_uy_k, E_k, Bx_k, By_k};
  for (int f = 0; f < 6; f++) {
    memcpy(c[dum], st[f], nc * sizeof(ocplx));
    c2r_destroy(Nx, Ny, c[dum], r[rho + f]);
  }
  /* :88-119 (forcing on the grid x_i=(i-1)Lx/Nx, y_j=(j-1)Ly/Ny) */
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nx; i++) {
      size_t k = IX(i, j, Nx);
      double x = (double)i * (Lx / (double)Nx), y = (double)j * (Ly / (double)Ny);
      r[rho][k] = r[rho][k] / NN;
      r[rho_ux][k] = r[rho_ux][k] / NN;
      r[rho_uy][k] = r[rho_uy][k] / NN;
      r[E][k] = r[E][k] / NN;
      r[Bx][k] = r[Bx][k] / NN;
      r[By][k] = r[By][k] / NN;
      r[ux][k] = r[rho_ux][k] / r[rho][k];
      r[uy][k] = r[rho_uy][k] / r[rho][k];
      r[Fx][k] = -r[rho][k] * A * sin(kf * y);
      r[Fy][k] = +r[rho][k] * A * sin(kf * x);
      r[B2][k] = r[Bx][k] * r[Bx][k] + r[By][k] * r[By][k];
    }
  /* :124-134 */
  ora_r2c_2d(Nx, Ny, r[ux], c[ux_k]);
  ora_r2c_2d(Nx, Ny, r[uy], c[uy_k]);
  ora_r2c_2d(Nx, Ny, r[Fx], c[Fx_k]);
  ora_r2c_2d(Nx, Ny, r[Fy], c[Fy_k]);
  /* :142-159 */
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      size_t k = IX(i, j, Nh);
      c[ikx_ux][k] = ik_mul(kx, c[ux_k][k]);
      c[iky_uy][k] = ik_mul(ky, c[uy_k][k]);
      c[iky_Bx][k] = ik_mul(ky, Bx_k[k]);
      c[ikx_By][k] = ik_mul(kx, By_k[k]);
    }
  /* :164-174 */
  c2r_destroy(Nx, Ny, c[ikx_ux], r[d_ux_dx]);
  c2r_destroy(Nx, Ny, c[iky_uy], r[d_uy_dy]);
  c2r_destroy(Nx, Ny, c[iky_Bx], r[d_Bx_dy]);
  c2r_destroy(Nx, Ny, c[ikx_By], r[d_By_dx]);
  /* :180-214 */
  const int fix = P->fix_curlB;
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nx; i++) {
      size_t k = IX(i, j, Nx);
      r[d_ux_dx][k] = r[d_ux_dx][k] / NN;
      r[d_uy_dy][k] = r[d_uy_dy][k] / NN;
      if (!fix) {
        r[d_Bx_dy][k] = r[d_ux_dx][k] / NN;   /* :186 (reference defect) */
        r[d_By_dx][k] = r[d_uy_dy][k] / NN;   /* :187 (reference defect) */
      } else {
        r[d_Bx_dy][k] = r[d_Bx_dy][k] / NN;
        r[d_By_dx][k] = r[d_By_dx][k] / NN;
      }
      r[curl_B][k] = r[d_By_dx][k] - r[d_Bx_dy][k];
      r[Pr][k] = CS * CS * r[rho][k];
      double b2 = r[B2][k];
      r[Mx1][k] = r[rho_ux][k] * r[ux][k] + r[Pr][k] + b2 / 2.0 - r[Bx][k] * r[Bx][k];
      r[Mx2][k] = r[rho_ux][k] * r[uy][k] - r[Bx][k] * r[By][k];
      r[My1][k] = r[rho_ux][k] * r[uy][k] - r[Bx][k] * r[By][k];
      r[My2][k] = r[rho_uy][k] * r[uy][k] + r[Pr][k] + b2 / 2.0 - r[By][k] * r[By][k];
      r[Ex][k] = (r[E][k] + r[Pr][k] + b2 / 2.0) * r[ux][k] - r[ux][k] * r[Bx][k] * r[Bx][k] -
                 r[uy][k] * r[Bx][k] * r[By][k];
      r[Ex][k] = r[Ex][k] - eta * r[By][k] * r[curl_B][k];
      r[Ey][k] = (r[E][k] + r[Pr][k] + b2 / 2.0) * r[uy][k] - r[ux][k] * r[Bx][k] * r[By][k] -
                 r[uy][k] * r[By][k] * r[By][k];
      r[Ey][k] = r[Ey][k] + eta * r[Bx][k] * r[curl_B][k];
      double dv = r[d_ux_dx][k] + r[d_uy_dy][k];
      r[EV][k] = dv * dv;
      r[Magx][k] = r[uy][k] * r[Bx][k] - r[By][k] * r[ux][k];
      r[Magy][k] = r[ux][k] * r[By][k] - r[Bx][k] * r[uy][k];
    }
  /* :220-245 nine r2c */
  ora_r2c_2d(Nx, Ny, r[Mx1], c[Mx1k]);
  ora_r2c_2d(Nx, Ny, r[Mx2], c[Mx2k]);
  ora_r2c_2d(Nx, Ny, r[My1], c[My1k]);
  ora_r2c_2d(Nx, Ny, r[My2], c[My2k]);
  ora_r2c_2d(Nx, Ny, r[Ex], c[Exk]);
  ora_r2c_2d(Nx, Ny, r[Ey], c[Eyk]);
  ora_r2c_2d(Nx, Ny, r[EV], c[EVk]);
  ora_r2c_2d(Nx, Ny, r[Magx], c[Magxk]);
  ora_r2c_2d(Nx, Ny, r[Magy], c[Magyk]);
  /* :262-422 derivatives, dealiasing, assembly */
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      size_t k = IX(i, j, Nh);
      ocplx a_rux = ik_mul(kx, rho_ux_k[k]);
      ocplx a_ruy = ik_mul(ky, rho_uy_k[k]);
      ocplx a_mx1 = ik_mul(kx, c[Mx1k][k]);
      ocplx a_mx2 = ik_mul(ky, c[Mx2k][k]);
      ocplx a_my1 = ik_mul(kx, c[My1k][k]);
      ocplx a_my2 = ik_mul(ky, c[My2k][k]);
      ocplx kx2ux = rmul(kx * kx, c[ux_k][k]);
      ocplx ky2ux = rmul(ky * ky, c[ux_k][k]);
      ocplx kx2uy = rmul(kx * kx, c[uy_k][k]);
      ocplx ky2uy = rmul(ky * ky, c[uy_k][k]);
      ocplx a_ex = ik_mul(kx, c[Exk][k]);
      ocplx a_ey = ik_mul(ky, c[Eyk][k]);
      ocplx ev = c[EVk][k];
      ocplx a_magx = ik_mul(ky, c[Magxk][k]);
      ocplx a_magy = ik_mul(kx, c[Magyk][k]);
      ocplx kx2bx = rmul(kx * kx, Bx_k[k]);
      ocplx ky2bx = rmul(ky * ky, Bx_k[k]);
      ocplx kx2by = rmul(kx * kx, By_k[k]);
      ocplx ky2by = rmul(ky * ky, By_k[k]);
      if (masked(kx, ky, Nx, Ny)) {
        a_rux = 0; a_ruy = 0; a_mx1 = 0; a_mx2 = 0; a_my1 = 0; a_my2 = 0;
        kx2ux = 0; ky2ux = 0; kx2uy = 0; ky2uy = 0;
        a_ex = 0; a_ey = 0; ev = 0; a_magx = 0; a_magy = 0;
        kx2bx = 0; ky2bx = 0; kx2by = 0; ky2by = 0;
      }
      d_rho[k] = -(a_rux + a_ruy);
      ocplx t = -(a_mx1 + a_mx2);
      d_rho_ux[k] = t - rmul(mu, kx2ux + ky2ux) + c[Fx_k][k];
      t = -(a_my1 + a_my2);
      d_rho_uy[k] = t - rmul(mu, kx2uy + ky2uy) + c[Fy_k][k];
      t = -(a_ex + a_ey);
      d_E[k] = t + rmul(mu, ev);
      d_Bx[k] = -a_magx - rmul(eta, kx2bx + ky2bx);
      d_By[k] = -a_magy - rmul(eta, kx2by + ky2by);
    }
  for (int q = 0; q < NR_; q++) fftw_free(r[q]);
  for (int q = 0; q < NC_; q++) fftw_free(c[q]);
}

/* ab2com: src/ab2com.f95:66-79 */
void ora_ab2com(int Nx, int Ny, int Nh, const ora_com_params *P,
                const ocplx *const state[6], ocplx *const state_new[6],
                const ocplx *const d_old[6], const ocplx *const d_new[6]) {
  (void)Nx;
  const double dt = P->dt;
  OMP_FOR
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      size_t k = IX(i, j, Nh);
      for (int f = 0; f < 6; f++)
        state_new[f][k] = state[f][k] + rmul(dt, rmul(3.0 / 2.0, d_new[f][k]) - rmul(1.0 / 2.0, d_old[f][k]));
    }
}

/* Classical RK4 of the coupled MHD system (new; the reference has no *2com RK4). */
void ora_rk4com(int Nx, int Ny, int Nh, double pi, double time, const ora_com_params *P,
                ocplx *const state[6]) {
  const double dt = P->dt;
  const size_t nc = (size_t)Nh * Ny;
  ocplx *us[6], *acc[6], *k[6];
  for (int f = 0; f < 6; f++) {
    us[f] = cnew(Nh, Ny); acc[f] = cnew(Nh, Ny); k[f] = cnew(Nh, Ny);
    memcpy(us[f], state[f], nc * sizeof(ocplx));
  }
  static const double cstage[3] = {0.5, 0.5, 1.0};
  static const double wstage[4] = {1.0, 2.0, 2.0, 1.0};
  for (int s = 0; s < 4; s++) {
    ora_derive2com(Nx, Ny, Nh, pi, time + (s == 0 ? 0.0 : cstage[s - 1] * dt), P,
                   us[0], us[1], us[2], us[3], us[4], us[5], k[0], k[1], k[2], k[3], k[4], k[5]);
    for (int f = 0; f < 6; f++) {
      ocplx *a = acc[f], *kk = k[f], *u = state[f], *v = us[f];
      const double wa = wstage[s] * dt / 6.0, cs = s < 3 ? cstage[s] * dt : 0.0;
      OMP_FOR
      for (size_t q = 0; q < nc; q++) {
        a[q] = (s == 0 ? u[q] : a[q]) + rmul(wa, kk[q]);
        if (s < 3) v[q] = u[q] + rmul(cs, kk[q]);
      }
    }
  }
  for (int f = 0; f < 6; f++) {
    memcpy(state[f], acc[f], nc * sizeof(ocplx));
    fftw_free(us[f]); fftw_free(acc[f]); fftw_free(k[f]);
  }
}

/* ======================================================================= */
/* derive2csh: src/derive2csh.f95:3-149 (pi = 3.1428 there, :16)            */
/* ======================================================================= */
void ora_derive2csh(int Nx, int Ny, int Nh, double nu, double time,
                    const ocplx *omegak, ocplx *dt_omegak_new) {
  (void)time;
  const double pi = (double)3.1428f; /* real(kind=8), parameter :: pi = 3.1428 (a REAL*4 literal) */
  const double Lx = 2.0 * pi, Ly = 2.0 * pi;
  ocplx *ukx = cnew(Nh, Ny), *uky = cnew(Nh, Ny), *ikxw = cnew(Nh, Ny), *ikyw = cnew(Nh, Ny);
  ocplx *NLkx = cnew(Nh, Ny), *NLky = cnew(Nh, Ny);
  double *ux = rnew(Nx, Ny), *uy = rnew(Nx, Ny), *dwx = rnew(Nx, Ny), *dwy = rnew(Nx, Ny);
  double *a = rnew(Nx, Ny), *b = rnew(Nx, Ny);
  for (int i = 0; i < Nh; i++) {
    double kx = 2.0 * pi * (double)i / Lx;
    for (int j = 0; j < Ny; j++) {
      double ky = (j < Ny / 2) ? 2.0 * pi * (double)j / Ly : 2.0 * pi * ((double)j - Ny) / Ly;
      size_t k = IX(i, j, Nh);
      if (i == 0 && j == 0) {
        ukx[k] = 0; uky[k] = 0;
      } else {
        ocplx psik = omegak[k] / (kx * kx + ky * ky);
        ukx[k] = ik_mul(ky, psik);
        uky[k] = -ik_mul(kx, psik);
      }
      ikxw[k] = ik_mul(kx, omegak[k]);
      ikyw[k] = ik_mul(ky, omegak[k]);
    }
  }
  c2r_destroy(Nx, Ny, ukx, ux);
  c2r_destroy(Nx, Ny, uky, uy);
  c2r_destroy(Nx, Ny, ikxw, dwx);
  c2r_destroy(Nx, Ny, ikyw, dwy);
  const double NN = (double)Nx * (double)Ny;
  for (size_t k = 0; k < (size_t)Nx * Ny; k++) {
    ux[k] = ux[k] / NN; uy[k] = uy[k] / NN; dwx[k] = dwx[k] / NN; dwy[k] = dwy[k] / NN;
    a[k] = ux[k] * dwx[k];
    b[k] = uy[k] * dwy[k];
  }
  ora_r2c_2d(Nx, Ny, a, NLkx);
  ora_r2c_2d(Nx, Ny, b, NLky);
  for (int i = 0; i < Nh; i++) {
    double kx = 2.0 * pi * (double)i / Lx;
    for (int j = 0; j < Ny; j++) {
      double ky = (j < Ny / 2) ? 2.0 * pi * (double)j / Ly : 2.0 * pi * ((double)j - Ny) / Ly;
      size_t k = IX(i, j, Nh);
      if (sqrt(kx * kx + ky * ky) >= ((double)(Nx + Ny) / 2.0) / 3.0) { NLkx[k] = 0; NLky[k] = 0; }
      ocplx nl = NLkx[k] + NLky[k];
      nl = nl + rmul(nu * (kx * kx + ky * ky), omegak[k]);
      dt_omegak_new[k] = -nl;
    }
  }
  fftw_free(ukx); fftw_free(uky); fftw_free(ikxw); fftw_free(ikyw); fftw_free(NLkx); fftw_free(NLky);
  fftw_free(ux); fftw_free(uy); fftw_free(dwx); fftw_free(dwy); fftw_free(a); fftw_free(b);
}

/* ab2csh: src/ab2csh.f95:3-16 ; ab2css: src/ab2css.f95:6-22 (same update) */
void ora_ab2csh(int Nx, int Ny, int Nh, double dt, const ocplx *omegak, ocplx *omegak_new,
                const ocplx *dt_omegak_old, const ocplx *dt_omegak_new) {
  (void)Nx;
  for (size_t k = 0; k < (size_t)Nh * Ny; k++)
    omegak_new[k] = omegak[k] + rmul(dt, rmul(3.0 / 2.0, dt_omegak_new[k]) - rmul(1.0 / 2.0, dt_omegak_old[k]));
}
void ora_ab2css(int Nx, int Ny, int Nh, double dt, const ocplx *omegak, ocplx *omegak_new,
                const ocplx *dt_omegak_old, const ocplx *dt_omegak_new) {
  ora_ab2csh(Nx, Ny, Nh, dt, omegak, omegak_new, dt_omegak_old, dt_omegak_new);
}

/* derive2css: src/derive2css.f95:6-136 with Lx, Ly, lambda explicit */
void ora_derive2css(int Nx, int Ny, int Nh, double alpha, double nu, double time,
                    double Lx, double Ly, double lambda,
                    const ocplx *omegak, ocplx *dt_omegak_new) {
  (void)time;
  const double pi = (double)3.1428f;
  ocplx *ukx = cnew(Nh, Ny), *uky = cnew(Nh, Ny), *wd = cnew(Nh, Ny), *ikxw = cnew(Nh, Ny),
        *ikyw = cnew(Nh, Ny), *NLkx = cnew(Nh, Ny), *NLky = cnew(Nh, Ny);
  double *ux = rnew(Nx, Ny), *uy = rnew(Nx, Ny), *dwx = rnew(Nx, Ny), *dwy = rnew(Nx, Ny);
  double *a = rnew(Nx, Ny), *b = rnew(Nx, Ny);
  for (int i = 0; i < Nh; i++)
    for (int j = 0; j < Ny; j++) {
      double kx = 2.0 * pi * (double)i / Lx;
      double ky = (j < Ny / 2) ? 2.0 * pi * (double)j / Ly : 2.0 * pi * (double)(j - Ny) / Ly;
      size_t k = IX(i, j, Nh);
      ocplx psik;
      if (j < Ny / 2 && i == 0 && j == 0) {
        psik = 0; ukx[k] = 0; uky[k] = 0;
      } else {
        psik = omegak[k] / (kx * kx + ky * ky + lambda);
        ukx[k] = ik_mul(ky, psik);
        uky[k] = -ik_mul(kx, psik);
      }
      wd[k] = rmul(kx * kx + ky * ky, psik);
      ikxw[k] = ik_mul(kx, wd[k]);
      ikyw[k] = ik_mul(ky, wd[k]);
    }
  c2r_destroy(Nx, Ny, ukx, ux);
  c2r_destroy(Nx, Ny, uky, uy);
  c2r_destroy(Nx, Ny, ikxw, dwx);
  c2r_destroy(Nx, Ny, ikyw, dwy);
  const double NN = (double)Nx * (double)Ny;
  for (size_t k = 0; k < (size_t)Nx * Ny; k++) {
    ux[k] = ux[k] / NN; uy[k] = uy[k] / NN; dwx[k] = dwx[k] / NN; dwy[k] = dwy[k] / NN;
    a[k] = ux[k] * dwx[k];
    b[k] = uy[k] * dwy[k];
  }
  ora_r2c_2d(Nx, Ny, a, NLkx);
  ora_r2c_2d(Nx, Ny, b, NLky);
  for (int i = 0; i < Nh; i++)
    for (int j = 0; j < Ny; j++) {
      double kx = 2.0 * pi * (double)i / Lx;
      double ky = (j < Ny / 2) ? 2.0 * pi * (double)j / Ly : 2.0 * pi * (double)(j - Ny) / Ly;
      size_t k = IX(i, j, Nh);
      if (sqrt(kx * kx + ky * ky) >= ((double)(Nx + Ny) / 2.0) / 3.0 + 0) { NLkx[k] = 0; NLky[k] = 0; }
      ocplx nl = rmul(alpha, NLkx[k] + NLky[k]);
      nl = nl + rmul(nu * (kx * kx + ky * ky), wd[k]);
      dt_omegak_new[k] = -nl;
    }
  fftw_free(ukx); fftw_free(uky); fftw_free(wd); fftw_free(ikxw); fftw_free(ikyw);
  fftw_free(NLkx); fftw_free(NLky);
  fftw_free(ux); fftw_free(uy); fftw_free(dwx); fftw_free(dwy); fftw_free(a); fftw_free(b);
}

/* ======================================================================= */
/* drivers                                                                  */
/* ======================================================================= */
void ora_run_coh(int Nx, int Ny, double pi, const ora_coh_params *P, int stepper, int nsteps,
                 ocplx *nk, ocplx *ukx, ocplx *uky, ocplx *dn_old, ocplx *dux_old, ocplx *duy_old) {
  const int Nh = Nx / 2 + 1;
  const size_t nc = (size_t)Nh * Ny;
  ocplx *dn = cnew(Nh, Ny), *dux = cnew(Nh, Ny), *duy = cnew(Nh, Ny);
  ocplx *nn = cnew(Nh, Ny), *uxn = cnew(Nh, Ny), *uyn = cnew(Nh, Ny);
  for (int t = 0; t < nsteps; t++) {
    double time = t * P->dt;
    if (stepper == 1) {
      ora_rk4coh(Nx, Ny, Nh, pi, time, P, nk, ukx, uky);
      continue;
    }
    /* src/main2coh.f95:278-316 */
    ora_derive2coh(Nx, Ny, Nh, pi, time, P, nk, ukx, uky, dn, dux, duy);
    if (stepper == 0)
      ora_ab2coh(Nx, Ny, Nh, P, nk, ukx, uky, nn, uxn, uyn, dn_old, dux_old, duy_old, dn, dux, duy);
    else
      ora_euler2coh(Nx, Ny, Nh, P, nk, ukx, uky, nn, uxn, uyn, dn, dux, duy);
    memcpy(dn_old, dn, nc * sizeof(ocplx));
    memcpy(dux_old, dux, nc * sizeof(ocplx));
    memcpy(duy_old, duy, nc * sizeof(ocplx));
    memcpy(nk, nn, nc * sizeof(ocplx));
    memcpy(ukx, uxn, nc * sizeof(ocplx));
    memcpy(uky, uyn, nc * sizeof(ocplx));
  }
  fftw_free(dn); fftw_free(dux); fftw_free(duy); fftw_free(nn); fftw_free(uxn); fftw_free(uyn);
}

void ora_run_com(int Nx, int Ny, double pi, const ora_com_params *P, int stepper, int nsteps,
                 ocplx *const state[6], ocplx *const d_old[6]) {
  const int Nh = Nx / 2 + 1;
  const size_t nc = (size_t)Nh * Ny;
  ocplx *dn[6], *sn[6];
  for (int f = 0; f < 6; f++) { dn[f] = cnew(Nh, Ny); sn[f] = cnew(Nh, Ny); }
  for (int t = 0; t < nsteps; t++) {
    double time = t * P->dt;
    if (stepper == 1) {
      ora_rk4com(Nx, Ny, Nh, pi, time, P, state);
      continue;
    }
    /* src/main2com.f95:364-423 */
    ora_derive2com(Nx, Ny, Nh, pi, time, P, state[0], state[1], state[2], state[3], state[4], state[5],
                   dn[0], dn[1], dn[2], dn[3], dn[4], dn[5]);
    if (stepper == 0) {
      ora_ab2com(Nx, Ny, Nh, P, (const ocplx *const *)state, sn, (const ocplx *const *)d_old,
                 (const ocplx *const *)dn);
    } else {
      for (int f = 0; f < 6; f++)
        for (size_t q = 0; q < nc; q++) sn[f][q] = state[f][q] + rmul(P->dt, dn[f][q]);
    }
    for (int f = 0; f < 6; f++) {
      memcpy(d_old[f], dn[f], nc * sizeof(ocplx));
      memcpy(state[f], sn[f], nc * sizeof(ocplx));
    }
  }
  for (int f = 0; f < 6; f++) { fftw_free(dn[f]); fftw_free(sn[f]); }
}

/* ======================================================================= */
/* diagnostics                                                              */
/* ======================================================================= */
/* src/main2com.f95:425-616 (Energy, B_Field, C2, C3, div_B_Tot) + <u.B> */
void ora_diag_com(int Nx, int Ny, double pi, const ora_com_params *P, const ocplx *const state[6],
                  double out[6]) {
  const int Nh = Nx / 2 + 1;
  const double Lx = P->Lx, Ly = P->Ly, NN = (double)Nx * (double)Ny;
  double *rho = rnew(Nx, Ny), *rux = rnew(Nx, Ny), *ruy = rnew(Nx, Ny), *bx = rnew(Nx, Ny),
         *by = rnew(Nx, Ny), *divb = rnew(Nx, Ny), *ux = rnew(Nx, Ny), *uy = rnew(Nx, Ny),
         *om = rnew(Nx, Ny), *jb = rnew(Nx, Ny);
  ocplx *divk = cnew(Nh, Ny), *uxk = cnew(Nh, Ny), *uyk = cnew(Nh, Ny), *omk = cnew(Nh, Ny),
        *jk = cnew(Nh, Ny);
  const ocplx *Bxk = state[4], *Byk = state[5];
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      size_t k = IX(i, j, Nh);
      divk[k] = ik_mul(kx, Bxk[k]) + ik_mul(ky, Byk[k]);
    }
  ora_c2r_2d(Nx, Ny, state[0], rho);
  ora_c2r_2d(Nx, Ny, state[1], rux);
  ora_c2r_2d(Nx, Ny, state[2], ruy);
  ora_c2r_2d(Nx, Ny, state[4], bx);
  ora_c2r_2d(Nx, Ny, state[5], by);
  c2r_destroy(Nx, Ny, divk, divb);
  for (size_t k = 0; k < (size_t)Nx * Ny; k++) {
    rho[k] /= NN; rux[k] /= NN; ruy[k] /= NN; bx[k] /= NN; by[k] /= NN; divb[k] /= NN;
    ux[k] = rux[k] / rho[k];
    uy[k] = ruy[k] / rho[k];
  }
  ora_r2c_2d(Nx, Ny, ux, uxk);
  ora_r2c_2d(Nx, Ny, uy, uyk);
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      size_t k = IX(i, j, Nh);
      omk[k] = ik_mul(kx, uyk[k]) - ik_mul(ky, uxk[k]);
      jk[k] = ik_mul(kx, Byk[k]) - ik_mul(ky, Bxk[k]);
    }
  c2r_destroy(Nx, Ny, omk, om);
  c2r_destroy(Nx, Ny, jk, jb);
  double Energy = 0, B_Field = 0, C2 = 0, C3 = 0, divB = 0, Hc = 0;
  for (int i = 0; i < Nx; i++)   /* the reference sums with i outer, j inner (:587-588) */
    for (int j = 0; j < Ny; j++) {
      size_t k = IX(i, j, Nx);
      double w = om[k] / NN, jj = jb[k] / NN;
      Energy = Energy + (ux[k] * ux[k] + uy[k] * uy[k]) / NN;
      B_Field = B_Field + (bx[k] * bx[k] + by[k] * by[k]) / NN;
      C2 = C2 + (w * w) / NN;
      C3 = C3 + (jj * jj) / NN;
      divB = divB + divb[k] / NN;
      Hc = Hc + (ux[k] * bx[k] + uy[k] * by[k]) / NN;
    }
  out[0] = Energy; out[1] = B_Field; out[2] = C2; out[3] = C3; out[4] = divB; out[5] = Hc;
  fftw_free(rho); fftw_free(rux); fftw_free(ruy); fftw_free(bx); fftw_free(by); fftw_free(divb);
  fftw_free(ux); fftw_free(uy); fftw_free(om); fftw_free(jb);
  fftw_free(divk); fftw_free(uxk); fftw_free(uyk); fftw_free(omk); fftw_free(jk);
}

/* src/main2coh.f95:321-429 (Energy/2NN, y_Energy/2NN, C0..C3 /NN) */
void ora_diag_coh(int Nx, int Ny, double pi, const ora_coh_params *P,
                  const ocplx *nk, const ocplx *ukx, const ocplx *uky, double out[6]) {
  const int Nh = Nx / 2 + 1;
  const double Lx = P->Lx, Ly = P->Ly, NN = (double)Nx * (double)Ny;
  ocplx *omk = cnew(Nh, Ny);
  double *ux = rnew(Nx, Ny), *uy = rnew(Nx, Ny), *om = rnew(Nx, Ny), *n = rnew(Nx, Ny);
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      size_t k = IX(i, j, Nh);
      omk[k] = ik_mul(kx, uky[k]) - ik_mul(ky, ukx[k]);
    }
  ora_c2r_2d(Nx, Ny, nk, n);
  ora_c2r_2d(Nx, Ny, ukx, ux);
  ora_c2r_2d(Nx, Ny, uky, uy);
  c2r_destroy(Nx, Ny, omk, om);
  double Energy = 0, yE = 0, C0 = 0, C1 = 0, C2 = 0, C3 = 0;
  for (int i = 0; i < Nx; i++)
    for (int j = 0; j < Ny; j++) {
      size_t k = IX(i, j, Nx);
      double vx = ux[k] / NN, vy = uy[k] / NN, w = om[k] / NN;
      Energy = Energy + (vx * vx + vy * vy);
      yE = yE + vy * vy;
      C0 = C0 + 1.0;
      C1 = C1 + w;
      C2 = C2 + pow(w, 2.0);
      C3 = C3 + pow(w, 3.0);
    }
  out[0] = Energy / (2.0 * NN); out[1] = yE / (2.0 * NN);
  out[2] = C0 / NN; out[3] = C1 / NN; out[4] = C2 / NN; out[5] = C3 / NN;
  fftw_free(omk); fftw_free(ux); fftw_free(uy); fftw_free(om); fftw_free(n);
}

/* ---- shell spectrum E(k) (a definition of this build; the reference keeps
 * only a commented-out per-mode listing at src/main2com.f95:566-577) ----
 * E(k) = sum over floor(|k| + 1/2) = k of (|ux_k|^2 + |uy_k|^2) / 2 / (NxNy)^2,
 * half-spectrum modes with 0 < i < Nx/2 counted twice.  Velocity spectra are
 * the unnormalised forward transforms of the velocity. */
int ora_num_shells(int Nx, int Ny, double pi, double Lx, double Ly) {
  const double kxm = kx_of(Nx / 2, pi, Lx), kym = fabs(ky_of(Ny / 2, Ny, pi, Ly));
  return (int)floor(sqrt(kxm * kxm + kym * kym) + 0.5) + 1;
}

static void shell_spectrum(int Nx, int Ny, double pi, double Lx, double Ly, const ocplx *uxk,
                           const ocplx *uyk, int nbins, double *Ek) {
  const int Nh = Nx / 2 + 1;
  const double NN = (double)Nx * (double)Ny;
  for (int s = 0; s < nbins; s++) Ek[s] = 0.0;
  for (int j = 0; j < Ny; j++)
    for (int i = 0; i < Nh; i++) {
      const double kx = kx_of(i, pi, Lx), ky = ky_of(j, Ny, pi, Ly);
      const int s = (int)floor(sqrt(kx * kx + ky * ky) + 0.5);
      const size_t k = IX(i, j, Nh);
      const double w = (i > 0 && i < Nx / 2) ? 2.0 : 1.0;
      const double e = creal(uxk[k]) * creal(uxk[k]) + cimag(uxk[k]) * cimag(uxk[k]) +
                       creal(uyk[k]) * creal(uyk[k]) + cimag(uyk[k]) * cimag(uyk[k]);
      if (s < nbins) Ek[s] += 0.5 * w * e;
    }
  for (int s = 0; s < nbins; s++) Ek[s] = Ek[s] / NN / NN;
}

void ora_spectrum_coh(int Nx, int Ny, double pi, const ora_coh_params *P, const ocplx *ukx, const ocplx *uky,
                      int nbins, double *Ek) {
  shell_spectrum(Nx, Ny, pi, P->Lx, P->Ly, ukx, uky, nbins, Ek);
}

/* velocity of the MHD state as in src/main2com.f95:446-480: u = c2r(rho u)/c2r(rho) */
void ora_spectrum_com(int Nx, int Ny, double pi, const ora_com_params *P, const ocplx *const state[6], int nbins,
                      double *Ek) {
  const int Nh = Nx / 2 + 1;
  const double NN = (double)Nx * (double)Ny;
  double *rho = rnew(Nx, Ny), *ux = rnew(Nx, Ny), *uy = rnew(Nx, Ny);
  ocplx *uxk = cnew(Nh, Ny), *uyk = cnew(Nh, Ny);
  ora_c2r_2d(Nx, Ny, state[0], rho);
  ora_c2r_2d(Nx, Ny, state[1], ux);
  ora_c2r_2d(Nx, Ny, state[2], uy);
  for (size_t k = 0; k < (size_t)Nx * Ny; k++) {
    rho[k] /= NN;
    ux[k] = (ux[k] / NN) / rho[k];
    uy[k] = (uy[k] / NN) / rho[k];
  }
  ora_r2c_2d(Nx, Ny, ux, uxk);
  ora_r2c_2d(Nx, Ny, uy, uyk);
  shell_spectrum(Nx, Ny, pi, P->Lx, P->Ly, uxk, uyk, nbins, Ek);
  fftw_free(rho); fftw_free(ux); fftw_free(uy); fftw_free(uxk); fftw_free(uyk);
}

/* ======================================================================= */
/* 3D MHD: derive3com (src/derive3com.f95:5-1047), ab3com (src/ab3com.f95)   */
/* ======================================================================= */
/* Fortran (Nx,Ny,Nz) is C [Nz][Ny][Nx]: dfftw_plan_dft_c2r_3d(p,Nx,Ny,Nz,...)
 * is fftw_plan_dft_c2r_3d(Nz,Ny,Nx,...) (lib/fftw/api/f77funcs.h). */
static void c2r3_destroy(int Nx, int Ny, int Nz, ocplx *in, double *out) {
  fftw_plan p = fftw_plan_dft_c2r_3d(Nz, Ny, Nx, (fftw_complex *)in, out, FFTW_ESTIMATE);
  fftw_execute(p);
  fftw_destroy_plan(p);
}
static void r2c3(int Nx, int Ny, int Nz, const double *in, ocplx *out) {
  fftw_plan p = fftw_plan_dft_r2c_3d(Nz, Ny, Nx, (double *)in, (fftw_complex *)out, FFTW_ESTIMATE);
  fftw_execute(p);
  fftw_destroy_plan(p);
}

void ora_derive3com(int Nx, int Ny, int Nz, double pi, const ora_com3_params *P, const ocplx *const st[8],
                    ocplx *const dnew[8]) {
  const int Nh = Nx / 2 + 1;
  const size_t nc = (size_t)Nh * Ny * Nz, nr = (size_t)Nx * Ny * Nz;
  const double NN = (double)Nx * (double)Ny * (double)Nz; /* dfloat(Nx)*dfloat(Ny)*dfloat(Nz) */
  double *R[8], *U[3], *Dv[9], *F[19];
  ocplx *tmp = (ocplx *)xmalloc(sizeof(ocplx) * nc), *uk[3], *Fk[19];
  for (int q = 0; q < 8; q++) R[q] = (double *)xmalloc(sizeof(double) * nr);
  for (int q = 0; q < 3; q++) { U[q] = (double *)xmalloc(sizeof(double) * nr); uk[q] = (ocplx *)xmalloc(sizeof(ocplx) * nc); }
  for (int q = 0; q < 9; q++) Dv[q] = (double *)xmalloc(sizeof(double) * nr);
  for (int q = 0; q < 19; q++) { F[q] = (double *)xmalloc(sizeof(double) * nr); Fk[q] = (ocplx *)xmalloc(sizeof(ocplx) * nc); }
  /* state c2r from *_dum copies (:60-135) */
  for (int q = 0; q < 8; q++) {
    memcpy(tmp, st[q], sizeof(ocplx) * nc);
    c2r3_destroy(Nx, Ny, Nz, tmp, R[q]);
  }
  /* normalisation and velocity (:160-182); the forcing (:184-188) is not used */
  OMP_FOR
  for (size_t p = 0; p < nr; p++) {
    for (int q = 0; q < 8; q++) R[q][p] = R[q][p] / NN;
    U[0][p] = R[1][p] / R[0][p];
    U[1][p] = R[2][p] / R[0][p];
    U[2][p] = R[3][p] / R[0][p];
  }
  for (int q = 0; q < 3; q++) r2c3(Nx, Ny, Nz, U[q], uk[q]); /* (:198-215) */
  /* first derivatives (:232-340): i kx ux, i ky uy, i kz uz, i ky Bx, i kz Bx,
   * i kx By, i kz By, i kx Bz, i ky Bz */
  const ocplx *dsrc[9] = {uk[0], uk[1], uk[2], st[5], st[5], st[6], st[6], st[7], st[7]};
  const int dk[9] = {0, 1, 2, 1, 2, 0, 2, 0, 1};
  for (int q = 0; q < 9; q++) {
    OMP_FOR
    for (int k = 0; k < Nz; k++)
      for (int j = 0; j < Ny; j++)
        for (int i = 0; i < Nh; i++) {
          const double kx = kx_of(i, pi, P->Lx), ky = ky_of(j, Ny, pi, P->Ly), kz = ky_of(k, Nz, pi, P->Lz);
          const double kk = dk[q] == 0 ? kx : (dk[q] == 1 ? ky : kz);
          const size_t m = (size_t)i + (size_t)Nh * ((size_t)j + (size_t)Ny * k);
          tmp[m] = ik_mul(kk, dsrc[q][m]);
        }
    c2r3_destroy(Nx, Ny, Nz, tmp, Dv[q]);
  }
  /* real-space fluxes (:343-414) */
  const double CS = P->CS, eta = P->eta;
  OMP_FOR
  for (size_t p = 0; p < nr; p++) {
    for (int q = 0; q < 9; q++) Dv[q][p] = Dv[q][p] / NN;
    const double rho = R[0][p], rux = R[1][p], ruy = R[2][p], ruz = R[3][p], E = R[4][p];
    const double Bx = R[5][p], By = R[6][p], Bz = R[7][p];
    const double ux = U[0][p], uy = U[1][p], uz = U[2][p];
    const double B2 = Bx * Bx + By * By + Bz * Bz;
    const double cxB = Dv[8][p] - Dv[6][p], cyB = Dv[7][p] - Dv[4][p], czB = Dv[5][p] - Dv[3][p];
    const double Pp = CS * CS * rho;
    F[0][p] = rux * ux + Pp + B2 / 2.0 - Bx * Bx;
    F[1][p] = rux * uy - Bx * By;
    F[2][p] = rux * uz - Bx * Bz;
    F[3][p] = rux * uy - Bx * By; /* Mom_y_1 as written */
    F[4][p] = ruy * uy + Pp + B2 / 2.0 - By * By;
    F[5][p] = ruy * uz - By * Bz;
    F[6][p] = ruz * ux - Bz * Bx;
    F[7][p] = ruz * uy - Bz * By;
    F[8][p] = ruz * uz + Pp + B2 / 2.0 - Bz * Bz;
    F[9][p] = (E + Pp + B2 / 2.0) * ux - ux * Bx * Bx - uy * Bx * By - uz * Bx * Bz - eta * (By * czB + Bz * cyB);
    F[10][p] = (E + Pp + B2 / 2.0) * uy - ux * Bx * By - uy * By * By - uz * By * Bz + eta * (Bx * czB - Bz * cxB);
    F[11][p] = (E + Pp + B2 / 2.0) * uz - ux * Bz * Bx - uy * Bz * By - uz * Bz * Bz + eta * (Bx * cyB + By * cxB);
    const double dv = Dv[0][p] + Dv[1][p] + Dv[2][p];
    F[12][p] = dv * dv;
    F[13][p] = ux * By - uy * Bx;
    F[14][p] = ux * Bz - uz * Bx;
    F[15][p] = ux * By - uy * Bx; /* Mag_y_1 as written */
    F[16][p] = uy * Bz - uz * By;
    F[17][p] = ux * Bz - uz * Bx; /* Mag_z_1 as written */
    F[18][p] = uy * Bz - uz * By; /* Mag_z_2 as written */
  }
  for (int q = 0; q < 19; q++) r2c3(Nx, Ny, Nz, F[q], Fk[q]); /* (:416-500) */
  /* spectral derivatives, mask and sums (:502-1043) */
  const double thr = ((double)(Nx + Ny + Nz) / 3.0) / 3.0 + 0;
  const double mu = P->mu;
  OMP_FOR
  for (int k = 0; k < Nz; k++)
    for (int j = 0; j < Ny; j++)
      for (int i = 0; i < Nh; i++) {
        const size_t m = (size_t)i + (size_t)Nh * ((size_t)j + (size_t)Ny * k);
        const double kx = kx_of(i, pi, P->Lx), ky = ky_of(j, Ny, pi, P->Ly), kz = ky_of(k, Nz, pi, P->Lz);
        if (sqrt(kx * kx + ky * ky + kz * kz) >= thr) {
          for (int q = 0; q < 8; q++) dnew[q][m] = 0;
          continue;
        }
        ocplx v3[3];
        for (int c = 0; c < 3; c++) {
          const ocplx u = uk[c][m];
          v3[c] = rmul(kx * kx, u) + rmul(ky * ky, u) + rmul(kz * kz, u);
          v3[c] = CMPLX(creal(v3[c]) / 450.0, cimag(v3[c]) / 450.0);
        }
        ocplx vb[3];
        for (int c = 0; c < 3; c++) {
          const ocplx b = st[5 + c][m];
          vb[c] = rmul(kx * kx, b) + rmul(ky * ky, b) + rmul(kz * kz, b);
          vb[c] = CMPLX(creal(vb[c]) / 450.0, cimag(vb[c]) / 450.0);
        }
        dnew[0][m] = -(ik_mul(kx, st[1][m]) + ik_mul(ky, st[2][m]) + ik_mul(kz, st[3][m]));
        dnew[1][m] = -(ik_mul(kx, Fk[0][m]) + ik_mul(ky, Fk[1][m]) + ik_mul(kz, Fk[2][m])) - v3[0];
        dnew[2][m] = -(ik_mul(kx, Fk[3][m]) + ik_mul(ky, Fk[4][m]) + ik_mul(kz, Fk[5][m])) - v3[1];
        dnew[3][m] = -(ik_mul(kx, Fk[6][m]) + ik_mul(ky, Fk[7][m]) + ik_mul(kz, Fk[8][m])) - v3[2];
        dnew[4][m] = -(ik_mul(kx, Fk[9][m]) + ik_mul(ky, Fk[10][m]) + ik_mul(kz, Fk[11][m])) + rmul(mu, Fk[12][m]);
        dnew[5][m] = (ik_mul(ky, Fk[13][m]) + ik_mul(kz, Fk[14][m])) - vb[0];
        dnew[6][m] = -(ik_mul(kx, Fk[15][m]) - ik_mul(kz, Fk[16][m])) - vb[1];
        dnew[7][m] = -(ik_mul(kx, Fk[17][m]) + ik_mul(ky, Fk[18][m])) - vb[2];
      }
  fftw_free(tmp);
  for (int q = 0; q < 8; q++) fftw_free(R[q]);
  for (int q = 0; q < 3; q++) { fftw_free(U[q]); fftw_free(uk[q]); }
  for (int q = 0; q < 9; q++) fftw_free(Dv[q]);
  for (int q = 0; q < 19; q++) { fftw_free(F[q]); fftw_free(Fk[q]); }
}

/* ab3com: src/ab3com.f95:44-61 (E_k_new = E_k: its update is commented out) */
void ora_ab3com(int Nx, int Ny, int Nz, double dt, const ocplx *const st[8], ocplx *const st_new[8],
                const ocplx *const d_old[8], const ocplx *const d_new[8]) {
  const size_t nc = (size_t)(Nx / 2 + 1) * Ny * Nz;
  for (int f = 0; f < 8; f++) {
    OMP_FOR
    for (size_t m = 0; m < nc; m++)
      st_new[f][m] = f == 4 ? st[f][m] : st[f][m] + rmul(dt, rmul(3.0 / 2.0, d_new[f][m]) - rmul(1.0 / 2.0, d_old[f][m]));
  }
}

/* time loop of src/main3com.f95:536-600: derive3com, ab3com, d_old = d_new */
void ora_run3com(int Nx, int Ny, int Nz, double pi, const ora_com3_params *P, int nsteps, ocplx *const st[8],
                 ocplx *const d_old[8]) {
  const size_t nc = (size_t)(Nx / 2 + 1) * Ny * Nz;
  ocplx *dn[8], *sn[8];
  for (int f = 0; f < 8; f++) { dn[f] = (ocplx *)xmalloc(sizeof(ocplx) * nc); sn[f] = (ocplx *)xmalloc(sizeof(ocplx) * nc); }
  for (int t = 0; t < nsteps; t++) {
    ora_derive3com(Nx, Ny, Nz, pi, P, (const ocplx *const *)st, dn);
    ora_ab3com(Nx, Ny, Nz, P->dt, (const ocplx *const *)st, sn, (const ocplx *const *)d_old, (const ocplx *const *)dn);
    for (int f = 0; f < 8; f++) {
      memcpy(d_old[f], dn[f], nc * sizeof(ocplx));
      memcpy(st[f], sn[f], nc * sizeof(ocplx));
    }
  }
  for (int f = 0; f < 8; f++) { fftw_free(dn[f]); fftw_free(sn[f]); }
}
