/* CPU oracle for the TARA2D pseudo-spectral RHS + time-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a C restatement of the reference's
 * Fortran subroutines (src/derive2coh.f95, src/ab2coh.f95, src/euler2coh.f95,
 * src/pc*2coh.f95, src/rk4*2coh.f95, src/derive2com.f95, src/ab2com.f95,
 * src/derive2csh.f95, src/ab2csh.f95, src/derive2css.f95, src/ab2css.f95,
 * src/derive3com.f95, src/ab3com.f95),
 * linked against the reference's own vendored FFTW 3.3.9 compiled from its
 * sources (oracle/_ref/libfftw3_ref.a).  Only the tests, the smoke check and
 * the CPU-baseline leg of the benchmark may load it, and only as the checker.
 *
 * Parity status: the FFT stage is pinned (it IS the reference's FFTW); the
 * RHS/stepper algebra is a line-by-line restatement that the reference cannot
 * pin, because the reference has no tests or golden vectors and its Fortran
 * cannot be compiled here (no Fortran compiler).  It is cross-checked against
 * an independent numpy restatement and analytic known answers in tests/.
 *
 * Conventions (all arrays are Fortran column-major, 0-based here):
 *   real     (Nx,Ny): a[i + Nx*j]
 *   complex  (Nh,Ny): a[i + Nh*j], Nh = Nx/2+1
 * Physical parameters that the reference takes from COMMON /comm/ are passed
 * explicitly, because the two program units lay that block out differently
 * (src/derive2coh.f95:30 vs src/derive2com.f95:48).
 */
#ifndef TARA_ORACLE_H
#define TARA_ORACLE_H
#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex ocplx;

/* COMMON /comm/ of the hydro units: Lx,Ly,mux,muy,ms,CS,dt (src/main2coh.f95:29) */
typedef struct { double Lx, Ly, mux, muy, ms, CS, dt; } ora_coh_params;

/* COMMON /comm/ of the MHD units: Lx,Ly,spheat,mu,ms,CS,mu_0,eta,dt,kf,A
 * (src/main2com.f95:43) plus two switches for reference defects:
 *   fix_curlB  0 = reference (d_Bx_dy/d_By_dx built from the velocity
 *                  derivatives and divided twice, src/derive2com.f95:186-187)
 *              1 = corrected curl B = dBy/dx - dBx/dy
 *   The forcing grid is x_i=(i-1)Lx/Nx, y_j=(j-1)Ly/Ny (the reference reads
 *   uninitialised x,y there, src/derive2com.f95:16,109-110). */
typedef struct {
  double Lx, Ly, spheat, mu, ms, CS, mu_0, eta, dt, kf, A;
  int fix_curlB;
} ora_com_params;

/* ---- hydro (*2coh) ---- */
void ora_derive2coh(int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                    const ocplx *nk, const ocplx *ukx, const ocplx *uky,
                    ocplx *dn_dt_new, ocplx *dux_dt_new, ocplx *duy_dt_new);
void ora_ab2coh(int Nx, int Ny, int Nh, const ora_coh_params *P,
                const ocplx *nk, const ocplx *ukx, const ocplx *uky,
                ocplx *nk_new, ocplx *ukx_new, ocplx *uky_new,
                const ocplx *dn_dt_old, const ocplx *dux_dt_old, const ocplx *duy_dt_old,
                const ocplx *dn_dt_new, const ocplx *dux_dt_new, const ocplx *duy_dt_new);
void ora_euler2coh(int Nx, int Ny, int Nh, const ora_coh_params *P,
                   const ocplx *nk, const ocplx *ukx, const ocplx *uky,
                   ocplx *nk_new, ocplx *ukx_new, ocplx *uky_new,
                   const ocplx *dn_dt, const ocplx *dux_dt, const ocplx *duy_dt);
/* which = 0: nk, 1: ukx, 2: uky.  out = the advanced field.
 * Reference (bug-compatible) semantics, src/pcnk2coh.f95 / src/rk4nk2coh.f95. */
void ora_pc2coh(int which, int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                const ocplx *nk, const ocplx *ukx, const ocplx *uky, ocplx *out,
                const ocplx *dn_dt, const ocplx *dux_dt, const ocplx *duy_dt);
void ora_rk42coh(int which, int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                 const ocplx *nk, const ocplx *ukx, const ocplx *uky, ocplx *out,
                 const ocplx *dn_dt, const ocplx *dux_dt, const ocplx *duy_dt);
/* Coupled classical RK4 step of all three hydro fields (no reference counterpart). */
void ora_rk4coh(int Nx, int Ny, int Nh, double pi, double time, const ora_coh_params *P,
                ocplx *nk, ocplx *ukx, ocplx *uky);

/* ---- MHD (*2com) ---- */
void ora_derive2com(int Nx, int Ny, int Nh, double pi, double time, const ora_com_params *P,
                    const ocplx *rho_k, const ocplx *rho_ux_k, const ocplx *rho_uy_k,
                    const ocplx *E_k, const ocplx *Bx_k, const ocplx *By_k,
                    ocplx *d_rho, ocplx *d_rho_ux, ocplx *d_rho_uy,
                    ocplx *d_E, ocplx *d_Bx, ocplx *d_By);
/* AB2 on the six fields; state[f], state_new[f], d_old[f], d_new[f], f=0..5 in the
 * order rho, rho_ux, rho_uy, E, Bx, By (src/ab2com.f95:66-79). */
void ora_ab2com(int Nx, int Ny, int Nh, const ora_com_params *P,
                const ocplx *const state[6], ocplx *const state_new[6],
                const ocplx *const d_old[6], const ocplx *const d_new[6]);
/* Coupled classical RK4 step of the six MHD fields, in place (no reference counterpart). */
void ora_rk4com(int Nx, int Ny, int Nh, double pi, double time, const ora_com_params *P,
                ocplx *const state[6]);

/* ---- incompressible vorticity (*2csh) and screened vorticity (*2css) ---- */
void ora_derive2csh(int Nx, int Ny, int Nh, double nu, double time,
                    const ocplx *omegak, ocplx *dt_omegak_new);
void ora_ab2csh(int Nx, int Ny, int Nh, double dt, const ocplx *omegak, ocplx *omegak_new,
                const ocplx *dt_omegak_old, const ocplx *dt_omegak_new);
/* Lx, Ly and lambda are uninitialised locals in the reference
 * (src/derive2css.f95:12,24,32); they are explicit arguments here. */
void ora_derive2css(int Nx, int Ny, int Nh, double alpha, double nu, double time,
                    double Lx, double Ly, double lambda,
                    const ocplx *omegak, ocplx *dt_omegak_new);
void ora_ab2css(int Nx, int Ny, int Nh, double dt, const ocplx *omegak, ocplx *omegak_new,
                const ocplx *dt_omegak_old, const ocplx *dt_omegak_new);

/* ---- plain 2D transforms with the reference's calling convention ---- */
void ora_r2c_2d(int Nx, int Ny, const double *in, ocplx *out);   /* unnormalised */
void ora_c2r_2d(int Nx, int Ny, const ocplx *in, double *out);   /* unnormalised, input preserved */

/* ---- drivers (time loops of src/main2coh.f95:266-316, src/main2com.f95:352-423) ----
 * stepper: 0 = AB2 (reference), 1 = coupled RK4, 2 = Euler.
 * The AB2 history (*_dt_old) starts at zero. Diagnostics are not computed. */
void ora_run_coh(int Nx, int Ny, double pi, const ora_coh_params *P, int stepper, int nsteps,
                 ocplx *nk, ocplx *ukx, ocplx *uky, ocplx *dn_old, ocplx *dux_old, ocplx *duy_old);
void ora_run_com(int Nx, int Ny, double pi, const ora_com_params *P, int stepper, int nsteps,
                 ocplx *const state[6], ocplx *const d_old[6]);

/* ---- diagnostics (src/main2com.f95:425-616, src/main2coh.f95:321-429) ----
 * out_com: [Energy, B_Field, C2(<omega^2>), C3(<j^2>), div_B_Tot, cross helicity <u.B>]
 * out_coh: [Energy, y_Energy, C0, C1, C2, C3] (already divided as in the Energy.dat write) */
void ora_diag_com(int Nx, int Ny, double pi, const ora_com_params *P, const ocplx *const state[6],
                  double out[6]);
void ora_diag_coh(int Nx, int Ny, double pi, const ora_coh_params *P,
                  const ocplx *nk, const ocplx *ukx, const ocplx *uky, double out[6]);

/* ---- shell spectrum E(k) = sum_{floor(|k|+1/2)=k} (|ux_k|^2+|uy_k|^2)/2/(NxNy)^2 ----
 * (not in the reference, which only lists modes in commented-out code at
 * src/main2com.f95:566-577); nbins from ora_num_shells. */
int ora_num_shells(int Nx, int Ny, double pi, double Lx, double Ly);
void ora_spectrum_coh(int Nx, int Ny, double pi, const ora_coh_params *P, const ocplx *ukx, const ocplx *uky,
                      int nbins, double *Ek);
void ora_spectrum_com(int Nx, int Ny, double pi, const ora_com_params *P, const ocplx *const state[6], int nbins,
                      double *Ek);

/* ---- 3D MHD (src/derive3com.f95, src/ab3com.f95, time loop src/main3com.f95:536-600) ----
 * arrays: real (Nx,Ny,Nz) a[i + Nx*(j + Ny*k)], complex (Nh,Ny,Nz) a[i + Nh*(j + Ny*k)];
 * fields rho, rho ux, rho uy, rho uz, E, Bx, By, Bz.  Lx, Ly, Lz as the driver
 * holds them (already times pi); mu, CS, eta, dt of COMMON /comm/ (src/main3com.f95:56). */
typedef struct { double Lx, Ly, Lz, mu, CS, eta, dt; } ora_com3_params;
void ora_derive3com(int Nx, int Ny, int Nz, double pi, const ora_com3_params *P, const ocplx *const st[8],
                    ocplx *const dnew[8]);
void ora_ab3com(int Nx, int Ny, int Nz, double dt, const ocplx *const st[8], ocplx *const st_new[8],
                const ocplx *const d_old[8], const ocplx *const d_new[8]);
void ora_run3com(int Nx, int Ny, int Nz, double pi, const ora_com3_params *P, int nsteps, ocplx *const st[8],
                 ocplx *const d_old[8]);

/* number of OpenMP threads the pointwise loops use (0 = runtime default) */
void ora_set_threads(int n);
int  ora_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
