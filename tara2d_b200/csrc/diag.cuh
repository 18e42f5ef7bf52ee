// On-device diagnostics of the drivers: the volume averages written to
// Energy.dat and the shell-averaged kinetic energy spectrum E(k).
//
// MHD (src/main2com.f95:425-616):
//   k_col_inv     y-inverse of rho, rho ux, rho uy, Bx, By, i ky Bx, i ky By
//   k_row_diag    per row: c2r of rho, rho ux, rho uy, Bx, By, div B and j,
//                 u = rho u / rho, the row sums of |u|^2, |B|^2, j^2, div B,
//                 u.B; r2c of ux and uy
//   k_col_fwd_simple (unmasked)  y-forward of ux, uy: the velocity spectra
//   k_spectrum    per ky row: E(k) shells and <omega^2> = sum |omega_k|^2/(NxNy)^2
//                 with omega_k = i kx uy_k - i ky ux_k (Parseval; omega_k is the
//                 spectrum of a real field, so the half-spectrum sum with
//                 weight 2 on 0 < kx index < Nx/2 is the full sum)
//   k_diag_final  fixed-order compensated sums of the per-CTA partials
// Hydro (src/main2coh.f95:321-429):
//   k_col_inv     y-inverse of ux, uy, i ky ux
//   k_row_diag    c2r of ux, uy and omega; row sums of |u|^2, uy^2, 1, omega,
//                 omega^2, omega^3
//   k_spectrum    E(k) of the state velocity spectra
//   k_diag_final
//
// E(k) = sum over k - 1/2 <= |k| < k + 1/2 of (|ux_k|^2 + |uy_k|^2)/2/(NxNy)^2,
// each half-spectrum mode counted twice for 0 < kx index < Nx/2.  All sums are
// in FP64 whatever the field precision.
#pragma once
#include "models.h"

namespace tara {

constexpr int kDiagQ = 8;  // per-CTA partial sums of the row pass

// Diagnostic slots (doubles) of one record: kDiagOut values, then E(k).
constexpr int kDiagOut = 8;

template <class T> struct DiagWork {
  double* part_row = nullptr;   // [row CTAs][kDiagQ]
  double* part_spec = nullptr;  // [Ny]  <omega^2> partials of the spectrum pass
  double* ek_acc = nullptr;     // [nbins] shell accumulators (zero between uses)
  int nbins = 0, row_ctas = 0;
  void* mem = nullptr;
  int alloc(const Grid<T>& g, cudaStream_t st);
  void release();
};

// Shells of E(k): floor(|k| + 1/2) for |k| up to the corner of the grid.
int diag_num_shells(int Nx, int Ny, double Lx, double Ly, double pi);

// Computes one diagnostics record into rec[kDiagOut + nbins] (device memory).
//   out (MHD):   Energy, B_Field, C2 = <omega^2>, C3 = <j^2>, div_B_Tot, <u.B>, 0, 0
//   out (hydro): Energy/2, y_Energy/2, C0, C1, C2, C3, 0, 0 (as written to Energy.dat)
template <class T>
int diag_record(int model, const Grid<T>& g, DiagWork<T>& dw, Cx<T>* const* state, FieldPool<T>& H,
                FieldPool<T>& X, FieldPool<T>& spec, double* rec, cudaStream_t st);

}  // namespace tara
