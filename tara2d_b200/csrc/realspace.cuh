// Real-space views of a session's state: the state fields after a normalised
// c2r (what every reference driver computes before its diagnostics and file
// output, src/main2com.f95:446-480, src/main2coh.f95:321-360), the vorticity,
// and the inverse: a state from real-space fields (the drivers' initial
// condition path, src/main2com.f95:257-262).
#pragma once
#include "xform.cuh"

namespace tara {

// real[q] = c2r(state[q]) / (Nx Ny), q < nf (nf <= 6); work: nf fields
template <class T>
int state_to_real(const Grid<T>& g, int nf, Cx<T>* const* state, T* const* real, Cx<T>* const* work,
                  cudaStream_t st);
// state[q] = r2c(real[q]), q < nf; work: nf fields
template <class T>
int real_to_state(const Grid<T>& g, int nf, const T* const* real, Cx<T>* const* state, Cx<T>* const* work,
                  cudaStream_t st);
// omega = c2r(i kx uy_k - i ky ux_k) / (Nx Ny), the velocity spectra being the
// state (hydro) or r2c of (rho u)/rho (MHD).  rtmp: 3 real fields; work: 3
// spectral fields.
template <class T>
int vorticity_real(const Grid<T>& g, int model, Cx<T>* const* state, T* omega, T* const* rtmp,
                   Cx<T>* const* work, cudaStream_t st);
// FP64 host-layout staging <-> field precision, n values
template <class T> void copy_to_real(const double* src, T* dst, size_t n, cudaStream_t st);
template <class T> void copy_from_real(const T* src, double* dst, size_t n, cudaStream_t st);

}  // namespace tara
