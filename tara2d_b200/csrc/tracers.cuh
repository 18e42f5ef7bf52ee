// Tracer particles of the incompressible vorticity driver (tracers.cu).
#pragma once
#include "models.h"

namespace tara {

// ux, uy (real [Ny][Nx]) = the velocity of the vorticity spectrum omega:
// c2r(i ky psi_k)/(NxNy), c2r(-i kx psi_k)/(NxNy), psi = omega/(k^2 + lam).
// work: 4 spectral fields.
template <class T>
int tracer_velocity_real(const Grid<T>& g, const Cx<T>* omega, T lam, T* ux, T* uy, Cx<T>* const* work,
                         cudaStream_t st);
// np particles (device arrays): velocities at (xp, yp) into vxp, vyp and,
// when move, one forward-Euler step of dt with the positions wrapped.
template <class T>
int tracers_update(const Grid<T>& g, const T* ux, const T* uy, int np, double* xp, double* yp, double* vxp,
                   double* vyp, double dt, bool move, cudaStream_t st);

}  // namespace tara
