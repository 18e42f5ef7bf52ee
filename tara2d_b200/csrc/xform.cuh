// Plain 2D real transforms between device spectral fields ([Ny][ld] complex)
// and device real fields ([Ny][Nx], rows contiguous), with the reference's
// FFTW semantics (unnormalised forward transform; c2r optionally divided by
// Nx*Ny as every reference caller does after a c2r).
#pragma once
#include "models.h"

namespace tara {

// nf fields, nf <= 8.  work: nf half-real / x-transformed fields ([Ny][ld]).
template <class T>
int c2r_fields(const Grid<T>& g, int nf, const Cx<T>* const* spec, T* const* real, Cx<T>* const* work,
               bool normalise, cudaStream_t st);
template <class T>
int r2c_fields(const Grid<T>& g, int nf, const T* const* real, Cx<T>* const* spec, Cx<T>* const* work,
               cudaStream_t st);

}  // namespace tara
