// Seeded initial conditions built on the device (ic.cu).
#pragma once
#include "models.h"

namespace tara {

// The real-space state fields of initial condition `ic` into r[0..nf) (nf of
// the model; r holds at least 6 fields).  work: 4 spectral fields.
template <class T>
int ic_random_state(const Grid<T>& g, int model, const tara_params& p, const tara_ic& ic, T* const* r,
                    Cx<T>* const* work, cudaStream_t st);

}  // namespace tara
