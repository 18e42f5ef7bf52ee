// Learned subgrid closure of the MHD path: the pieces the session needs.
#pragma once
#include "plan.h"

namespace tara {

// coarse grid size of the closure
int closure_grid(const tara_closure* c);
// Spectra of the predicted subgrid stress (xx, xy, yy) and EMF for the RHS
// input `in` (six MHD state spectra on the closure's coarse grid g), written
// to out4 on stream st.  Launches only (graph-capturable).
int closure_terms(tara_closure* c, const Grid<double>& g, Cx<double>* const* in, Cx<double>* const* out4,
                  cudaStream_t st);

// The state of FP64 MHD ensemble member m (ensemble.cu): its grid, its six
// spectral state fields and the ensemble's stream.  TARA_EINVAL for another
// model or precision.
int ens_member_state(tara_ensemble* e, int m, const Grid<double>** g, Cx<double>** state6, cudaStream_t* st);

}  // namespace tara
