// Explicit instantiation of the hydro RHS for float (see coh_impl.cuh).
#include "coh_impl.cuh"

namespace tara {
template int coh_rhs<float>(const Grid<float>&, CohWork<float>&, const CohParamsT<float>&, Cx<float>* const[3],
                          const StepArgs<float>&, cudaStream_t);
}  // namespace tara
