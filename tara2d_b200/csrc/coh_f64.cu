// Explicit instantiation of the hydro RHS for double (see coh_impl.cuh).
#include "coh_impl.cuh"

namespace tara {
template int coh_rhs<double>(const Grid<double>&, CohWork<double>&, const CohParamsT<double>&, Cx<double>* const[3],
                          const StepArgs<double>&, cudaStream_t);
}  // namespace tara
