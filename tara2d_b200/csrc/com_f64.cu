// Explicit instantiation of the MHD RHS for double (see com_impl.cuh).
#include "com_impl.cuh"

namespace tara {
template int com_rhs<double>(const Grid<double>&, ComWork<double>&, const ComParamsT<double>&, Cx<double>* const[6],
                         const StepArgs<double>&, cudaStream_t);
}  // namespace tara
