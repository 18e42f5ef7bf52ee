// Explicit instantiation of the MHD RHS for float (see com_impl.cuh).
#include "com_impl.cuh"

namespace tara {
template int com_rhs<float>(const Grid<float>&, ComWork<float>&, const ComParamsT<float>&, Cx<float>* const[6],
                         const StepArgs<float>&, cudaStream_t);
}  // namespace tara
