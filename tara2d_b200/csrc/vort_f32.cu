// Explicit instantiation of the vorticity RHS for float (see vort_impl.cuh).
#include "vort_impl.cuh"

namespace tara {
template int vort_rhs<float>(const Grid<float>&, VortWork<float>&, const VortParamsT<float>&, Cx<float>* const[1],
                          const StepArgs<float>&, cudaStream_t);
}  // namespace tara
