// Explicit instantiation of the vorticity RHS for double (see vort_impl.cuh).
#include "vort_impl.cuh"

namespace tara {
template int vort_rhs<double>(const Grid<double>&, VortWork<double>&, const VortParamsT<double>&, Cx<double>* const[1],
                          const StepArgs<double>&, cudaStream_t);
}  // namespace tara
