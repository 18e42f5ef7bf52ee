#include "models.h"
namespace tara {
template <class T>
int vort_rhs(const Grid<T>&, VortWork<T>&, const VortParamsT<T>&, Cx<T>* const[1], const StepArgs<T>&, cudaStream_t) {
  set_error("not built yet"); return TARA_EUNSUPPORTED;
}
template int vort_rhs<double>(const Grid<double>&, VortWork<double>&, const VortParamsT<double>&, Cx<double>* const[1], const StepArgs<double>&, cudaStream_t);
template int vort_rhs<float>(const Grid<float>&, VortWork<float>&, const VortParamsT<float>&, Cx<float>* const[1], const StepArgs<float>&, cudaStream_t);
}
