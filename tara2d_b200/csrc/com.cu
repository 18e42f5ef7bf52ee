#include "models.h"
namespace tara {
template <class T>
int com_rhs(const Grid<T>&, ComWork<T>&, const ComParamsT<T>&, Cx<T>* const[6], const StepArgs<T>&, cudaStream_t) {
  set_error("not built yet"); return TARA_EUNSUPPORTED;
}
template int com_rhs<double>(const Grid<double>&, ComWork<double>&, const ComParamsT<double>&, Cx<double>* const[6], const StepArgs<double>&, cudaStream_t);
template int com_rhs<float>(const Grid<float>&, ComWork<float>&, const ComParamsT<float>&, Cx<float>* const[6], const StepArgs<float>&, cudaStream_t);
template <class T>
int vort_rhs(const Grid<T>&, VortWork<T>&, const VortParamsT<T>&, Cx<T>* const[1], const StepArgs<T>&, cudaStream_t) {
  set_error("not built yet"); return TARA_EUNSUPPORTED;
}
template int vort_rhs<double>(const Grid<double>&, VortWork<double>&, const VortParamsT<double>&, Cx<double>* const[1], const StepArgs<double>&, cudaStream_t);
template int vort_rhs<float>(const Grid<float>&, VortWork<float>&, const VortParamsT<float>&, Cx<float>* const[1], const StepArgs<float>&, cudaStream_t);
}
