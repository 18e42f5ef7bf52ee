// Real-space views of the state (see realspace.cuh).
#include "realspace.cuh"

namespace tara {

namespace {

template <class T>
__global__ void k_quotient(const T* __restrict__ num0, const T* __restrict__ num1, const T* __restrict__ den,
                           T* out0, T* out1, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const T r = den[q];
    out0[q] = num0[q] / r;
    out1[q] = num1[q] / r;
  }
}

// omega_k = i kx uy_k - i ky ux_k into w (may alias neither input)
template <class T>
__global__ void k_curl_spec(Tables<T> tb, const Cx<T>* __restrict__ ux, const Cx<T>* __restrict__ uy, Cx<T>* w) {
  const size_t n = (size_t)tb.Nh * tb.Ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(q / tb.Nh), i = (int)(q % tb.Nh);
    const size_t o = (size_t)j * tb.ld + i;
    w[o] = ikmul(__ldg(tb.kx + i), ldg(uy + o)) - ikmul(__ldg(tb.ky + j), ldg(ux + o));
  }
}

template <class T>
__global__ void k_to_real(const double* __restrict__ s, T* d, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    d[q] = (T)s[q];
}
template <class T>
__global__ void k_from_real(const T* __restrict__ s, double* d, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    d[q] = (double)s[q];
}

}  // namespace

template <class T>
int state_to_real(const Grid<T>& g, int nf, Cx<T>* const* state, T* const* real, Cx<T>* const* work,
                  cudaStream_t st) {
  const Cx<T>* src[8];
  for (int q = 0; q < nf; q++) src[q] = state[q];
  return c2r_fields(g, nf, src, real, work, true, st);
}

template <class T>
int real_to_state(const Grid<T>& g, int nf, const T* const* real, Cx<T>* const* state, Cx<T>* const* work,
                  cudaStream_t st) {
  return r2c_fields(g, nf, real, state, work, st);
}

template <class T>
int vorticity_real(const Grid<T>& g, int model, Cx<T>* const* state, T* omega, T* const* rtmp, Cx<T>* const* work,
                   cudaStream_t st) {
  const size_t nn = (size_t)g.Nx * g.Ny;
  const Cx<T>* ux;
  const Cx<T>* uy;
  if (model == TARA_MODEL_COM) {
    // u = (rho u)/rho in real space, then its spectrum   (src/main2com.f95:473-480, 500-520)
    TARA_TRY(state_to_real(g, 3, state, rtmp, work, st));
    k_quotient<T><<<592, 256, 0, st>>>(rtmp[1], rtmp[2], rtmp[0], rtmp[1], rtmp[2], nn);
    const T* r[2] = {rtmp[1], rtmp[2]};
    Cx<T>* s[2] = {work[0], work[1]};
    // one field at a time, work[2] holding the x-transformed rows
    TARA_TRY(r2c_fields(g, 1, r, s, work + 2, st));
    TARA_TRY(r2c_fields(g, 1, r + 1, s + 1, work + 2, st));
    ux = work[0];
    uy = work[1];
  } else if (model == TARA_MODEL_COH) {
    ux = state[1];
    uy = state[2];
  } else {
    set_error("vorticity output is defined for the hydro and MHD models");
    return TARA_EUNSUPPORTED;
  }
  k_curl_spec<T><<<592, 256, 0, st>>>(g.tb, ux, uy, work[2]);
  TARA_CUDA_TRY(cudaGetLastError());
  const Cx<T>* w[1] = {work[2]};
  T* o[1] = {omega};
  Cx<T>* wk[1] = {work[0]};
  return c2r_fields(g, 1, w, o, wk, true, st);
}

template <class T> void copy_to_real(const double* src, T* dst, size_t n, cudaStream_t st) {
  k_to_real<T><<<592, 256, 0, st>>>(src, dst, n);
}
template <class T> void copy_from_real(const T* src, double* dst, size_t n, cudaStream_t st) {
  k_from_real<T><<<592, 256, 0, st>>>(src, dst, n);
}

#define TARA_RS_INST(T)                                                                                         \
  template int state_to_real<T>(const Grid<T>&, int, Cx<T>* const*, T* const*, Cx<T>* const*, cudaStream_t);  \
  template int real_to_state<T>(const Grid<T>&, int, const T* const*, Cx<T>* const*, Cx<T>* const*,            \
                                cudaStream_t);                                                                  \
  template int vorticity_real<T>(const Grid<T>&, int, Cx<T>* const*, T*, T* const*, Cx<T>* const*, cudaStream_t); \
  template void copy_to_real<T>(const double*, T*, size_t, cudaStream_t);                                      \
  template void copy_from_real<T>(const T*, double*, size_t, cudaStream_t);
TARA_RS_INST(double)
TARA_RS_INST(float)
#undef TARA_RS_INST

}  // namespace tara
