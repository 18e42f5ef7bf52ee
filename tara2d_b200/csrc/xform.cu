// Plain 2D real transforms (see xform.cuh): the column passes of the RHS
// kernels plus one row kernel per direction, one thread group per row.
#include "xform.cuh"

namespace tara {

namespace {

template <class T> struct RowPlainArgs {
  Tables<T> tb;
  const Cx<T>* src[8];
  Cx<T>* dst[8];
  int rb, normalise;
};

// c2r along x of half-real rows (src, pitch ld) into real rows (dst viewed
// as Nx/2 complex pairs per row)
template <class T, int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(M / P)) k_row_c2r_plain(const RowPlainArgs<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, 1> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* xs = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * RF::SMEM_ELEMS;
  const int y = blockIdx.x * a.rb + th.row;
  const Cx<T>* h = a.src[blockIdx.y] + (size_t)y * tb.ld;
  Cx<T>* out = a.dst[blockIdx.y] + (size_t)y * M;
  Cx<T> v[P];
  row_c2r<RF>(xs, th.lane, v, tb, [&](int k) { return ldg(h + k); }, sync);
  fft_emit<RF>(th.lane, v, [&](int, int n, Cx<T> z) {
    st(out + n, a.normalise ? cx<T>(normalise(z.x, tb), normalise(z.y, tb)) : z);
  });
}

// r2c along x of real rows (src as Nx/2 complex pairs per row) into
// x-transformed rows (dst, pitch ld)
template <class T, int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(M / P)) k_row_r2c_plain(const RowPlainArgs<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, 1> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* xs = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * RF::SMEM_ELEMS;
  const int y = blockIdx.x * a.rb + th.row;
  const Cx<T>* in = a.src[blockIdx.y] + (size_t)y * M;
  Cx<T>* xo = a.dst[blockIdx.y] + (size_t)y * tb.ld;
  Cx<T> v[P];
  row_r2c_begin<RF>(th.lane, v, tb, [&](int n) { return ldg(in + n); });
  row_r2c_finish<RF>(xs, th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
}

template <int Nx, class T>
void launch_row_plain(bool inverse, const RowPlainArgs<T>& a0, int nf, int Ny, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  RowPlainArgs<T> a = a0;
  const size_t per_row = (size_t)RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>);
  a.rb = 1;
  while (a.rb * 2 * NTR <= 128 && Ny % (a.rb * 2) == 0 && (a.rb * 2) * per_row <= 96 * 1024) a.rb *= 2;
  const size_t smem = per_row * a.rb;
  const dim3 grid(Ny / a.rb, nf);
  if (inverse) {
    auto kern = k_row_c2r_plain<T, M, P>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<grid, NTR * a.rb, smem, st>>>(a);
  } else {
    auto kern = k_row_r2c_plain<T, M, P>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<grid, NTR * a.rb, smem, st>>>(a);
  }
}

}  // namespace

template <class T>
int c2r_fields(const Grid<T>& g, int nf, const Cx<T>* const* spec, T* const* real, Cx<T>* const* work,
               bool normalise, cudaStream_t st) {
  if (nf < 1 || nf > 8) { set_error("1..8 fields per transform call"); return TARA_EINVAL; }
  ColInvArgs<T> ci{};
  ci.tb = g.tb;
  for (int q = 0; q < nf; q++) ci.job[q] = ColInvJob<T>{spec[q], work[q], MUL_ONE, (T)0};
  run_col_inv(ci, nf, st);
  RowPlainArgs<T> ra{};
  ra.tb = g.tb;
  ra.normalise = normalise ? 1 : 0;
  for (int q = 0; q < nf; q++) {
    ra.src[q] = work[q];
    ra.dst[q] = reinterpret_cast<Cx<T>*>(real[q]);
  }
  TARA_DISPATCH_LEN(g.Nx, launch_row_plain, true, ra, nf, g.Ny, st)
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

template <class T>
int r2c_fields(const Grid<T>& g, int nf, const T* const* real, Cx<T>* const* spec, Cx<T>* const* work,
               cudaStream_t st) {
  if (nf < 1 || nf > 6) { set_error("1..6 fields per forward transform call"); return TARA_EINVAL; }
  RowPlainArgs<T> ra{};
  ra.tb = g.tb;
  for (int q = 0; q < nf; q++) {
    ra.src[q] = reinterpret_cast<const Cx<T>*>(real[q]);
    ra.dst[q] = work[q];
  }
  TARA_DISPATCH_LEN(g.Nx, launch_row_plain, false, ra, nf, g.Ny, st)
  ColFwdSimpleArgs<T> cf{};
  cf.tb = g.tb;
  cf.nomask = 1;
  cf.step.mode = STEP_RHS;
  for (int q = 0; q < nf; q++) {
    cf.X[q] = work[q];
    cf.sign[q] = (T)1;
    cf.step.out[q] = spec[q];
  }
  run_col_fwd_simple(cf, nf, st);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

template int c2r_fields<double>(const Grid<double>&, int, const Cx<double>* const*, double* const*,
                                Cx<double>* const*, bool, cudaStream_t);
template int c2r_fields<float>(const Grid<float>&, int, const Cx<float>* const*, float* const*, Cx<float>* const*,
                               bool, cudaStream_t);
template int r2c_fields<double>(const Grid<double>&, int, const double* const*, Cx<double>* const*,
                                Cx<double>* const*, cudaStream_t);
template int r2c_fields<float>(const Grid<float>&, int, const float* const*, Cx<float>* const*, Cx<float>* const*,
                               cudaStream_t);

}  // namespace tara
