// Diagnostics kernels (see diag.cuh for the pipeline).
#include <cmath>
#include "diag.cuh"

namespace tara {

namespace {

// Sum of NQ per-thread values over the CTA (any blockDim.x), written by
// thread 0 to out[0..NQ).  Pairwise within warps, then in warp order.
template <int NQ>
__device__ void cta_sum(double (&q)[NQ], double* out) {
  __shared__ double red[32][NQ];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int wsize = min(32, (int)blockDim.x - wid * 32);
  const unsigned mask = wsize == 32 ? 0xffffffffu : ((1u << wsize) - 1u);
#pragma unroll
  for (int k = 0; k < NQ; k++)
    for (int o = 16; o > 0; o >>= 1) {
      const double t = __shfl_down_sync(mask, q[k], o);
      if (lane + o < wsize) q[k] += t;
    }
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NQ; k++) red[wid][k] = q[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) / 32;
    for (int k = 0; k < NQ; k++) {
      double s = 0;
      for (int w = 0; w < nw; w++) s += red[w][k];
      out[k] = s;
    }
  }
}

template <class T> struct RowDiagArgs {
  Tables<T> tb;
  const Cx<T>* H[7];
  Cx<T>* X[2];
  double* part;
  int rb;
};

template <class T, class RF, class SYNC, class HV>
__device__ __forceinline__ void c2r_normalised(Cx<T>* dst, int lane, Cx<T>* v, const Tables<T>& tb, HV&& hv,
                                               SYNC sync) {
  row_c2r<RF>(dst, lane, v, tb, hv, sync);
  sync();
  fft_emit<RF>(lane, v, [&](int, int n, Cx<T> z) { dst[n] = cx<T>(normalise(z.x, tb), normalise(z.y, tb)); });
}

// MHD row pass.  H: 0 rho, 1 rho ux, 2 rho uy, 3 Bx, 4 By, 5 i ky Bx, 6 i ky By
// (half-real).  Six arrays per row: 0 rho -> By, 1 ux, 2 uy, 3 Bx, 4 div B, 5 j.
// Row sums: 0 |u|^2, 1 |B|^2, 2 j^2, 3 div B, 4 u.B     (src/main2com.f95:587-598)
template <class T, int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(4 * (M / P))) k_row_diag_com(const RowDiagArgs<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = 4, ARR = RF::SMEM_ELEMS;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* base = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * 6 * ARR;
  auto arr = [&](int q) { return base + q * ARR; };
  const size_t ro = (size_t)(blockIdx.x * a.rb + th.row) * tb.ld;
  const T* kx = tb.kx;
  Cx<T> v[P];
  {  // rho, rho ux, rho uy, Bx
    const Cx<T>* h = a.H[th.g] + ro;
    c2r_normalised<T, RF>(arr(th.g), th.lane, v, tb, [&](int k) { return ldg(h + k); }, sync);
  }
  __syncthreads();
  for (int m = th.g * NTR + th.lane; m < M; m += G * NTR) {  // u = rho u / rho   (:473-480)
    const Cx<T> r = arr(0)[m], mx = arr(1)[m], my = arr(2)[m];
    arr(1)[m] = cx<T>(mx.x / r.x, mx.y / r.y);
    arr(2)[m] = cx<T>(my.x / r.x, my.y / r.y);
  }
  __syncthreads();
  {  // By, div B = c2r(i kx Bx + i ky By), j = c2r(i kx By - i ky Bx)   (:427-441, :500-540)
    const Cx<T>* hbx = a.H[3] + ro;
    const Cx<T>* hby = a.H[4] + ro;
    const Cx<T>* hkbx = a.H[5] + ro;
    const Cx<T>* hkby = a.H[6] + ro;
    if (th.g == 0) {
      c2r_normalised<T, RF>(arr(0), th.lane, v, tb, [&](int k) { return ldg(hby + k); }, sync);
    } else if (th.g == 1) {
      c2r_normalised<T, RF>(arr(4), th.lane, v, tb,
                            [&](int k) { return ikmul(__ldg(kx + k), ldg(hbx + k)) + ldg(hkby + k); }, sync);
    } else if (th.g == 2) {
      c2r_normalised<T, RF>(arr(5), th.lane, v, tb,
                            [&](int k) { return ikmul(__ldg(kx + k), ldg(hby + k)) - ldg(hkbx + k); }, sync);
    }
  }
  __syncthreads();
  double q[kDiagQ] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int m = th.g * NTR + th.lane; m < M; m += G * NTR) {
    const Cx<T> ux = arr(1)[m], uy = arr(2)[m], bx = arr(3)[m], by = arr(0)[m], db = arr(4)[m], jb = arr(5)[m];
    const double u0 = ux.x, u1 = ux.y, v0 = uy.x, v1 = uy.y, b0 = bx.x, b1 = bx.y, c0 = by.x, c1 = by.y;
    q[0] += (u0 * u0 + v0 * v0) + (u1 * u1 + v1 * v1);
    q[1] += (b0 * b0 + c0 * c0) + (b1 * b1 + c1 * c1);
    q[2] += (double)jb.x * jb.x + (double)jb.y * jb.y;
    q[3] += (double)db.x + (double)db.y;
    q[4] += (u0 * b0 + v0 * c0) + (u1 * b1 + v1 * c1);
  }
  __syncthreads();
  if (th.g < 2) {  // r2c of ux, uy for the vorticity and the spectrum
    const int g = th.g;
    row_r2c_begin<RF>(th.lane, v, tb, [&](int n) { return arr(1 + g)[n]; });
    Cx<T>* xo = a.X[g] + ro;
    row_r2c_finish<RF>(arr(3 + g), th.lane, NTR, v, tb, [&](int k, Cx<T> X) { st(xo + k, X); }, sync);
  }
  cta_sum<kDiagQ>(q, a.part + (size_t)blockIdx.x * kDiagQ);
}

// Hydro row pass.  H: 0 ux, 1 uy, 2 i ky ux.  Arrays: 0 ux, 1 uy, 2 omega.
// Row sums: 0 |u|^2, 1 uy^2, 2 count, 3 omega, 4 omega^2, 5 omega^3
// (src/main2coh.f95:321-429)
template <class T, int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(3 * (M / P))) k_row_diag_coh(const RowDiagArgs<T> a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = 3, ARR = RF::SMEM_ELEMS;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<T>& tb = a.tb;
  Cx<T>* base = reinterpret_cast<Cx<T>*>(smraw) + (size_t)th.row * 3 * ARR;
  auto arr = [&](int q) { return base + q * ARR; };
  const size_t ro = (size_t)(blockIdx.x * a.rb + th.row) * tb.ld;
  const T* kx = tb.kx;
  Cx<T> v[P];
  {
    const Cx<T>* hux = a.H[0] + ro;
    const Cx<T>* huy = a.H[1] + ro;
    const Cx<T>* hkux = a.H[2] + ro;
    const int g = th.g;
    c2r_normalised<T, RF>(arr(g), th.lane, v, tb, [&](int k) -> Cx<T> {
      if (g == 0) return ldg(hux + k);
      if (g == 1) return ldg(huy + k);
      return ikmul(__ldg(kx + k), ldg(huy + k)) - ldg(hkux + k);  // omega = i kx uy - i ky ux
    }, sync);
  }
  __syncthreads();
  double q[kDiagQ] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int m = th.g * NTR + th.lane; m < M; m += G * NTR) {
    const Cx<T> ux = arr(0)[m], uy = arr(1)[m], w = arr(2)[m];
    const double u[2] = {ux.x, ux.y}, vv[2] = {uy.x, uy.y}, om[2] = {w.x, w.y};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      q[0] += u[h] * u[h] + vv[h] * vv[h];
      q[1] += vv[h] * vv[h];
      q[2] += 1.0;
      q[3] += om[h];
      q[4] += om[h] * om[h];
      q[5] += om[h] * om[h] * om[h];
    }
  }
  cta_sum<kDiagQ>(q, a.part + (size_t)blockIdx.x * kDiagQ);
}

template <class T> struct SpecArgs {
  Tables<T> tb;
  const Cx<T>* ux;
  const Cx<T>* uy;
  double* ek_acc;
  double* part;   // per row: sum of w |omega_k|^2 (vort != 0)
  int nbins, vort;
};

__device__ __forceinline__ int shell_of(double kx, double ky) { return (int)floor(sqrt(kx * kx + ky * ky) + 0.5); }

// One CTA per ky row; the row's shells form one contiguous range.
template <class T>
__global__ void __launch_bounds__(256) k_spectrum(const SpecArgs<T> a) {
  extern __shared__ double bins[];
  const int j = blockIdx.x;
  const int Nh = a.tb.Nh, Nx = a.tb.Nx;
  const double ky = (double)a.tb.ky[j];
  const int s_lo = shell_of((double)a.tb.kx[0], ky);
  const int s_hi = min(shell_of((double)a.tb.kx[Nh - 1], ky), a.nbins - 1);
  const int nb = s_hi - s_lo + 1;
  for (int s = threadIdx.x; s < nb; s += blockDim.x) bins[s] = 0.0;
  __syncthreads();
  double qv[1] = {0.0};
  const size_t ro = (size_t)j * a.tb.ld;
  for (int i = threadIdx.x; i < Nh; i += blockDim.x) {
    const Cx<T> X = ldg(a.ux + ro + i), Y = ldg(a.uy + ro + i);
    const double wgt = (i > 0 && i < Nx / 2) ? 2.0 : 1.0;
    const double x0 = X.x, x1 = X.y, y0 = Y.x, y1 = Y.y;
    const double kx = (double)a.tb.kx[i];
    const int s = shell_of(kx, ky);
    if (s <= s_hi) atomicAdd(&bins[s - s_lo], 0.5 * wgt * ((x0 * x0 + x1 * x1) + (y0 * y0 + y1 * y1)));
    if (a.vort) {
      // omega_k = i kx uy_k - i ky ux_k
      const double o0 = -(kx * y1) + ky * x1, o1 = kx * y0 - ky * x0;
      qv[0] += wgt * (o0 * o0 + o1 * o1);
    }
  }
  __syncthreads();
  for (int s = threadIdx.x; s < nb; s += blockDim.x) atomicAdd(a.ek_acc + s_lo + s, bins[s]);
  if (a.vort) cta_sum<1>(qv, a.part + j);
}

// Neumaier-compensated sum of n values with stride st
__device__ double comp_sum(const double* p, int n, int stride) {
  double s = 0.0, c = 0.0;
  for (int k = 0; k < n; k++) {
    const double x = p[(size_t)k * stride];
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  return s + c;
}

struct FinalArgs {
  const double* part_row;
  const double* part_spec;
  double* ek_acc;
  double* rec;
  int row_ctas, ny, nbins, model;
  double nn;
};

__global__ void k_diag_final(const FinalArgs a) {
  __shared__ double sums[kDiagQ + 1];
  const int t = threadIdx.x;
  if (t < kDiagQ) sums[t] = comp_sum(a.part_row + t, a.row_ctas, kDiagQ);
  if (t == kDiagQ) sums[t] = a.model == TARA_MODEL_COM ? comp_sum(a.part_spec, a.ny, 1) : 0.0;
  __syncthreads();
  const double nn = a.nn;
  if (t == 0) {
    double* o = a.rec;
    if (a.model == TARA_MODEL_COM) {
      o[0] = sums[0] / nn;         // Energy
      o[1] = sums[1] / nn;         // B_Field
      o[2] = sums[kDiagQ] / nn / nn;  // C2 = <omega^2>
      o[3] = sums[2] / nn;         // C3 = <j^2>
      o[4] = sums[3] / nn;         // div_B_Tot
      o[5] = sums[4] / nn;         // <u.B>
    } else {
      o[0] = sums[0] / (2.0 * nn);  // Energy/(2 NxNy)
      o[1] = sums[1] / (2.0 * nn);  // y_Energy/(2 NxNy)
      o[2] = sums[2] / nn;          // C0
      o[3] = sums[3] / nn;          // C1
      o[4] = sums[4] / nn;          // C2
      o[5] = sums[5] / nn;          // C3
    }
    o[6] = 0.0;
    o[7] = 0.0;
  }
  for (int s = t; s < a.nbins; s += blockDim.x) {
    a.rec[kDiagOut + s] = a.ek_acc[s] / nn / nn;
    a.ek_acc[s] = 0.0;
  }
}

template <int Nx, class T>
void launch_row_diag(int model, const RowDiagArgs<T>& a0, int Ny, int& ctas, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  const int G = model == TARA_MODEL_COM ? 4 : 3, NA = model == TARA_MODEL_COM ? 6 : 3;
  RowDiagArgs<T> a = a0;
  const size_t per_row = (size_t)NA * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<T>);
  a.rb = 1;
  while (a.rb * 2 * G * NTR <= 128 && Ny % (a.rb * 2) == 0 && (a.rb * 2) * per_row <= 110 * 1024) a.rb *= 2;
  const size_t smem = per_row * a.rb;
  ctas = Ny / a.rb;
  if (model == TARA_MODEL_COM) {
    auto kern = k_row_diag_com<T, M, P>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<ctas, G * NTR * a.rb, smem, st>>>(a);
  } else {
    auto kern = k_row_diag_coh<T, M, P>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<ctas, G * NTR * a.rb, smem, st>>>(a);
  }
}

}  // namespace

int diag_num_shells(int Nx, int Ny, double Lx, double Ly, double pi) {
  std::vector<double> kx, ky;
  std::vector<int> cut;
  wavenumbers(Nx, Ny, Lx, Ly, pi, kx, ky, cut);
  const double kxm = kx[Nx / 2], kym = std::fabs(ky[Ny / 2]);
  return (int)std::floor(std::sqrt(kxm * kxm + kym * kym) + 0.5) + 1;
}

template <class T>
int DiagWork<T>::alloc(const Grid<T>& g, cudaStream_t st) {
  nbins = diag_num_shells(g.Nx, g.Ny, g.Lx, g.Ly, g.pi);
  const size_t n = (size_t)g.Ny * kDiagQ + (size_t)g.Ny + (size_t)nbins;
  if (cudaMalloc(&mem, n * sizeof(double)) != cudaSuccess) {
    mem = nullptr;
    set_error("cudaMalloc of diagnostics buffers failed");
    return TARA_ENOMEM;
  }
  part_row = (double*)mem;
  part_spec = part_row + (size_t)g.Ny * kDiagQ;
  ek_acc = part_spec + g.Ny;
  TARA_CUDA_TRY(cudaMemsetAsync(mem, 0, n * sizeof(double), st));
  return TARA_OK;
}

template <class T>
void DiagWork<T>::release() {
  if (mem) cudaFree(mem);
  mem = nullptr;
  part_row = part_spec = ek_acc = nullptr;
}

template <class T>
int diag_record(int model, const Grid<T>& g, DiagWork<T>& dw, Cx<T>* const* state, FieldPool<T>& H,
                FieldPool<T>& X, FieldPool<T>& spec, double* rec, cudaStream_t st) {
  if (model != TARA_MODEL_COM && model != TARA_MODEL_COH) {
    set_error("diagnostics are defined for the hydro and MHD models");
    return TARA_EUNSUPPORTED;
  }
  const bool com = model == TARA_MODEL_COM;
  const int NA = com ? 6 : 3;
  if ((size_t)NA * (g.Nx / 2 + g.Nx / 32 + 1) * sizeof(Cx<T>) > 220 * 1024) {
    set_error("diagnostics row pass does not fit in shared memory at this Nx and precision");
    return TARA_EUNSUPPORTED;
  }
  ColInvArgs<T> ci{};
  ci.tb = g.tb;
  int njobs;
  if (com) {
    // rho, rho ux, rho uy, Bx, By, i ky Bx, i ky By
    const int src[7] = {0, 1, 2, 4, 5, 4, 5};
    const int mul[7] = {MUL_ONE, MUL_ONE, MUL_ONE, MUL_ONE, MUL_ONE, MUL_IKY, MUL_IKY};
    for (int q = 0; q < 7; q++) ci.job[q] = ColInvJob<T>{state[src[q]], H[q], mul[q], (T)0};
    njobs = 7;
  } else {
    // ux, uy, i ky ux
    ci.job[0] = ColInvJob<T>{state[1], H[0], MUL_ONE, (T)0};
    ci.job[1] = ColInvJob<T>{state[2], H[1], MUL_ONE, (T)0};
    ci.job[2] = ColInvJob<T>{state[1], H[2], MUL_IKY, (T)0};
    njobs = 3;
  }
  run_col_inv(ci, njobs, st);

  RowDiagArgs<T> ra{};
  ra.tb = g.tb;
  for (int q = 0; q < njobs; q++) ra.H[q] = H[q];
  ra.X[0] = X[0];
  ra.X[1] = X[1];
  ra.part = dw.part_row;
  int ctas = 0;
  TARA_DISPATCH_LEN(g.Nx, launch_row_diag, model, ra, g.Ny, ctas, st)
  dw.row_ctas = ctas;

  SpecArgs<T> sa{};
  sa.tb = g.tb;
  if (com) {
    // velocity spectra: plain forward y transform of the x-transformed rows
    ColFwdSimpleArgs<T> cf{};
    cf.tb = g.tb;
    cf.X[0] = X[0];
    cf.X[1] = X[1];
    cf.sign[0] = cf.sign[1] = (T)1;
    cf.nomask = 1;
    cf.step.mode = STEP_RHS;
    cf.step.out[0] = spec[0];
    cf.step.out[1] = spec[1];
    run_col_fwd_simple(cf, 2, st);
    sa.ux = spec[0];
    sa.uy = spec[1];
  } else {
    sa.ux = state[1];
    sa.uy = state[2];
  }
  sa.ek_acc = dw.ek_acc;
  sa.part = dw.part_spec;
  sa.nbins = dw.nbins;
  sa.vort = com ? 1 : 0;
  k_spectrum<T><<<g.Ny, 256, (size_t)dw.nbins * sizeof(double), st>>>(sa);

  FinalArgs fa{};
  fa.part_row = dw.part_row;
  fa.part_spec = dw.part_spec;
  fa.ek_acc = dw.ek_acc;
  fa.rec = rec;
  fa.row_ctas = ctas;
  fa.ny = g.Ny;
  fa.nbins = dw.nbins;
  fa.model = model;
  fa.nn = (double)g.Nx * (double)g.Ny;
  k_diag_final<<<1, 256, 0, st>>>(fa);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

template struct DiagWork<double>;
template struct DiagWork<float>;
template int diag_record<double>(int, const Grid<double>&, DiagWork<double>&, Cx<double>* const*,
                                 FieldPool<double>&, FieldPool<double>&, FieldPool<double>&, double*, cudaStream_t);
template int diag_record<float>(int, const Grid<float>&, DiagWork<float>&, Cx<float>* const*, FieldPool<float>&,
                                FieldPool<float>&, FieldPool<float>&, double*, cudaStream_t);

}  // namespace tara
