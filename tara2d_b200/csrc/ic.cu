// Seeded initial conditions of the benchmark configurations, built on the
// device.  The reference builds its initial states on the host and
// transforms them with FFTW r2c (src/main2coh.f95:141-222,
// src/main2com.f95:230-300); the configurations replace its point-vortex /
// uniform-B profiles with seeded random-phase and Orszag-Tang states.
//
// Random numbers: value = mix(mix(seed ^ stream * C1) + (index + 1) * C2),
// mix = the splitmix64 finaliser (S. Vigna, public domain: xor-shift 30,
// multiply, xor-shift 27, multiply, xor-shift 31), C1 = 0xD1B54A32D192ED03,
// C2 = 0x9E3779B97F4A7C15; uniform u = (value >> 11) * 2^-53.  Every value
// depends only on (seed, stream, index), so the host restatement in
// tara2d_b200/initial.py (hashed_*) reproduces the same fields.
//
// Solenoidal random-phase field (stream s): on every half-spectrum mode
// (kx index i < Nx/2+1, ky index j) psi_k = a(|k|) e^{2 pi i u(s, j*Nh + i)}
// with a = sqrt(E(|k|)/|k|^3) (E the shell spectrum, a = 0 at k = 0 and
// outside [kmin, kmax]); u = c2r(i ky psi_k)/(NxNy), v = c2r(-i kx psi_k)/(NxNy)
// (the imaginary parts of the kx = 0 and Nyquist bins are dropped by the
// c2r, as in FFTW), then scaled to the requested energy or rms (FP64 sums).
#include <vector>
#include "ic.cuh"
#include "realspace.cuh"
#include "xform.cuh"

namespace tara {

namespace {

__host__ __device__ inline unsigned long long ic_mix(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ inline double ic_u01(unsigned long long seed, unsigned long long stream, unsigned long long index) {
  const unsigned long long key = ic_mix(seed ^ (stream * 0xD1B54A32D192ED03ull));
  return (double)(ic_mix(key + (index + 1) * 0x9E3779B97F4A7C15ull) >> 11) * 0x1.0p-53;
}

constexpr double kTwoPi = 6.283185307179586476925286766559;
enum : int { SHAPE_PEAKED = 0, SHAPE_FLAT = 1 };  // E(k) = k^4 exp(-(k/k0)^2) ; E(k) = k

// i ky psi_k and -i kx psi_k of the random-phase streamfunction, [Ny][ld]
template <class T>
__global__ void k_ic_modes(Tables<T> tb, unsigned long long seed, unsigned long long stream, int shape, double k0,
                           double kmin, double kmax, Cx<T>* A, Cx<T>* B) {
  const int Nh = tb.Nh, ld = tb.ld;
  const size_t n = (size_t)tb.Ny * Nh;
  for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < n; m += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(m % Nh), j = (int)(m / Nh);
    const double kx = tb.kx[i], ky = tb.ky[j];
    const double k = sqrt(kx * kx + ky * ky);
    double amp = 0.0;
    if (k > 0.0 && k >= kmin && k <= kmax) {
      const double e = shape == SHAPE_PEAKED ? k * k * k * k * exp(-(k / k0) * (k / k0)) : k;
      amp = sqrt(e / (k * k * k));
    }
    double s, c;
    sincos(kTwoPi * ic_u01(seed, stream, m), &s, &c);
    const double px = amp * c, py = amp * s;
    A[(size_t)j * ld + i] = cx<T>((T)(-ky * py), (T)(ky * px));
    B[(size_t)j * ld + i] = cx<T>((T)(kx * py), (T)(-kx * px));
  }
}

constexpr int kSumBlocks = 256, kSumThreads = 256;
// partial sums of a^2 + b^2 over n points, one per block (fixed order)
template <class T>
__global__ void __launch_bounds__(kSumThreads) k_ic_sumsq(const T* a, const T* b, size_t n, double* part) {
  __shared__ double red[kSumThreads];
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)kSumThreads + threadIdx.x; k < n; k += (size_t)kSumBlocks * kSumThreads) {
    const double x = a[k], y = b[k];
    s += x * x + y * y;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

struct IcAssembly {
  int model, kind;
  int Nx, Ny;
  double dx, dy;
  unsigned long long seed;
  double su, sb;     // scales of the random fields (u; B)
  double noise;      // hydro density noise
  double cs2, gam1;  // CS^2, spheat - 1
};

// Real-space state from the (unscaled) random fields, in place: hydro
// r[1], r[2] = u -> (n, ux, uy); MHD r[1], r[2] = u, r[4], r[5] = B ->
// (rho, rho ux, rho uy, E, Bx, By) with P = CS^2 rho and
// E = P/(spheat-1) + rho |u|^2/2 + |B|^2/2 (src/main2com.f95:247-255).
template <class T>
__global__ void k_ic_assemble(IcAssembly a, T* r0, T* r1, T* r2, T* r3, T* r4, T* r5) {
  const size_t n = (size_t)a.Nx * a.Ny;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    if (a.model == TARA_MODEL_COH) {
      // density 1 + noise * N(0,1), Box-Muller from two uniforms of stream 3
      const double u1 = 1.0 - ic_u01(a.seed, 3, 2 * k), u2 = ic_u01(a.seed, 3, 2 * k + 1);
      const double g = sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2);
      r0[k] = (T)(1.0 + a.noise * g);
      r1[k] = (T)(a.su * (double)r1[k]);
      r2[k] = (T)(a.su * (double)r2[k]);
      continue;
    }
    double ux = a.su * (double)r1[k], uy = a.su * (double)r2[k];
    double bx = a.sb * (double)r4[k], by = a.sb * (double)r5[k];
    if (a.kind == TARA_IC_ORSZAG_TANG) {  // u = (-sin y, sin x), B = (-sin y, sin 2x) + perturbations
      const double x = (double)(k % a.Nx) * a.dx, y = (double)(k / a.Nx) * a.dy;
      ux += -sin(y);
      uy += sin(x);
      bx += -sin(y);
      by += sin(2.0 * x);
    }
    const double rho = 1.0, P = a.cs2 * rho;
    const double E = P / a.gam1 + 0.5 * rho * (ux * ux + uy * uy) + 0.5 * (bx * bx + by * by);
    r0[k] = (T)rho;
    r1[k] = (T)(rho * ux);
    r2[k] = (T)(rho * uy);
    r3[k] = (T)E;
    r4[k] = (T)bx;
    r5[k] = (T)by;
  }
}

// random solenoidal field of stream `stream` into real ru, rv; returns
// mean(u^2 + v^2) (FP64)
template <class T>
int solenoidal(const Grid<T>& g, unsigned long long seed, int stream, int shape, double k0, double kmin, double kmax,
               T* ru, T* rv, Cx<T>* const* work, double* dpart, double* mean_sq, cudaStream_t st) {
  k_ic_modes<T><<<1184, 256, 0, st>>>(g.tb, seed, stream, shape, k0, kmin, kmax, work[0], work[1]);
  TARA_CUDA_TRY(cudaGetLastError());
  const Cx<T>* spec[2] = {work[0], work[1]};
  T* real[2] = {ru, rv};
  Cx<T>* w2[2] = {work[2], work[3]};
  TARA_TRY(c2r_fields(g, 2, spec, real, w2, true, st));
  const size_t n = (size_t)g.Nx * g.Ny;
  k_ic_sumsq<T><<<kSumBlocks, kSumThreads, 0, st>>>(ru, rv, n, dpart);
  TARA_CUDA_TRY(cudaGetLastError());
  std::vector<double> part(kSumBlocks);
  TARA_CUDA_TRY(cudaMemcpyAsync(part.data(), dpart, kSumBlocks * sizeof(double), cudaMemcpyDeviceToHost, st));
  TARA_CUDA_TRY(cudaStreamSynchronize(st));
  double s = 0.0;
  for (double v : part) s += v;
  *mean_sq = s / (double)n;
  return TARA_OK;
}

}  // namespace

template <class T>
int ic_random_state(const Grid<T>& g, int model, const tara_params& p, const tara_ic& ic, T* const* r,
                    Cx<T>* const* work, cudaStream_t st) {
  if (model != TARA_MODEL_COH && model != TARA_MODEL_COM) {
    set_error("device initial conditions are built for the hydro and MHD models");
    return TARA_EUNSUPPORTED;
  }
  const bool ot = ic.kind == TARA_IC_ORSZAG_TANG;
  if ((ic.kind != TARA_IC_RANDOM_PHASE && !ot) || (ot && model != TARA_MODEL_COM)) {
    set_error("unknown initial condition for this model");
    return TARA_EINVAL;
  }
  if (!ot && !(ic.k0 > 0.0)) { set_error("k0 must be positive"); return TARA_EINVAL; }
  double* dpart = nullptr;
  TARA_CUDA_TRY(cudaMalloc(&dpart, kSumBlocks * sizeof(double)));
  const int shape = ot ? SHAPE_FLAT : SHAPE_PEAKED;
  const double kmin = ot ? ic.kmin : 0.0, kmax = ot ? ic.kmax : 1e300;
  // scale so that <|u|^2>/2 = e (random phase) or sqrt(<|u|^2>) = e (perturbation rms)
  auto scale = [&](double msq, double e) {
    if (!(msq > 0.0)) return 0.0;
    return ot ? e / sqrt(msq) : sqrt(e / (0.5 * msq));
  };
  IcAssembly a{};
  a.model = model;
  a.kind = ic.kind;
  a.Nx = g.Nx;
  a.Ny = g.Ny;
  a.dx = g.Lx / g.Nx;
  a.dy = g.Ly / g.Ny;
  a.seed = ic.seed;
  a.noise = ic.e2;
  a.cs2 = p.CS * p.CS;
  a.gam1 = p.spheat - 1.0;
  double msq = 0.0;
  int rc = solenoidal(g, ic.seed, 1, shape, ic.k0, kmin, kmax, r[1], r[2], work, dpart, &msq, st);
  a.su = scale(msq, ic.e1);
  if (rc == TARA_OK && model == TARA_MODEL_COM) {
    rc = solenoidal(g, ic.seed, 2, shape, ic.k0, kmin, kmax, r[4], r[5], work, dpart, &msq, st);
    a.sb = scale(msq, ic.e2);
  }
  if (rc == TARA_OK) {
    k_ic_assemble<T><<<1184, 256, 0, st>>>(a, r[0], r[1], r[2], r[3], r[4], r[5]);
    if (cudaGetLastError() != cudaSuccess) rc = TARA_ECUDA;
  }
  cudaStreamSynchronize(st);
  cudaFree(dpart);
  return rc;
}

template int ic_random_state<double>(const Grid<double>&, int, const tara_params&, const tara_ic&, double* const*,
                                     Cx<double>* const*, cudaStream_t);
template int ic_random_state<float>(const Grid<float>&, int, const tara_params&, const tara_ic&, float* const*,
                                    Cx<float>* const*, cudaStream_t);

}  // namespace tara
