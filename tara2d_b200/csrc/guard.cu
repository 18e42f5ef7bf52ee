// Time-step control and state checks of the sessions: the CFL update of a
// step, the check for non-finite values, and the self-test of the bounded
// mbarrier wait used by the TMA kernels.
#include <cmath>
#include "models.h"

namespace tara {

// One thread.  c.dev->lam holds the largest signal-speed rate of the state
// at the start of the step (folded by the row pass); from it the dt of this
// step as a factor of the configured dt, read by every stepper update of the
// step (StepArgs::scale).
__global__ void k_cfl_update(CflDev* d, int mode, double number, double dt_max, int* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double rate = __longlong_as_double((long long)d->lam);
  d->lam = 0ull;
  double scale = 1.0;
  if (!(rate <= 1.7976931348623157e308)) {  // NaN or inf somewhere in the state
    atomicCAS(status, TARA_OK, TARA_ENAN);
    scale = 0.0;
  } else {
    const double dt_cfl = rate > 0.0 ? number / rate : INFINITY;
    if (mode == CFL_CHECK) {
      if (dt_max > dt_cfl) {
        atomicCAS(status, TARA_OK, TARA_ECFL);
        scale = 0.0;
      }
    } else if (dt_cfl < dt_max) {
      if (dt_cfl < 1e-6 * dt_max) {
        atomicCAS(status, TARA_OK, TARA_ECFL);
        scale = 0.0;
      } else {
        scale = dt_cfl / dt_max;
      }
    }
  }
  d->scale = scale;
  d->dt = scale == 1.0 ? dt_max : scale * dt_max;
  d->t += d->dt;
}

int launch_cfl_update(const CflCfg& c, int* status, cudaStream_t st) {
  k_cfl_update<<<1, 32, 0, st>>>(c.dev, c.mode, c.number, c.dt, status);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

template <class T> struct FiniteArgs {
  const Cx<T>* f[6];
  int nf, Nh, ld, Ny;
  int* status;
};
// One CTA per row: every value of the nf fields in it; TARA_ENAN into the
// status word (first error kept) when one is not finite.
template <class T>
__global__ void __launch_bounds__(256) k_finite(const FiniteArgs<T> a) {
  bool bad = false;
  for (int j = blockIdx.x; j < a.Ny; j += gridDim.x)
    for (int q = 0; q < a.nf; q++) {
      const Cx<T>* row = a.f[q] + (size_t)j * a.ld;
      for (int i = threadIdx.x; i < a.Nh; i += blockDim.x) {
        const Cx<T> v = ldg(row + i);
        bad |= !isfinite(v.x) || !isfinite(v.y);
      }
    }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicCAS(a.status, TARA_OK, TARA_ENAN);
}

template <class T>
int launch_finite_check(const Grid<T>& g, Cx<T>* const* f, int nf, cudaStream_t st) {
  FiniteArgs<T> a{};
  for (int q = 0; q < nf && q < 6; q++) a.f[q] = f[q];
  a.nf = nf < 6 ? nf : 6;
  a.Nh = g.Nh;
  a.ld = g.ld;
  a.Ny = g.Ny;
  a.status = g.tb.status;
  const int grid = g.Ny < 4 * g.tb.sm_count ? g.Ny : 4 * g.tb.sm_count;
  k_finite<T><<<grid, 256, 0, st>>>(a);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}
template int launch_finite_check<double>(const Grid<double>&, Cx<double>* const*, int, cudaStream_t);
template int launch_finite_check<float>(const Grid<float>&, Cx<float>* const*, int, cudaStream_t);

// One CTA: thread 0 arms an mbarrier with one arrival and 16 expected bytes
// that no copy delivers (none is issued), then every thread waits on it with
// the bounded wait of the TMA kernels.  The wait must run out.
__global__ void k_wait_selftest(unsigned long long limit_ns, int* status, unsigned long long* waited) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);
  __syncthreads();
  const unsigned long long t0 = global_ns();
  const bool ok = mbar_wait_bounded(&bar, 0, limit_ns);
  const unsigned long long t1 = global_ns();
  if (threadIdx.x == 0) {
    *status = ok ? TARA_OK : TARA_ETIMEOUT;
    *waited = t1 - t0;
  }
}

}  // namespace tara

extern "C" int tara_selftest_bounded_wait(long long limit_ns, long long* waited_ns) {
  using namespace tara;
  if (limit_ns < 1000 || limit_ns > 10000000000ll) {
    set_error("tara_selftest_bounded_wait: limit must be 1 us .. 10 s");
    return TARA_EINVAL;
  }
  void* mem = nullptr;
  TARA_CUDA_TRY(cudaMalloc(&mem, 16));
  int* st = static_cast<int*>(mem);
  unsigned long long* w = reinterpret_cast<unsigned long long*>(static_cast<char*>(mem) + 8);
  k_wait_selftest<<<1, 64>>>((unsigned long long)limit_ns, st, w);
  cudaError_t e = cudaGetLastError();
  int status = TARA_ECUDA;
  unsigned long long waited = 0;
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&status, st, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&waited, w, sizeof(waited), cudaMemcpyDeviceToHost);
  cudaFree(mem);
  if (e != cudaSuccess) {
    set_error(std::string("tara_selftest_bounded_wait: ") + cudaGetErrorString(e));
    return TARA_ECUDA;
  }
  if (waited_ns) *waited_ns = (long long)waited;
  if (status == TARA_ETIMEOUT) set_error("bounded wait ran out (self-test)");
  return status;
}
