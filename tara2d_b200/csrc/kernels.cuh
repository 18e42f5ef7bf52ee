// Generic column kernels (inverse y pass, forward y pass + dealias + time
// step) and the launch configurations shared by every model.
#pragma once
#include "spectral.cuh"
#include "tma.cuh"
#include "../../include/tara2d_gpu.h"

namespace tara {

// ------------------------------------------------------------ configurations
// Column pass: CB adjacent kx columns per CTA, P values per thread.
template <class T, int L> struct ColCfg { static constexpr int CB = 4, P = 16; };
template <int L> struct ColCfg<double, L> {
  static constexpr int P = (L == 384) ? 24 : 16;
  static constexpr int CB = (L <= 256) ? 8 : (L <= 1024 ? 4 : 2);
};
template <int L> struct ColCfg<float, L> {
  static constexpr int P = (L == 384) ? 24 : 16;
  static constexpr int CB = (L <= 1024) ? 8 : 4;
};
// Column pass of the MHD epilogue (two live value sets per thread: the FFT
// and the derivative being assembled), so fewer values per thread.  FP64
// columns of 1024 points run 4 kx columns per CTA (512 threads, 64-byte tile
// rows): 118.6 against 124.5 us per launch with 2 columns at 1024^2.
template <class T, int L> struct ColFwdComCfg { static constexpr int CB = 4, P = 16; };
template <int L> struct ColFwdComCfg<double, L> {
  static constexpr int P = (L == 384) ? 24 : (L >= 512 ? 8 : 16);
  static constexpr int CB = (L <= 256) ? 8 : (L == 384 || L == 1024 ? 4 : 2);
};
template <int L> struct ColFwdComCfg<float, L> {
  static constexpr int P = (L == 384) ? 24 : (L >= 512 && L < 4096 ? 8 : 16);
  static constexpr int CB = (L <= 256) ? 8 : (L >= 4096 ? 2 : 4);
};
// Row pass: P values per thread (M = Nx/2 points per row FFT).
template <int M> struct RowCfg { static constexpr int P = 16; };
template <> struct RowCfg<8> { static constexpr int P = 8; };
template <> struct RowCfg<192> { static constexpr int P = 24; };

#define TARA_DISPATCH_LEN(n, FN, ...)                    \
  switch (n) {                                           \
    case 16: FN<16>(__VA_ARGS__); break;                 \
    case 32: FN<32>(__VA_ARGS__); break;                 \
    case 64: FN<64>(__VA_ARGS__); break;                 \
    case 128: FN<128>(__VA_ARGS__); break;               \
    case 256: FN<256>(__VA_ARGS__); break;               \
    case 384: FN<384>(__VA_ARGS__); break;               \
    case 512: FN<512>(__VA_ARGS__); break;               \
    case 1024: FN<1024>(__VA_ARGS__); break;             \
    case 2048: FN<2048>(__VA_ARGS__); break;             \
    case 4096: FN<4096>(__VA_ARGS__); break;             \
    default: break;                                      \
  }

// Minimum resident CTAs per SM requested from the register allocator: at
// least 16 warps per SM for CTAs of up to 256 threads.
#define TARA_MINB(nt) ((nt) <= 128 ? 4 : ((nt) <= 256 ? 2 : 1))
// Launch bound of a row kernel whose rows need tpr threads each: small rows
// are packed several per CTA up to 128 threads.
#define TARA_ROW_LB(tpr) ((tpr) >= 128 ? ((tpr) <= 1024 ? (tpr) : 1024) : 128)

// ------------------------------------------------------------ multipliers
// MUL_ONE..MUL_KY2 depend on ky only.  The streamfunction modes depend on kx
// as well: psi = omega/(kx^2 + ky^2 + lambda), zero at k = 0, and
// wd = (kx^2 + ky^2) psi  (src/derive2csh.f95:28-56, src/derive2css.f95:20-56).
enum : int { MUL_ONE = 0, MUL_IKY = 1, MUL_KY2 = 2, MUL_PSI = 3, MUL_IKY_PSI = 4, MUL_WD = 5, MUL_IKY_WD = 6 };

template <class T>
__device__ __forceinline__ Cx<T> apply_ymul(int mul, T ky, Cx<T> x) {
  if (mul == MUL_IKY) return ikmul(ky, x);       // (0,1)*ky*x
  if (mul == MUL_KY2) return rmul(ky * ky, x);   // ky*ky*x
  return x;
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
// kx*kx + ky*ky rounded as written (no fused multiply-add)
template <class T> __device__ __forceinline__ T ksq(T kx, T ky) { return mul_rn(kx, kx) + mul_rn(ky, ky); }

// Streamfunction multipliers at (kx index c, ky index j); lam = 0 gives the
// unscreened model.
template <class T>
__device__ __forceinline__ Cx<T> apply_psi_mul(int mul, T lam, T kx, T ky, bool origin, Cx<T> w) {
  const T k2 = ksq(kx, ky);
  // one reciprocal of k^2 + lam per mode (the reference divides both
  // components; the results differ in the last bit)
  const T iden = (T)1 / (k2 + lam);
  const Cx<T> psi = origin ? cx<T>(0, 0) : cx<T>(w.x * iden, w.y * iden);
  switch (mul) {
    case MUL_PSI: return psi;
    case MUL_IKY_PSI: return ikmul(ky, psi);
    case MUL_WD: return rmul(k2, psi);
    default: return ikmul(ky, rmul(k2, psi));  // MUL_IKY_WD
  }
}

// ------------------------------------------------------------ inverse y pass
template <class T> struct ColInvJob {
  const Cx<T>* src;
  Cx<T>* dst;
  int mul;
  T lam;  // screening constant of the streamfunction modes
};

// Multiplier of job jb at (column c, row i).
template <class T>
__device__ __forceinline__ Cx<T> apply_job_mul(const ColInvJob<T>& jb, const Tables<T>& tb, int c, int i, Cx<T> x) {
  const T ky = __ldg(tb.ky + i);
  if (jb.mul < MUL_PSI) return apply_ymul(jb.mul, ky, x);
  return apply_psi_mul(jb.mul, jb.lam, __ldg(tb.kx + c), ky, c == 0 && i == 0, x);
}
template <class T> struct ColInvArgs {
  Tables<T> tb;
  ColInvJob<T> job[8];
};

// y-inverse of the CB kx columns c0.. of one job, by CB*L/P threads (tid)
// sharing the exchange tile sm.
template <class T, int L, int CB, int P>
__device__ __forceinline__ void col_inv_tile(const ColInvJob<T>& jb, const Tables<T>& tb, int c0, Cx<T>* sm,
                                             int tid) {
  using F = FFTB<L, CB, P>;
  const int Nh = tb.Nh, ld = tb.ld;
  Cx<T> v[P];
  fft_run<F, +1>(sm, tid, v, TwGlobal<T>{tb.tw_col}, [&](int t, int i) -> Cx<T> {
    const int c = c0 + t;
    if (c >= Nh) return cx<T>(0, 0);
    return apply_job_mul(jb, tb, c, i, ldg(jb.src + (size_t)i * ld + c));
  }, SyncBlock{});
  fft_emit<F>(tid, v, [&](int t, int i, Cx<T> x) {
    const int c = c0 + t;
    if (c < Nh) st(jb.dst + (size_t)i * ld + c, x);
  });
}

// blockIdx.x: tile of CB kx columns; blockIdx.y: job
template <class T, int L, int CB, int P>
__global__ void __launch_bounds__(CB * L / P, TARA_MINB(CB * L / P)) k_col_inv(const ColInvArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  col_inv_tile<T, L, CB, P>(a.job[blockIdx.y], a.tb, blockIdx.x * CB, reinterpret_cast<Cx<T>*>(smraw), threadIdx.x);
}

// TMA-staged, persistent variant: each CTA loops over (tile, job) items; the
// next item's column tile is loaded by the TMA unit into the other of two
// shared-memory buffers while the current one is transformed in place.
template <class T> struct ColInvTmaArgs {
  ColInvJob<T> job[8];
  CUtensorMap map[8];
  Tables<T> tb;
  int njobs, ntiles;
};

template <int L, int CB, int P> struct ColTmaLayout {
  using F = FFTB<L, CB, P>;
  static constexpr int BOX = L <= 256 ? L : (L % 256 == 0 ? 256 : 128);  // rows per TMA box (divides L)
  // complex elements per buffer: a multiple of 16, so that every buffer starts
  // on the 128-byte boundary a TMA destination needs, for 8- and 16-byte elements
  static constexpr int BUFE = (F::SMEM_ELEMS + 15) / 16 * 16;
  template <class T> static constexpr size_t bytes() { return 2 * (size_t)BUFE * sizeof(Cx<T>) + 64; }
};

template <class T, int L, int CB, int P>
__global__ void __launch_bounds__(CB * L / P, 1) k_col_inv_tma(const __grid_constant__ ColInvTmaArgs<T> a) {
  using F = FFTB<L, CB, P>;
  using LY = ColTmaLayout<L, CB, P>;
  constexpr unsigned TILE_BYTES = (unsigned)(CB * L * sizeof(Cx<T>));
  extern __shared__ __align__(128) unsigned char smtile[];  // TMA destinations: 128-byte aligned
  Cx<T>* buf0 = reinterpret_cast<Cx<T>*>(smtile);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smtile + 2 * (size_t)LY::BUFE * sizeof(Cx<T>));
  const int tid = threadIdx.x;
  const int nitems = a.ntiles * a.njobs;
  const int Nh = a.tb.Nh, ld = a.tb.ld;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init_fence();
  }
  __syncthreads();
  auto issue = [&](int item, int b) {
    const int job = item % a.njobs, tile = item / a.njobs;
    Cx<T>* dst = buf0 + b * LY::BUFE;
    mbar_expect_tx(&bars[b], TILE_BYTES);
#pragma unroll 1
    for (int y = 0; y < L; y += LY::BOX) tma_load_2d(dst + y * CB, &a.map[job], 2 * tile * CB, y, &bars[b]);
  };
  int item = blockIdx.x;
  if (tid == 0 && item < nitems) issue(item, 0);
  int it = 0;
  bool failed = false;
  for (; item < nitems; item += gridDim.x, it++) {
    const int b = it & 1;
    const unsigned parity = (it >> 1) & 1;
    const int next = item + gridDim.x;
    if (tid == 0 && next < nitems) {
      fence_proxy_async_smem();
      issue(next, b ^ 1);
    }
    const bool ok = mbar_wait_bounded(&bars[b], parity, a.tb.wait_ns);
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    const int job = item % a.njobs, tile = item / a.njobs;
    const ColInvJob<T> jb = a.job[job];
    Cx<T>* sm = buf0 + b * LY::BUFE;
    const int c0 = tile * CB;
    Cx<T> v[P];
    fft_run<F, +1>(sm, tid, v, TwGlobal<T>{a.tb.tw_col}, [&](int t, int i) -> Cx<T> {
      // columns past Nh hold the TMA fill value (zero); keep kx in range
      const int c = c0 + t < Nh ? c0 + t : Nh - 1;
      return apply_job_mul(jb, a.tb, c, i, sm[i * CB + t]);
    }, SyncBlock{});
    fft_emit<F>(tid, v, [&](int t, int i, Cx<T> x) {
      const int c = c0 + t;
      if (c < Nh) st(jb.dst + (size_t)i * ld + c, x);
    });
    __syncthreads();  // all reads of this buffer are done before it is refilled
  }
  if (failed) {
    // record the failure, then let the loads still in flight land (bounded)
    if (tid == 0) atomicExch(a.tb.status, TARA_ETIMEOUT);
    const int b = it & 1;
    mbar_wait_bounded(&bars[b], (it >> 1) & 1, a.tb.wait_ns);
    if (item + (int)gridDim.x < nitems) mbar_wait_bounded(&bars[b ^ 1], ((it + 1) >> 1) & 1, a.tb.wait_ns);
  }
}

// ------------------------------------------------------------ time steppers
enum : int { STEP_RHS = 0, STEP_AB2 = 1, STEP_EULER = 2, STEP_RK4 = 3 };

template <class T> struct StepArgs {
  int mode;
  int stage;   // RK4 stage 0..3
  T dt;
  T wa;        // RK4: weight*dt/6 of this stage
  T cs;        // RK4: c*dt of the next stage input
  Cx<T>* out[6];  // STEP_RHS: derivative output
  Cx<T>* u[6];    // base state (read only)
  Cx<T>* unew[6]; // new state (AB2, Euler, last RK4 stage); never aliases u or the RHS input
  Cx<T>* dold[6]; // AB2 history, replaced by the new derivative (same element, same thread)
  Cx<T>* acc[6];  // RK4 accumulator
  Cx<T>* us[6];   // RK4 next stage input; never aliases the current stage input
  // CFL control (nullptr: off): dt, wa and cs are multiplied by *scale, the
  // factor the CFL update of this step wrote on the device (1 leaves them
  // exactly as given; 0 stops the step)
  const double* scale;
};

// Device state of the CFL control of a session (see k_cfl_update).
struct CflDev {
  unsigned long long lam;  // max over the grid of the signal-speed rate, as the bits of a non-negative double
  double scale;            // dt of this step / the configured dt
  double t;                // model time advanced under CFL control
  double dt;               // dt of the last step
};

// Folds one thread's largest signal-speed rate m into *lam: a maximum over
// the threads of the warp that call it together (their bit patterns: a
// non-negative double orders like its bits, and a NaN or inf exceeds every
// finite value), then one atomicMax per warp.  Partial warps are fine.
__device__ __forceinline__ double nan_max(double a, double b) { return (b > a || b != b) ? b : a; }
__device__ __forceinline__ void cfl_fold(double m, unsigned long long* lam) {
  const unsigned mask = __activemask();
  const unsigned long long b = (unsigned long long)__double_as_longlong(m);
  const unsigned hi = (unsigned)(b >> 32), lo = (unsigned)(b & 0xffffffffu);
  const unsigned mhi = __reduce_max_sync(mask, hi);
  const unsigned mlo = __reduce_max_sync(mask, hi == mhi ? lo : 0u);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(lam, ((unsigned long long)mhi << 32) | mlo);
}
// Signal-speed rate of one grid point, (|ux| + c)/dx + (|uy| + c)/dy.
__device__ __forceinline__ double cfl_rate(double ux, double uy, double c, double idx, double idy) {
  return (fabs(ux) + c) * idx + (fabs(uy) + c) * idy;
}
// CFL arguments of a row pass (lam == nullptr: not computed).
struct CflRow {
  unsigned long long* lam;
  double idx, idy;  // 1/dx, 1/dy
  double cs2;       // squared sound speed
};

// d = derivative of field f at element idx.  Operation order follows
// src/ab2coh.f95:22 / src/ab2com.f95:69 and src/euler2coh.f95:104.
template <class T>
__device__ __forceinline__ void step_apply(const StepArgs<T>& s, int f, size_t idx, Cx<T> d) {
  T dt = s.dt, wa = s.wa, cs = s.cs;
  if (s.scale) {
    const T sc = (T)*s.scale;
    dt *= sc;
    wa *= sc;
    cs *= sc;
  }
  switch (s.mode) {
    case STEP_RHS:
      st(s.out[f] + idx, d);
      break;
    case STEP_AB2: {
      Cx<T> old = ld(s.dold[f] + idx);
      Cx<T> u = ld(s.u[f] + idx);
      Cx<T> inc = rmul((T)1.5, d) - rmul((T)0.5, old);
      st(s.unew[f] + idx, u + rmul(dt, inc));
      st(s.dold[f] + idx, d);
      break;
    }
    case STEP_EULER: {
      Cx<T> u = ld(s.u[f] + idx);
      st(s.unew[f] + idx, u + rmul(dt, d));
      st(s.dold[f] + idx, d);
      break;
    }
    default: {  // RK4
      if (s.stage == 0) {
        Cx<T> u = ld(s.u[f] + idx);
        st(s.acc[f] + idx, u + rmul(wa, d));
        st(s.us[f] + idx, u + rmul(cs, d));
      } else if (s.stage < 3) {
        Cx<T> u = ld(s.u[f] + idx);
        Cx<T> a = ld(s.acc[f] + idx);
        st(s.acc[f] + idx, a + rmul(wa, d));
        st(s.us[f] + idx, u + rmul(cs, d));
      } else {
        Cx<T> a = ld(s.acc[f] + idx);
        st(s.unew[f] + idx, a + rmul(wa, d));
      }
      break;
    }
  }
}

// The update of step_apply for the N elements a thread holds: every load is
// issued before the first store.  Element by element, each element's loads
// would wait for the previous element's stores (the compiler cannot tell that
// they never alias), so a thread would wait on memory N times in a row.
// pos(e, idx) gives element e's index and whether it exists.  Same
// arithmetic as step_apply, element for element.
// nxt (optional, may be d): receives each element's next RHS input (the new
// state, or the next RK4 stage input).
template <class T, int N, class POS>
__device__ __forceinline__ void step_apply_n(const StepArgs<T>& s, int f, POS&& pos, const Cx<T>* d,
                                             Cx<T>* nxt = nullptr) {
  if (s.mode == STEP_RHS) {
#pragma unroll
    for (int e = 0; e < N; e++) {
      size_t idx;
      if (pos(e, idx)) st(s.out[f] + idx, d[e]);
    }
    return;
  }
  T dt = s.dt, wa = s.wa, cs = s.cs;
  if (s.scale) {
    const T sc = (T)*s.scale;
    dt *= sc;
    wa *= sc;
    cs *= sc;
  }
  const bool rk4 = s.mode == STEP_RK4;
  const bool need0 = s.mode == STEP_AB2 || (rk4 && s.stage > 0);  // AB2 history or RK4 accumulator
  const bool need1 = !rk4 || s.stage < 3;                          // state
  const Cx<T>* p0 = s.mode == STEP_AB2 ? s.dold[f] : s.acc[f];
  const Cx<T>* p1 = s.u[f];
  Cx<T> x0[N], x1[N];
#pragma unroll
  for (int e = 0; e < N; e++) {
    size_t idx;
    x0[e] = x1[e] = cx<T>(0, 0);
    if (pos(e, idx)) {
      if (need0) x0[e] = ld(p0 + idx);
      if (need1) x1[e] = ld(p1 + idx);
    }
  }
#pragma unroll
  for (int e = 0; e < N; e++) {
    size_t idx;
    const bool ok = pos(e, idx);
    const Cx<T> de = d[e];
    Cx<T> nv = cx<T>(0, 0);
    if (s.mode == STEP_AB2) {
      const Cx<T> inc = rmul((T)1.5, de) - rmul((T)0.5, x0[e]);
      nv = x1[e] + rmul(dt, inc);
      if (ok) {
        st(s.unew[f] + idx, nv);
        st(s.dold[f] + idx, de);
      }
    } else if (s.mode == STEP_EULER) {
      nv = x1[e] + rmul(dt, de);
      if (ok) {
        st(s.unew[f] + idx, nv);
        st(s.dold[f] + idx, de);
      }
    } else if (s.stage == 0) {
      nv = x1[e] + rmul(cs, de);
      if (ok) {
        st(s.acc[f] + idx, x1[e] + rmul(wa, de));
        st(s.us[f] + idx, nv);
      }
    } else if (s.stage < 3) {
      nv = x1[e] + rmul(cs, de);
      if (ok) {
        st(s.acc[f] + idx, x0[e] + rmul(wa, de));
        st(s.us[f] + idx, nv);
      }
    } else {
      nv = x0[e] + rmul(wa, de);
      if (ok) st(s.unew[f] + idx, nv);
    }
    if (nxt) nxt[e] = ok ? nv : cx<T>(0, 0);
  }
}

// ------------------------------------------------------------ forward y pass
// One output field per CTA row of the grid (blockIdx.y = f): forward y DFT of
// X[f], circular 2/3 dealiasing, sign, then the stepper update.
template <class T> struct ColFwdSimpleArgs {
  Tables<T> tb;
  const Cx<T>* X[6];
  T sign[6];  // derivative = sign * dealiased transform
  int nomask;  // 1: plain forward transform (no dealiasing)
  StepArgs<T> step;
};

// Output field f, kx columns c0..c0+CB-1, by CB*L/P threads (tid).
template <class T, int L, int CB, int P>
__device__ __forceinline__ void col_fwd_simple_tile(const ColFwdSimpleArgs<T>& a, int f, int c0, Cx<T>* sm,
                                                    int tid) {
  using F = FFTB<L, CB, P>;
  const int Nh = a.tb.Nh, ld = a.tb.ld;
  const Cx<T>* X = a.X[f];
  Cx<T> v[P];
  fft_run<F, -1>(sm, tid, v, TwGlobal<T>{a.tb.tw_col}, [&](int t, int i) -> Cx<T> {
    const int c = c0 + t;
    if (c >= Nh) return cx<T>(0, 0);
    return ldg(X + (size_t)i * ld + c);
  }, SyncBlock{});
  const T sg = a.sign[f];
  constexpr int RL = F::Pl::R[F::S - 1];
  // derivative values in the order fft_emit visits them: element e = q*RL + r
#pragma unroll
  for (int e = 0; e < P; e++) {
    int t, j;
    F::template out_pos<F::S - 1>(tid, e / RL, e % RL, t, j);
    const int c = min(c0 + t, Nh - 1);
    const bool masked = !a.nomask && c >= __ldg(a.tb.cut + j);
    const Cx<T> val = masked ? cx<T>(0, 0) : v[e];
    v[e] = cx<T>(sg * val.x, sg * val.y);
  }
  step_apply_n<T, P>(a.step, f, [&](int e, size_t& idx) {
    int t, j;
    F::template out_pos<F::S - 1>(tid, e / RL, e % RL, t, j);
    const int c = c0 + t;
    idx = (size_t)j * ld + c;
    return c < Nh;
  }, v);
}

template <class T, int L, int CB, int P>
__global__ void __launch_bounds__(CB * L / P, TARA_MINB(CB * L / P)) k_col_fwd_simple(const ColFwdSimpleArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  col_fwd_simple_tile<T, L, CB, P>(a, blockIdx.y, blockIdx.x * CB, reinterpret_cast<Cx<T>*>(smraw), threadIdx.x);
}

template <class T, int L>
inline size_t col_smem_bytes() {
  return (size_t)FFTB<L, ColCfg<T, L>::CB, ColCfg<T, L>::P>::SMEM_ELEMS * sizeof(Cx<T>);
}

template <class T, int L>
inline int launch_col_inv(const ColInvArgs<T>& a, int njobs, cudaStream_t st) {
  constexpr int CB = ColCfg<T, L>::CB, P = ColCfg<T, L>::P;
  auto kern = k_col_inv<T, L, CB, P>;
  const size_t smem = col_smem_bytes<T, L>();
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid((a.tb.Nh + CB - 1) / CB, njobs);
  kern<<<grid, CB * L / P, smem, st>>>(a);
  return 0;
}

template <class T, int L>
inline int launch_col_fwd_simple(const ColFwdSimpleArgs<T>& a, int nf, cudaStream_t st) {
  constexpr int CB = ColCfg<T, L>::CB, P = ColCfg<T, L>::P;
  auto kern = k_col_fwd_simple<T, L, CB, P>;
  const size_t smem = col_smem_bytes<T, L>();
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid((a.tb.Nh + CB - 1) / CB, nf);
  kern<<<grid, CB * L / P, smem, st>>>(a);
  return 0;
}

template <int L, class T>
inline void col_inv_dispatch(const ColInvArgs<T>& a, int njobs, cudaStream_t st) {
  constexpr int CB = ColCfg<T, L>::CB, P = ColCfg<T, L>::P;
  using LY = ColTmaLayout<L, CB, P>;
  ColInvTmaArgs<T> t{};
  t.tb = a.tb;
  t.njobs = njobs;
  t.ntiles = (a.tb.Nh + CB - 1) / CB;
  // two column tiles must fit in shared memory (not so for the longest columns)
  constexpr bool fits = LY::template bytes<T>() <= 220 * 1024;
  bool maps_ok = fits && !a.tb.no_tma && (a.tb.ld * sizeof(Cx<T>)) % 16 == 0 && (2 * CB * sizeof(T)) % 16 == 0;
  for (int q = 0; q < njobs && maps_ok; q++) {
    t.job[q] = a.job[q];
    maps_ok = make_col_tile_map<T>(&t.map[q], a.job[q].src, a.tb.ld, a.tb.Ny, CB, LY::BOX) == TARA_OK;
  }
  if (!maps_ok) {  // layouts the TMA unit cannot describe use the register-staged kernel
    launch_col_inv<T, L>(a, njobs, st);
    return;
  }
  auto kern = k_col_inv_tma<T, L, CB, P>;
  const size_t smem = LY::template bytes<T>();
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CB * L / P, smem);
  const int nitems = t.ntiles * njobs;
  int grid = a.tb.sm_count * (per_sm > 0 ? per_sm : 1);
  if (grid > nitems) grid = nitems;
  kern<<<grid, CB * L / P, smem, st>>>(t);
}
template <int L, class T>
inline void col_fwd_simple_dispatch(const ColFwdSimpleArgs<T>& a, int nf, cudaStream_t st) {
  launch_col_fwd_simple<T, L>(a, nf, st);
}

template <class T>
inline void run_col_inv(const ColInvArgs<T>& a, int njobs, cudaStream_t st) {
  TARA_DISPATCH_LEN(a.tb.Ny, col_inv_dispatch, a, njobs, st)
}
template <class T>
inline void run_col_fwd_simple(const ColFwdSimpleArgs<T>& a, int nf, cudaStream_t st) {
  TARA_DISPATCH_LEN(a.tb.Ny, col_fwd_simple_dispatch, a, nf, st)
}

// ------------------------------------------------------------ y round trip
// dst = y-inverse( mul(ky) * y-forward(src) ): the y-derivative of an
// x-transformed field, returned as a half-real field.
template <class T> struct ColRtArgs {
  Tables<T> tb;
  const Cx<T>* src;
  Cx<T>* dst;
  int mul;
};
template <class T, int L, int CB, int P>
__global__ void __launch_bounds__(CB * L / P, TARA_MINB(CB * L / P)) k_col_rt(const ColRtArgs<T> a) {
  using F = FFTB<L, CB, P>;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  const int c0 = blockIdx.x * CB;
#include "col_rt_body.inc"
}
// The same pass as a device function of the calling CTA (CB*L/P threads).
template <class T, int L, int CB, int P>
__device__ __forceinline__ void col_rt_tile(const ColRtArgs<T>& a, int c0) {
  using F = FFTB<L, CB, P>;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
#include "col_rt_body.inc"
}
template <int L, class T>
inline void col_rt_dispatch(const ColRtArgs<T>& a, cudaStream_t st) {
  constexpr int CB = ColCfg<T, L>::CB, P = ColCfg<T, L>::P;
  auto kern = k_col_rt<T, L, CB, P>;
  const size_t smem = col_smem_bytes<T, L>();
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<(a.tb.Nh + CB - 1) / CB, CB * L / P, smem, st>>>(a);
}
template <class T>
inline void run_col_rt(const ColRtArgs<T>& a, cudaStream_t st) {
  TARA_DISPATCH_LEN(a.tb.Ny, col_rt_dispatch, a, st)
}

// rows per CTA for a row kernel with ntr threads per row
inline int rows_per_cta(int ntr, int Ny, size_t smem_per_row) {
  int rb = 1;
  while (rb * 2 * ntr <= 64 && Ny % (rb * 2) == 0 && (rb * 2) * smem_per_row <= 96 * 1024) rb *= 2;
  return rb;
}

}  // namespace tara
