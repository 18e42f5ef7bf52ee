// Device building blocks of the pseudo-spectral RHS: the column (y) pass and
// the row (x) real-FFT passes, written on top of the Stockham engine in
// fft_core.cuh.
//
// Layouts on the device (one field):
//   spectral  [Ny][ld]  Cx<T>, element (kx index i, ky index j) at j*ld + i,
//             i < Nh = Nx/2+1, ld = Nh rounded up (128-byte rows).  This is the
//             reference's Fortran (Nh,Ny) array with a row pitch.
//   half-real [Ny][ld]  Cx<T>: the same array after the inverse y transform
//             (every kx column transformed, nothing dropped yet).
//
// 2D c2r (reference semantics, FFTW 3.3.9 rank-geq2 rdft2):
//   1. complex inverse DFT along y of every kx column (column pass),
//   2. c2r along x of every row; the imaginary parts of the kx = 0 and
//      kx = Nx/2 bins are ignored (row pass).
// 2D r2c: r2c along x of every row, then forward DFT along y.
#pragma once
#include <cuda_runtime.h>
#include "fft_core.cuh"

namespace tara {

// Per-grid read-only tables (device pointers).
template <class T>
struct Tables {
  const Cx<T>* tw_col;   // e^{-2 pi i m/Ny},     m < Ny
  const Cx<T>* tw_row;   // e^{-2 pi i m/(Nx/2)}, m < Nx/2
  const Cx<T>* tw_real;  // e^{-2 pi i k/Nx},     k <= Nx/2
  const T* kx;           // kx(i) = 2 pi i/Lx,                    i < Nh
  const T* ky;           // ky(j) = 2 pi j/Ly or 2 pi (j-Ny)/Ly,  j < Ny
  const int* cut;        // row j: modes with kx index >= cut[j] are dealiased
  int Nx, Ny, Nh, ld;
  T inv_nn;              // 1/(Nx*Ny)
  T nn;                  // Nx*Ny
  int nn_pow2;           // Nx*Ny is a power of two (so x*inv_nn == x/nn exactly)
  int* status;           // device status word (TARA_ETIMEOUT after a bounded wait ran out)
  int sm_count;          // multiprocessors of the device (persistent grids)
  int no_tma;            // 1: column passes use the register-staged kernels (no TMA, no bounded waits)
  unsigned long long wait_ns;  // limit of every bounded wait of the TMA kernels, in ns of %globaltimer
};

template <class T> __device__ __forceinline__ Cx<T> ldg(const Cx<T>* p);
template <> __device__ __forceinline__ Cx<double> ldg(const Cx<double>* p) {
  double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return cx<double>(v.x, v.y);
}
template <> __device__ __forceinline__ Cx<float> ldg(const Cx<float>* p) {
  float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return cx<float>(v.x, v.y);
}
// plain (coherent) load, for buffers written earlier in the same kernel
template <class T> __device__ __forceinline__ Cx<T> ld(const Cx<T>* p) { return *p; }
template <class T> __device__ __forceinline__ void st(Cx<T>* p, Cx<T> v) {
  if constexpr (sizeof(T) == 8) {
    *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y);
  } else {
    *reinterpret_cast<float2*>(p) = make_float2(v.x, v.y);
  }
}

template <class T> struct TwGlobal {
  const Cx<T>* p;
  __device__ __forceinline__ Cx<T> operator()(int m) const { return ldg(p + m); }
};

template <class T> __device__ __forceinline__ T normalise(T x, const Tables<T>& tb) {
  return tb.nn_pow2 ? x * tb.inv_nn : x / tb.nn;
}

// BatchFFT with its shared-memory exchange layout.  Element (t, i) lives at
// sidx(t, i) = i*B + t + i/R0: one pad slot every R0 rows breaks the bank
// conflicts of the first stage's stores (stride R0 between neighbouring
// butterflies).
template <int L, int B, int P> struct FFTB : BatchFFT<L, B, P> {
  static constexpr int B_ = B;
  static constexpr int L_ = L;
  static constexpr int PADR = BatchFFT<L, B, P>::Pl::R[0];
  static constexpr int SMEM_ELEMS = L * B + L / PADR + 1;
  __host__ __device__ static constexpr int sidx(int t, int i) { return i * B + t + i / PADR; }
};
template <int L, int P> using RowFFT = FFTB<L, 1, P>;

// ------------------------------------------------------------------ stages
template <class F, int s, class T>
__device__ __forceinline__ void fft_store(Cx<T>* sm, int tid, const Cx<T>* v) {
  constexpr int R = F::Pl::R[s];
#pragma unroll
  for (int q = 0; q < F::P / R; q++)
#pragma unroll
    for (int r = 0; r < R; r++) {
      int t, i;
      F::template out_pos<s>(tid, q, r, t, i);
      sm[F::sidx(t, i)] = v[q * R + r];
    }
}
template <class F, int s, class T>
__device__ __forceinline__ void fft_load(const Cx<T>* sm, int tid, Cx<T>* v) {
  constexpr int R = F::Pl::R[s];
#pragma unroll
  for (int q = 0; q < F::P / R; q++)
#pragma unroll
    for (int r = 0; r < R; r++) {
      int t, i;
      F::template in_pos<s>(tid, q, r, t, i);
      v[q * R + r] = sm[F::sidx(t, i)];
    }
}
// The exchange of BatchFFT::halves_exchange in registers: each thread keeps
// slot 2q + hb and trades slot 2q + 1 - hb with lane tid ^ 16 (tid is the
// lane: the transform's 32 threads are one whole warp).
template <class F, class T> __device__ __forceinline__ void warp_halves_swap(int tid, Cx<T>* v) {
  const bool hi = tid & 16;
#pragma unroll
  for (int q = 0; q < F::P / 2; q++) {
    Cx<T> o = hi ? v[2 * q] : v[2 * q + 1];
    o.x = __shfl_xor_sync(0xffffffffu, o.x, 16);
    o.y = __shfl_xor_sync(0xffffffffu, o.y, 16);
    if (hi) v[2 * q] = o;
    else v[2 * q + 1] = o;
  }
}
// Stages s..S-1 (s >= 1); the values of stage s-1 are in v.
template <class F, int s, int DIR, class T, class TW, class SYNC>
__device__ __forceinline__ void fft_rest(Cx<T>* sm, int tid, Cx<T>* v, const TW& tw, SYNC sync) {
  if constexpr (s < F::S) {
    if constexpr (F::template halves_exchange<s>()) {
      warp_halves_swap<F>(tid, v);
    } else {
      sync();
      fft_store<F, s - 1>(sm, tid, v);
      sync();
      fft_load<F, s>(sm, tid, v);
    }
    F::template compute<s, DIR>(tid, v, tw);
    fft_rest<F, s + 1, DIR>(sm, tid, v, tw, sync);
  }
}
// Stage-0 inputs from pro(t, i), stage-0 butterflies.
template <class F, int DIR, class T, class TW, class PRO>
__device__ __forceinline__ void fft_begin(int tid, Cx<T>* v, const TW& tw, PRO&& pro) {
  constexpr int R0 = F::Pl::R[0];
#pragma unroll
  for (int q = 0; q < F::P / R0; q++)
#pragma unroll
    for (int r = 0; r < R0; r++) {
      int t, i;
      F::template in_pos<0>(tid, q, r, t, i);
      v[q * R0 + r] = pro(t, i);
    }
  F::template compute<0, DIR>(tid, v, tw);
}
// The whole transform; on return v[] holds the last stage's outputs
// (positions F::out_pos<S-1>).  `sync` must synchronise every thread that
// shares `sm`.
template <class F, int DIR, class T, class TW, class PRO, class SYNC>
__device__ __forceinline__ void fft_run(Cx<T>* sm, int tid, Cx<T>* v, const TW& tw, PRO&& pro, SYNC sync) {
  fft_begin<F, DIR>(tid, v, tw, pro);
  fft_rest<F, 1, DIR>(sm, tid, v, tw, sync);
}
template <class F, class T, class EPI>
__device__ __forceinline__ void fft_emit(int tid, const Cx<T>* v, EPI&& epi) {
  constexpr int R = F::Pl::R[F::S - 1];
#pragma unroll
  for (int q = 0; q < F::P / R; q++)
#pragma unroll
    for (int r = 0; r < R; r++) {
      int t, i;
      F::template out_pos<F::S - 1>(tid, q, r, t, i);
      epi(t, i, v[q * R + r]);
    }
}

struct SyncBlock {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
// Barrier of one group of NTR consecutive threads: __syncwarp over the
// group's lanes for NTR <= 32 (groups sharing a warp synchronise
// independently), else named barrier `id` (1..15) of NTR threads.
template <int NTR> struct SyncGroup {
  int id;
  unsigned mask;
  __device__ __forceinline__ void operator()() const {
    if constexpr (NTR <= 32) {
      __syncwarp(mask);
    } else {
      asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(NTR) : "memory");
    }
  }
};

// Thread geometry of a row kernel: RB rows per CTA, G groups of NTR threads
// per row; each group runs one row FFT at a time.
template <int NTR, int G> struct RowThread {
  int row, g, lane, gid;
  __device__ __forceinline__ RowThread() {
    const int t = threadIdx.x;
    lane = t % NTR;
    gid = t / NTR;
    g = gid % G;
    row = gid / G;
  }
  __device__ __forceinline__ SyncGroup<NTR> sync() const {
    SyncGroup<NTR> s;
    s.id = 1 + gid;
    if constexpr (NTR < 32) {
      s.mask = ((1u << NTR) - 1u) << ((threadIdx.x & 31) / NTR * NTR);
    } else {
      s.mask = 0xffffffffu;
    }
    return s;
  }
};

// ----------------------------------------------------------- row helpers
// Inverse real transform of one row: X[0..M] -> x[0..2M-1] (unnormalised).
// hv(k) returns X[k] for 0 < k < M; for k = 0 and k = M only its real part
// is used (the kx = 0 / Nyquist bins of a c2r).  On return the thread holds
// z[n] = x[2n] + i x[2n+1] for its output positions n (RowF::out_pos).
// xs: exchange buffer of RowF::SMEM_ELEMS elements private to the group.
template <class RowF, class T, class HV, class SYNC>
__device__ __forceinline__ void row_c2r(Cx<T>* xs, int lane, Cx<T>* v, const Tables<T>& tb, HV&& hv, SYNC sync) {
  constexpr int M = RowF::L_;
  TwGlobal<T> tw{tb.tw_row};
  fft_run<RowF, +1>(xs, lane, v, tw, [&](int, int i) -> Cx<T> {
    Cx<T> A, B;
    if (i == 0) {
      A = cx<T>(hv(0).x, (T)0);
      B = cx<T>(hv(M).x, (T)0);
    } else {
      A = hv(i);
      B = conj(hv(M - i));
    }
    Cx<T> fe = A + B;
    Cx<T> w = ldg(tb.tw_real + i);  // e^{-2 pi i i/N}
    Cx<T> fo = cmul(A - B, conj(w));
    return cx<T>(fe.x - fo.y, fe.y + fo.x);
  }, sync);
}

// Forward real transform of one row, x[0..2M-1] -> X[0..M], in two parts so
// that the inputs can be gathered before the exchange buffer is claimed:
//   row_r2c_begin: gv(n) returns z[n] = x[2n] + i x[2n+1] at the stage-0
//                  positions; stage-0 butterflies;
//   row_r2c_finish: remaining stages in `zs`, then the real-to-complex
//                  post-processing; out(k, X) for k = 0..M (X[0], X[M] real).
template <class RowF, class T, class GV>
__device__ __forceinline__ void row_r2c_begin(int lane, Cx<T>* v, const Tables<T>& tb, GV&& gv) {
  fft_begin<RowF, -1>(lane, v, TwGlobal<T>{tb.tw_row}, [&](int, int i) { return gv(i); });
}
template <class RowF, class T, class OUT, class SYNC>
__device__ __forceinline__ void row_r2c_finish(Cx<T>* zs, int lane, int ntr, Cx<T>* v, const Tables<T>& tb,
                                               OUT&& out, SYNC sync) {
  constexpr int M = RowF::L_;
  fft_rest<RowF, 1, -1>(zs, lane, v, TwGlobal<T>{tb.tw_row}, sync);
  sync();
  fft_emit<RowF>(lane, v, [&](int, int i, Cx<T> z) { zs[RowF::sidx(0, i)] = z; });
  sync();
  for (int k = lane; k <= M; k += ntr) {
    Cx<T> zk = zs[RowF::sidx(0, k == M ? 0 : k)];
    Cx<T> zm = conj(zs[RowF::sidx(0, k == 0 ? 0 : M - k)]);
    Cx<T> e = rmul((T)0.5, zk + zm);
    Cx<T> d = zk - zm;
    Cx<T> o = cx<T>((T)0.5 * d.y, (T)-0.5 * d.x);  // (zk - zm)/(2i)
    Cx<T> w = ldg(tb.tw_real + k);
    Cx<T> X = e + cmul(w, o);
    if (k == 0 || k == M) X.y = (T)0;
    out(k, X);
  }
}

}  // namespace tara
