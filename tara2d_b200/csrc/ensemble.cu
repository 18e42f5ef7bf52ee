// Batched ensembles: many independent hydro (*2coh) and MHD (*2com) runs of
// different grid sizes and viscosities advanced together.
//
// Layout: one arena holds every member's fields back to back, each member a
// block in its own [N][ld] layout: hydro 20 fields [u_A(3) u_B(3) dold(3) |
// H(8) X(3)], MHD 38 fields [u_A(6) u_B(6) dold(6) | H(7) X(13)].  Device
// tables of member descriptors (the argument blocks of every RHS phase, with
// the state buffers of both parities) drive persistent kernels per step.
// Hydro members, three launches:
//
//   k_ens_col_inv  items (member, column tile, job): y-inverse, 8 jobs/member
//   k_ens_row      items (member, block of rows): the hydro row pass
//   k_ens_col_fwd  items (member, column tile, field): y-forward, mask, AB2
//
// MHD members, one persistent cooperative launch per step (k_ens_com_step)
// that runs these phases one after another, separated by grid-wide barriers
// with bounded waits (where the device has no cooperative launches, one
// launch per phase; the column inverse only where the half-real fields do
// not hold the y-inverse of the state yet: the column forward pass writes it
// for the next step, as in a single-grid session):
//
//   k_ens_com_inv   items (member, column tile, job): y-inverse of 6 fields
//   k_ens_com_row1  items (member, block of rows): c2r, fluxes, 8 r2c
//   k_ens_com_rt    items (member, column tile): d(uy)/dy round trip
//   k_ens_com_row2  items (member, block of rows): curl-B and (div u)^2 terms
//   k_ens_com_fwd   items (member, column tile, field): y-forward, assembly,
//                   AB2/Euler update, y-inverse of the new state
//
// Each kernel runs a grid of (CTAs per SM) x (SMs) CTAs that walk a
// size-sorted item list (largest grids first), so members of every size share
// every launch; the phase boundaries are the only synchronisation.  A step is
// the same launches for any mix of members (three for the hydro members, one
// for the MHD ones), so step pairs are captured once into a CUDA graph and
// replayed.  Per-member arithmetic is the same
// device code as a single-grid session (col_inv_tile, row_coh_rows,
// col_fwd_simple_tile), so with the session's values-per-thread choice a
// member's state is bit-identical to a session run of that member.
//
// Tuning (the autotuner picks by timing, hydro phases): values per thread of
// the column passes and of the row pass (8 or 16; 384-point transforms always
// use 24) and CTAs per SM of each persistent grid.  The MHD phases use the
// single-grid sessions' values per thread (ColCfg, ColFwdComCfg, RowCfg) in
// CTAs of 128 threads, so an MHD member is bit-identical to a session run.
//
// The MHD per-member arithmetic is the single-grid device code
// (col_inv_tile, row_com1_rows, col_rt_tile, row_com2_rows,
// col_fwd_com_tile), reading its argument block from the member table in
// global memory; no pointer or tensor map is staged through shared memory.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <vector>
#include "coh_impl.cuh"
#include "com_impl.cuh"
#include "diag.cuh"
#include "closure.h"

using namespace tara;

namespace {

constexpr int kEnsColThreads = 256;
constexpr int kEnsRowThreads = 352;  // 11 groups x 32
constexpr int kEnsFields = 20;
enum { EF_UA = 0, EF_UB = 3, EF_DOLD = 6, EF_H = 9, EF_X = 17 };

// kx columns per column item: CB * L / P = 256 threads
template <int L, int PC> struct EnsCol {
  static constexpr int P = L == 384 ? 24 : PC;
  static constexpr int CB = kEnsColThreads * P / L;
};
// rows per row item: rows * 11 * (M / P) = 352 threads
template <int N, int PR> struct EnsRow {
  static constexpr int M = N / 2;
  static constexpr int P = N == 384 ? 24 : PR;
  static constexpr int ROWS = kEnsRowThreads / (11 * (M / P));
};

template <class T> struct EnsMember {
  ColInvArgs<T> inv[2];         // parity p: jobs read the state in buffer p
  RowCohArgs<T> row;
  ColFwdSimpleArgs<T> fwd[2];   // parity p: state p -> state 1-p, AB2/Euler history
  int N;
};

#define TARA_ENS_SIZES(FN, ...) \
  case 128: FN(128, __VA_ARGS__); break; \
  case 256: FN(256, __VA_ARGS__); break; \
  case 384: FN(384, __VA_ARGS__); break; \
  case 512: FN(512, __VA_ARGS__); break;

// The item's argument block is copied into shared memory, where every
// thread reads it at broadcast speed (the structs hold only pointers, sizes
// and scalars, so a word copy is a valid copy).
template <class A>
__device__ __forceinline__ void stage_args(A* dst, const A* src) {
  static_assert(sizeof(A) % 4 == 0, "argument block is not a whole number of words");
  const unsigned* s = reinterpret_cast<const unsigned*>(src);
  unsigned* d = reinterpret_cast<unsigned*>(dst);
  for (int k = threadIdx.x; k < (int)(sizeof(A) / 4); k += blockDim.x) d[k] = __ldg(s + k);
  __syncthreads();
}

template <class T, int PC>
__global__ void __launch_bounds__(kEnsColThreads, 2) k_ens_col_inv(const EnsMember<T>* __restrict__ mem,
                                                                 const int4* __restrict__ items, int nitems,
                                                                 int parity) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  __shared__ __align__(16) ColInvArgs<T> a;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    stage_args(&a, &mem[w.x].inv[parity]);
#define TARA_ENS_INV(L, _)                                                                          \
  col_inv_tile<T, L, EnsCol<L, PC>::CB, EnsCol<L, PC>::P>(a.job[w.z], a.tb, w.y * EnsCol<L, PC>::CB, sm, \
                                                          threadIdx.x)
    switch (mem[w.x].N) { TARA_ENS_SIZES(TARA_ENS_INV, 0) }
#undef TARA_ENS_INV
    __syncthreads();
  }
}

// two row CTAs per SM in FP32 (80 registers, a few words spilled); FP64 keeps one
template <class T> constexpr int ens_row_minb() { return sizeof(T) == 4 ? 2 : 1; }

template <class T, int PR>
__global__ void __launch_bounds__(kEnsRowThreads, ens_row_minb<T>()) k_ens_row(const EnsMember<T>* __restrict__ mem,
                                                             const int4* __restrict__ items, int nitems) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  __shared__ __align__(16) RowCohArgs<T> a;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    stage_args(&a, &mem[w.x].row);
#define TARA_ENS_ROW(N, _) \
  row_coh_rows<T, EnsRow<N, PR>::M, EnsRow<N, PR>::P>(a, w.y * EnsRow<N, PR>::ROWS, sm)
    switch (mem[w.x].N) { TARA_ENS_SIZES(TARA_ENS_ROW, 0) }
#undef TARA_ENS_ROW
    __syncthreads();
  }
}

template <class T, int PC>
__global__ void __launch_bounds__(kEnsColThreads, 2) k_ens_col_fwd(const EnsMember<T>* __restrict__ mem,
                                                                 const int4* __restrict__ items, int nitems,
                                                                 int parity) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  __shared__ __align__(16) ColFwdSimpleArgs<T> a;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    stage_args(&a, &mem[w.x].fwd[parity]);
#define TARA_ENS_FWD(L, _) \
  col_fwd_simple_tile<T, L, EnsCol<L, PC>::CB, EnsCol<L, PC>::P>(a, w.z, w.y * EnsCol<L, PC>::CB, sm, threadIdx.x)
    switch (mem[w.x].N) { TARA_ENS_SIZES(TARA_ENS_FWD, 0) }
#undef TARA_ENS_FWD
    __syncthreads();
  }
}

// ---------------------------------------------------------------- MHD members
constexpr int kEnsComThreads = 128;
constexpr int kEnsComFields = 38;
enum { EC_UA = 0, EC_UB = 6, EC_DOLD = 12, EC_H = 18, EC_X = 25 };

// Tile geometry per grid size, with the sessions' values per thread: every
// item is one CTA of kEnsComThreads threads.
template <class T, int L> struct EnsComInv {  // column inverse and d(uy)/dy round trip
  static constexpr int P = ColCfg<T, L>::P;
  static constexpr int CB = kEnsComThreads * P / L;
  static_assert(CB * L / P == kEnsComThreads, "column tile does not fill the CTA");
};
template <class T, int L> struct EnsComFwd {  // column forward pass
  static constexpr int P = ColFwdComCfg<T, L>::P;
  static constexpr int CB = kEnsComThreads * P / L;
  static_assert(CB * L / P == kEnsComThreads, "column tile does not fill the CTA");
};
template <int N> struct EnsComRow {  // rows per item of the two row passes
  static constexpr int M = N / 2, P = RowCfg<M>::P;
  static constexpr int R1 = kEnsComThreads / (8 * (M / P));
  static constexpr int R2 = kEnsComThreads / (4 * (M / P));
  static_assert(R1 * 8 * (M / P) == kEnsComThreads && R2 * 4 * (M / P) == kEnsComThreads,
                "row block does not fill the CTA");
};

template <class T> struct EnsComMember {
  ColInvArgs<T> inv[2];      // parity p: jobs read the state in buffer p
  RowCom1Args<T> row1;
  ColRtArgs<T> rt;
  RowCom2Args<T> row2;
  ColFwdComArgs<T> fwd[2];   // parity p: state p -> state 1-p, history, half-real fields of state 1-p
  int N;
};

// registers: FP32 members fit 128 per thread (4 CTAs per SM), FP64 ones get up to 255
template <class T> constexpr int ens_com_minb() { return sizeof(T) == 4 ? 4 : 2; }

#define TARA_ENS_COM_SIZES(FN) \
  case 128: FN(128); break;    \
  case 256: FN(256); break;    \
  case 384: FN(384); break;    \
  case 512: FN(512); break;

// The five MHD phases as loops of the calling CTA over its share of a phase's
// items (item it of CTA b: it = b, b + gridDim.x, ...).
template <class T>
__device__ __forceinline__ void ens_com_inv(const EnsComMember<T>* mem, const int4* items, int nitems, int parity) {
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<T>* sm = reinterpret_cast<Cx<T>*>(smraw);
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    const EnsComMember<T>& m = mem[w.x];
    const ColInvArgs<T>& a = m.inv[parity];
#define TARA_EC_INV(L)                                                                                   \
  col_inv_tile<T, L, EnsComInv<T, L>::CB, EnsComInv<T, L>::P>(a.job[w.z], a.tb, w.y * EnsComInv<T, L>::CB, sm, \
                                                              threadIdx.x)
    switch (m.N) { TARA_ENS_COM_SIZES(TARA_EC_INV) }
#undef TARA_EC_INV
    __syncthreads();
  }
}
template <class T>
__device__ __forceinline__ void ens_com_row1(const EnsComMember<T>* mem, const int4* items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    const EnsComMember<T>& m = mem[w.x];
#define TARA_EC_ROW1(N) \
  row_com1_rows<T, EnsComRow<N>::M, EnsComRow<N>::P, false>(m.row1, w.y * EnsComRow<N>::R1)
    switch (m.N) { TARA_ENS_COM_SIZES(TARA_EC_ROW1) }
#undef TARA_EC_ROW1
    __syncthreads();
  }
}
template <class T>
__device__ __forceinline__ void ens_com_rt(const EnsComMember<T>* mem, const int4* items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    const EnsComMember<T>& m = mem[w.x];
#define TARA_EC_RT(L) col_rt_tile<T, L, EnsComInv<T, L>::CB, EnsComInv<T, L>::P>(m.rt, w.y * EnsComInv<T, L>::CB)
    switch (m.N) { TARA_ENS_COM_SIZES(TARA_EC_RT) }
#undef TARA_EC_RT
    __syncthreads();
  }
}
template <class T>
__device__ __forceinline__ void ens_com_row2(const EnsComMember<T>* mem, const int4* items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    const EnsComMember<T>& m = mem[w.x];
#define TARA_EC_ROW2(N) row_com2_rows<T, EnsComRow<N>::M, EnsComRow<N>::P, 0>(m.row2, w.y * EnsComRow<N>::R2)
    switch (m.N) { TARA_ENS_COM_SIZES(TARA_EC_ROW2) }
#undef TARA_EC_ROW2
    __syncthreads();
  }
}
template <class T>
__device__ __forceinline__ void ens_com_fwd(const EnsComMember<T>* mem, const int4* items, int nitems, int parity) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 w = items[it];
    const EnsComMember<T>& m = mem[w.x];
#define TARA_EC_FWD(L) \
  col_fwd_com_tile<T, L, EnsComFwd<T, L>::CB, EnsComFwd<T, L>::P>(m.fwd[parity], w.z, w.y * EnsComFwd<T, L>::CB)
    switch (m.N) { TARA_ENS_COM_SIZES(TARA_EC_FWD) }
#undef TARA_EC_FWD
    __syncthreads();
  }
}

// One launch per phase (the fallback where cooperative launches are not
// available).
template <class T>
__global__ void __launch_bounds__(kEnsComThreads, ens_com_minb<T>())
    k_ens_com_inv(const EnsComMember<T>* __restrict__ mem, const int4* __restrict__ items, int nitems, int parity) {
  ens_com_inv<T>(mem, items, nitems, parity);
}
template <class T>
__global__ void __launch_bounds__(kEnsComThreads, ens_com_minb<T>())
    k_ens_com_row1(const EnsComMember<T>* __restrict__ mem, const int4* __restrict__ items, int nitems) {
  ens_com_row1<T>(mem, items, nitems);
}
template <class T>
__global__ void __launch_bounds__(kEnsComThreads, ens_com_minb<T>())
    k_ens_com_rt(const EnsComMember<T>* __restrict__ mem, const int4* __restrict__ items, int nitems) {
  ens_com_rt<T>(mem, items, nitems);
}
template <class T>
__global__ void __launch_bounds__(kEnsComThreads, ens_com_minb<T>())
    k_ens_com_row2(const EnsComMember<T>* __restrict__ mem, const int4* __restrict__ items, int nitems) {
  ens_com_row2<T>(mem, items, nitems);
}
template <class T>
__global__ void __launch_bounds__(kEnsComThreads, ens_com_minb<T>())
    k_ens_com_fwd(const EnsComMember<T>* __restrict__ mem, const int4* __restrict__ items, int nitems, int parity) {
  ens_com_fwd<T>(mem, items, nitems, parity);
}

// Grid-wide barrier of a cooperative launch (every CTA resident): one
// arrival counter and a generation word in global memory, zero when the
// ensemble is made and back to a zero count after every barrier.  Thread 0
// of each CTA arrives; the last to arrive resets the count and advances the
// generation, the others wait for the generation to change for at most
// limit_ns of %globaltimer.  false (on every thread) if the wait ran out.
struct EnsGridBar {
  unsigned count;
  unsigned gen;
};
__device__ __forceinline__ bool ens_grid_sync(EnsGridBar* bar, unsigned long long limit_ns) {
  __syncthreads();
  bool ok = true;
  if (threadIdx.x == 0) {
    volatile unsigned* gen = &bar->gen;
    const unsigned g = *gen;
    __threadfence();  // this CTA's writes before its arrival
    if (atomicAdd(&bar->count, 1u) == gridDim.x - 1) {
      atomicExch(&bar->count, 0u);
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      while (*gen == g) {
        if (global_ns() - t0 > limit_ns) {
          ok = false;
          break;
        }
      }
    }
    __threadfence();  // the other CTAs' writes after the barrier
  }
  return __syncthreads_and(ok);
}

// A whole MHD ensemble step in one persistent, cooperative launch: the
// phases (column inverse where `first`, row pass 1, d(uy)/dy, row pass 2,
// column forward + update) one after another, separated by grid barriers.
// A barrier that runs out records TARA_ETIMEOUT in *status and ends the
// step (the members' state is then not advanced consistently; the host
// reports the error).
template <class T>
__global__ void __launch_bounds__(kEnsComThreads, ens_com_minb<T>())
    k_ens_com_step(const EnsComMember<T>* __restrict__ mem, const int4* __restrict__ inv, int ninv,
                   const int4* __restrict__ row1, int nrow1, const int4* __restrict__ rt, int nrt,
                   const int4* __restrict__ row2, int nrow2, const int4* __restrict__ fwd, int nfwd, int parity,
                   int first, EnsGridBar* bar, int* status, unsigned long long wait_ns) {
  auto sync = [&]() {
    if (ens_grid_sync(bar, wait_ns)) return true;
    if (threadIdx.x == 0) atomicExch(status, TARA_ETIMEOUT);
    return false;
  };
  if (first) {
    ens_com_inv<T>(mem, inv, ninv, parity);
    if (!sync()) return;
  }
  ens_com_row1<T>(mem, row1, nrow1);
  if (!sync()) return;
  ens_com_rt<T>(mem, rt, nrt);
  if (!sync()) return;
  ens_com_row2<T>(mem, row2, nrow2);
  if (!sync()) return;
  ens_com_fwd<T>(mem, fwd, nfwd, parity);
}

// dynamic shared memory of each MHD phase kernel: the largest over the sizes
template <class T> size_t ens_com_col_smem() {
  size_t m = 0;
#define TARA_EC_CS(L)                                                                                    \
  m = std::max(m, (size_t)FFTB<L, EnsComInv<T, L>::CB, EnsComInv<T, L>::P>::SMEM_ELEMS);              \
  m = std::max(m, col_fwd_com_smem_elems<T, L, EnsComFwd<T, L>::CB, EnsComFwd<T, L>::P>())
  TARA_EC_CS(128);
  TARA_EC_CS(256);
  TARA_EC_CS(384);
  TARA_EC_CS(512);
#undef TARA_EC_CS
  return m * sizeof(Cx<T>);
}
template <class T> size_t ens_com_row_smem(int pass) {
  size_t m = 0;
#define TARA_EC_RS(N)                                                                               \
  m = std::max(m, (size_t)(pass == 1 ? EnsComRow<N>::R1 * 8 : EnsComRow<N>::R2 * 5) *                 \
                      RowFFT<EnsComRow<N>::M, EnsComRow<N>::P>::SMEM_ELEMS)
  TARA_EC_RS(128);
  TARA_EC_RS(256);
  TARA_EC_RS(384);
  TARA_EC_RS(512);
#undef TARA_EC_RS
  return m * sizeof(Cx<T>);
}
template <class T> int ens_com_inv_cb(int N) {
  switch (N) {
    case 128: return EnsComInv<T, 128>::CB;
    case 256: return EnsComInv<T, 256>::CB;
    case 384: return EnsComInv<T, 384>::CB;
    default: return EnsComInv<T, 512>::CB;
  }
}
template <class T> int ens_com_fwd_cb(int N) {
  switch (N) {
    case 128: return EnsComFwd<T, 128>::CB;
    case 256: return EnsComFwd<T, 256>::CB;
    case 384: return EnsComFwd<T, 384>::CB;
    default: return EnsComFwd<T, 512>::CB;
  }
}
inline int ens_com_rows(int N, int pass) {
  switch (N) {
    case 128: return pass == 1 ? EnsComRow<128>::R1 : EnsComRow<128>::R2;
    case 256: return pass == 1 ? EnsComRow<256>::R1 : EnsComRow<256>::R2;
    case 384: return pass == 1 ? EnsComRow<384>::R1 : EnsComRow<384>::R2;
    default: return pass == 1 ? EnsComRow<512>::R1 : EnsComRow<512>::R2;
  }
}

template <class T, int PC> size_t ens_col_smem() {
  size_t m = 0;
  m = std::max(m, (size_t)FFTB<128, EnsCol<128, PC>::CB, EnsCol<128, PC>::P>::SMEM_ELEMS);
  m = std::max(m, (size_t)FFTB<256, EnsCol<256, PC>::CB, EnsCol<256, PC>::P>::SMEM_ELEMS);
  m = std::max(m, (size_t)FFTB<384, EnsCol<384, PC>::CB, EnsCol<384, PC>::P>::SMEM_ELEMS);
  m = std::max(m, (size_t)FFTB<512, EnsCol<512, PC>::CB, EnsCol<512, PC>::P>::SMEM_ELEMS);
  return m * sizeof(Cx<T>);
}
template <class T, int PR> size_t ens_row_smem() {
  size_t m = 0;
#define TARA_ENS_RS(N) \
  m = std::max(m, (size_t)EnsRow<N, PR>::ROWS * 11 * RowFFT<EnsRow<N, PR>::M, EnsRow<N, PR>::P>::SMEM_ELEMS)
  TARA_ENS_RS(128);
  TARA_ENS_RS(256);
  TARA_ENS_RS(384);
  TARA_ENS_RS(512);
#undef TARA_ENS_RS
  return m * sizeof(Cx<T>);
}
int ens_cb(int N, int pc) { return N == 384 ? kEnsColThreads * 24 / 384 : kEnsColThreads * pc / N; }
int ens_rows(int N, int pr) { return kEnsRowThreads / (11 * ((N / 2) / (N == 384 ? 24 : pr))); }

__global__ void k_ens_f64_to_f32(const double2* __restrict__ src, Cx<float>* dst, int Nh, int ld, int Ny) {
  const size_t n = (size_t)Nh * Ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    dst[(q / Nh) * ld + q % Nh] = cx<float>((float)src[q].x, (float)src[q].y);
}
__global__ void k_ens_f32_to_f64(const Cx<float>* src, double2* __restrict__ dst, int Nh, int ld, int Ny) {
  const size_t n = (size_t)Nh * Ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const Cx<float> v = src[(q / Nh) * ld + q % Nh];
    dst[q] = make_double2((double)v.x, (double)v.y);
  }
}

}  // namespace

struct tara_ensemble {
  int precision = TARA_FP32;
  int n = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[8] = {};
  int status = TARA_OK;
  virtual ~tara_ensemble() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }
  virtual int init(const int* models, const int* N, const tara_params* p) = 0;
  virtual int set_state(int m, const double* const* f, int which) = 0;
  virtual int get_state(int m, double* const* f, int which) = 0;
  virtual int step(int stepper, int nsteps) = 0;
  virtual int set_tuning(const int* t) = 0;
  virtual void get_tuning(int* t) const = 0;
  virtual int time_phases(int stepper, int reps, float* ms3) = 0;
  virtual int save_state(bool restore) = 0;
  virtual int diagnostics(int m, double* out, int nout, double* Ek, int nbins) = 0;
  virtual int num_shells(int m) = 0;
  virtual int num_fields(int m) const = 0;
  virtual int device_status() = 0;
  // FP64 MHD member m: its grid and six state fields (else TARA_EINVAL)
  virtual int member_state(int m, const void** grid, void** state6) = 0;
};

namespace {

template <class T>
struct EnsembleT : tara_ensemble {
  std::vector<int> N;
  std::vector<int> model;                                 // TARA_MODEL_COH or TARA_MODEL_COM per member
  std::vector<int> slot;                                  // index of the member in hmem or hcom
  int nhyd = 0, ncom = 0;
  std::vector<tara_params> prm;
  std::map<int, std::unique_ptr<Grid<T>>> grids;        // tables per grid size
  std::map<int, std::unique_ptr<DiagWork<T>>> diags;
  std::vector<size_t> off;                                // element offset of each member block
  std::vector<size_t> elems;                              // elements per field of each member
  Cx<T>* arena = nullptr;
  double* stage = nullptr;                                // FP64 host-layout staging (largest member)
  double* drec = nullptr;                                 // one diagnostics record
  EnsMember<T>* dmem = nullptr;                           // hydro member table
  std::vector<EnsMember<T>> hmem;
  int4* ditems[3] = {nullptr, nullptr, nullptr};
  int nitems[3] = {0, 0, 0};
  EnsComMember<T>* dcom = nullptr;                        // MHD member table
  std::vector<EnsComMember<T>> hcom;
  int4* citems[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // inv, row1, rt, row2, fwd
  int ncitems[5] = {0, 0, 0, 0, 0};
  // the MHD members' half-real fields hold the y-inverse of their current
  // state (written by the previous column forward pass)
  bool com_h_valid = false;
  // MHD step as one cooperative launch (else one launch per phase)
  bool com_coop = false;
  EnsGridBar* dbar = nullptr;
  int tuning[6] = {16, 16, 16, 0, 0, 0};  // P col_inv, P row, P col_fwd, CTAs/SM of each (0 = most that fit)
  int parity = 0;
  int built_mode = -1;
  Cx<T>* backup = nullptr;
  size_t backup_elems = 0;
  int saved_parity = 0;
  cudaGraphExec_t graph = nullptr;
  int graph_mode = -1, graph_parity = -1;

  ~EnsembleT() override {
    if (st) cudaStreamSynchronize(st);
    drop_graph();
    for (auto& d : diags) d.second->release();
    for (auto& g : grids) g.second->release();
    for (auto& p : ditems)
      if (p) cudaFree(p);
    for (auto& p : citems)
      if (p) cudaFree(p);
    if (dmem) cudaFree(dmem);
    if (dcom) cudaFree(dcom);
    if (dbar) cudaFree(dbar);
    if (arena) cudaFree(arena);
    if (stage) cudaFree(stage);
    if (drec) cudaFree(drec);
    if (backup) cudaFree(backup);
  }
  void drop_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graph_mode = graph_parity = -1;
  }
  Cx<T>* field(int m, int f) const { return arena + off[m] + (size_t)f * elems[m]; }

  int nfields(int m) const { return model[m] == TARA_MODEL_COM ? 6 : 3; }
  int num_fields(int m) const override { return m >= 0 && m < n ? nfields(m) : 0; }
  int member_state(int m, const void** grid, void** state6) override {
    if (m < 0 || m >= n || model[m] != TARA_MODEL_COM || sizeof(T) != sizeof(double)) {
      set_error("training pairs come from an FP64 MHD ensemble member");
      return TARA_EINVAL;
    }
    *grid = grids[N[m]].get();
    for (int q = 0; q < 6; q++) state6[q] = fptr(m, 0, q);
    return TARA_OK;
  }
  int init(const int* models, const int* Nin, const tara_params* p) override {
    N.assign(Nin, Nin + n);
    model.assign(models, models + n);
    prm.assign(p, p + n);
    size_t total = 0, maxh = 0;
    off.resize(n);
    elems.resize(n);
    slot.resize(n);
    for (int m = 0; m < n; m++) {
      if (N[m] != 128 && N[m] != 256 && N[m] != 384 && N[m] != 512) {
        set_error("ensemble member grid sizes must be 128, 256, 384 or 512");
        return TARA_EUNSUPPORTED;
      }
      if (model[m] != TARA_MODEL_COH && model[m] != TARA_MODEL_COM) {
        set_error("ensemble members run the hydro or the MHD model");
        return TARA_EUNSUPPORTED;
      }
      if (model[m] == TARA_MODEL_COM && (p[m].A != 0.0 || p[m].fix_curlB != 0)) {
        set_error("MHD ensemble members run without forcing (A = 0) and with curl B as the reference builds it");
        return TARA_EUNSUPPORTED;
      }
      slot[m] = model[m] == TARA_MODEL_COM ? ncom++ : nhyd++;
      auto& g = grids[N[m]];
      if (!g) {
        g.reset(new Grid<T>());
        TARA_TRY(g->init(N[m], N[m], p[m].Lx, p[m].Ly, p[m].pi, st));
      } else if (g->Lx != p[m].Lx || g->Ly != p[m].Ly || g->pi != p[m].pi) {
        set_error("ensemble members of one grid size must share Lx, Ly and pi");
        return TARA_EINVAL;
      }
      off[m] = total;
      elems[m] = g->field_elems();
      total += elems[m] * (model[m] == TARA_MODEL_COM ? kEnsComFields : kEnsFields);
      maxh = std::max(maxh, (size_t)(N[m] / 2 + 1) * N[m]);
    }
    if (cudaMalloc(&arena, total * sizeof(Cx<T>)) != cudaSuccess) {
      arena = nullptr;
      set_error("cudaMalloc of the ensemble arena (" + std::to_string(total * sizeof(Cx<T>)) + " bytes) failed");
      return TARA_ENOMEM;
    }
    TARA_CUDA_TRY(cudaMemsetAsync(arena, 0, total * sizeof(Cx<T>), st));
    TARA_CUDA_TRY(cudaMalloc(&stage, maxh * sizeof(Cx<double>)));
    TARA_CUDA_TRY(cudaMalloc(&drec, (kDiagOut + 1024) * sizeof(double)));
    if (nhyd) TARA_CUDA_TRY(cudaMalloc(&dmem, (size_t)nhyd * sizeof(EnsMember<T>)));
    if (ncom) {
      TARA_CUDA_TRY(cudaMalloc(&dcom, (size_t)ncom * sizeof(EnsComMember<T>)));
      int dev = 0, coop = 0;
      TARA_CUDA_TRY(cudaGetDevice(&dev));
      TARA_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
      if (coop) {
        TARA_CUDA_TRY(cudaMalloc(&dbar, sizeof(EnsGridBar)));
        TARA_CUDA_TRY(cudaMemsetAsync(dbar, 0, sizeof(EnsGridBar), st));
        com_coop = true;
      }
    }
    build_members();
    TARA_TRY(upload_members());
    TARA_TRY(build_items());
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }

  int upload_members() {
    if (nhyd)
      TARA_CUDA_TRY(cudaMemcpyAsync(dmem, hmem.data(), (size_t)nhyd * sizeof(EnsMember<T>), cudaMemcpyHostToDevice, st));
    if (ncom)
      TARA_CUDA_TRY(cudaMemcpyAsync(dcom, hcom.data(), (size_t)ncom * sizeof(EnsComMember<T>), cudaMemcpyHostToDevice,
                                    st));
    return TARA_OK;
  }
  // argument blocks of an MHD member (src/derive2com.f95 per member)
  void build_com_member(int m) {
    EnsComMember<T>& e = hcom[slot[m]];
    const Tables<T>& tb = grids[N[m]]->tb;
    const tara_params& q = prm[m];
    e.N = N[m];
    Cx<T>* H[7];
    Cx<T>* X[13];
    for (int k = 0; k < 7; k++) H[k] = field(m, EC_H + k);
    for (int k = 0; k < 13; k++) X[k] = field(m, EC_X + k);
    for (int par = 0; par < 2; par++) {
      const int ubase = par ? EC_UB : EC_UA, nbase = par ? EC_UA : EC_UB;
      e.inv[par].tb = tb;
      for (int k = 0; k < 6; k++) e.inv[par].job[k] = ColInvJob<T>{field(m, ubase + k), H[k], MUL_ONE, (T)0};
      ColFwdComArgs<T>& f = e.fwd[par];
      f.tb = tb;
      for (int k = 0; k < 13; k++) f.X[k] = X[k];
      for (int k = 0; k < 6; k++) {
        f.in[k] = field(m, ubase + k);
        f.hnext[k] = H[k];
        f.step.u[k] = field(m, ubase + k);
        f.step.unew[k] = field(m, nbase + k);
        f.step.dold[k] = field(m, EC_DOLD + k);
      }
      f.mu = (T)q.mu;
      f.eta = (T)q.eta;
      f.forcing = 0;
      f.closure = 0;
      f.fuse = 1;
      f.hikybx = nullptr;
      f.step.dt = (T)q.dt;
      f.step.scale = nullptr;
    }
    RowCom1Args<T>& r1 = e.row1;
    r1.tb = tb;
    for (int k = 0; k < 6; k++) r1.H[k] = H[k];
    for (int k = 0; k < 11; k++) r1.X[k] = X[k];
    r1.cs2 = (T)(q.CS * q.CS);
    r1.rb = ens_com_rows(N[m], 1);
    r1.cfl = CflRow{nullptr, 0.0, 0.0, 0.0};
    e.rt.tb = tb;
    e.rt.src = X[XUY];
    e.rt.dst = H[HDUY];
    e.rt.mul = MUL_IKY;
    RowCom2Args<T>& r2 = e.row2;
    r2.tb = tb;
    r2.Xux = X[XUX];
    r2.Hduy = H[HDUY];
    r2.Hbx = H[HBX];
    r2.Hby = H[HBY];
    r2.Hikybx = nullptr;
    r2.Xex2 = X[XEX2];
    r2.Xey2 = X[XEY2];
    r2.Xev = X[XEV];
    r2.eta = (T)q.eta;
    r2.inv_nx = (T)(1.0 / N[m]);
    r2.rb = ens_com_rows(N[m], 2);
  }
  void build_members() {
    hmem.assign(nhyd, EnsMember<T>{});
    hcom.assign(ncom, EnsComMember<T>{});
    for (int m = 0; m < n; m++) {
      if (model[m] == TARA_MODEL_COM) {
        build_com_member(m);
        continue;
      }
      EnsMember<T>& e = hmem[slot[m]];
      const Tables<T>& tb = grids[N[m]]->tb;
      e.N = N[m];
      const int src[8] = {0, 0, 1, 1, 1, 2, 2, 2};
      const int mul[8] = {MUL_ONE, MUL_IKY, MUL_ONE, MUL_IKY, MUL_KY2, MUL_ONE, MUL_IKY, MUL_KY2};
      for (int par = 0; par < 2; par++) {
        const int ubase = par ? EF_UB : EF_UA, nbase = par ? EF_UA : EF_UB;
        e.inv[par].tb = tb;
        for (int q = 0; q < 8; q++) e.inv[par].job[q] = ColInvJob<T>{field(m, ubase + src[q]), field(m, EF_H + q), mul[q], (T)0};
        ColFwdSimpleArgs<T>& f = e.fwd[par];
        f.tb = tb;
        for (int q = 0; q < 3; q++) {
          f.X[q] = field(m, EF_X + q);
          f.sign[q] = (T)-1;
          f.step.u[q] = field(m, ubase + q);
          f.step.unew[q] = field(m, nbase + q);
          f.step.dold[q] = field(m, EF_DOLD + q);
        }
        f.step.dt = (T)prm[m].dt;
      }
      e.row.tb = tb;
      for (int q = 0; q < 8; q++) e.row.H[q] = field(m, EF_H + q);
      for (int q = 0; q < 3; q++) e.row.X[q] = field(m, EF_X + q);
      e.row.mux = (T)prm[m].mux;
      e.row.muy = (T)prm[m].muy;
      e.row.cs2 = (T)(prm[m].CS * prm[m].CS);
    }
  }
  int set_mode(int mode) {
    if (mode == built_mode) return TARA_OK;
    for (auto& e : hmem)
      for (auto& f : e.fwd) f.step.mode = mode;
    for (auto& e : hcom)
      for (auto& f : e.fwd) f.step.mode = mode;
    TARA_TRY(upload_members());
    built_mode = mode;
    return TARA_OK;
  }

  int build_items() {
    std::vector<int> order(n);
    for (int m = 0; m < n; m++) order[m] = m;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return N[a] > N[b]; });
    std::vector<int4> it[3], ic[5];
    for (int m : order) {
      const int Nh = N[m] / 2 + 1;
      if (model[m] == TARA_MODEL_COM) {
        const int s = slot[m];
        const int ti = (Nh + ens_com_inv_cb<T>(N[m]) - 1) / ens_com_inv_cb<T>(N[m]);
        const int tf = (Nh + ens_com_fwd_cb<T>(N[m]) - 1) / ens_com_fwd_cb<T>(N[m]);
        for (int t = 0; t < ti; t++)
          for (int j = 0; j < 6; j++) ic[0].push_back(make_int4(s, t, j, 0));
        for (int r = 0; r < N[m] / ens_com_rows(N[m], 1); r++) ic[1].push_back(make_int4(s, r, 0, 0));
        for (int t = 0; t < ti; t++) ic[2].push_back(make_int4(s, t, 0, 0));
        for (int r = 0; r < N[m] / ens_com_rows(N[m], 2); r++) ic[3].push_back(make_int4(s, r, 0, 0));
        for (int t = 0; t < tf; t++)
          for (int f = 0; f < 6; f++) ic[4].push_back(make_int4(s, t, f, 0));
        continue;
      }
      const int hs = slot[m];
      const int ti = (Nh + ens_cb(N[m], tuning[0]) - 1) / ens_cb(N[m], tuning[0]);
      for (int t = 0; t < ti; t++)
        for (int j = 0; j < 8; j++) it[0].push_back(make_int4(hs, t, j, 0));
      const int rows = ens_rows(N[m], tuning[1]);
      for (int r = 0; r < N[m] / rows; r++) it[1].push_back(make_int4(hs, r, 0, 0));
      const int tf = (Nh + ens_cb(N[m], tuning[2]) - 1) / ens_cb(N[m], tuning[2]);
      for (int t = 0; t < tf; t++)
        for (int f = 0; f < 3; f++) it[2].push_back(make_int4(hs, t, f, 0));
    }
    auto upload = [&](std::vector<int4>& v, int4*& d, int& nd) -> int {
      if (d) cudaFree(d);
      d = nullptr;
      nd = (int)v.size();
      if (v.empty()) return TARA_OK;
      TARA_CUDA_TRY(cudaMalloc(&d, v.size() * sizeof(int4)));
      TARA_CUDA_TRY(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
      return TARA_OK;
    };
    for (int k = 0; k < 3; k++) TARA_TRY(upload(it[k], ditems[k], nitems[k]));
    for (int k = 0; k < 5; k++) TARA_TRY(upload(ic[k], citems[k], ncitems[k]));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }

  template <class K>
  int grid_of(K kern, int threads, size_t smem, int want, int& grid) {
    if (smem > 48 * 1024) TARA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per = 0;
    TARA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem));
    if (per < 1) { set_error("ensemble kernel does not fit on a multiprocessor"); return TARA_EUNSUPPORTED; }
    if (want > 0 && want < per) per = want;
    grid = per * grids.begin()->second->tb.sm_count;
    return TARA_OK;
  }
  int launch_inv(int par) {
    if (!nitems[0]) return TARA_OK;
    int grid = 0;
    if (tuning[0] == 8) {
      const size_t smem = ens_col_smem<T, 8>();
      TARA_TRY(grid_of(k_ens_col_inv<T, 8>, kEnsColThreads, smem, tuning[3], grid));
      k_ens_col_inv<T, 8><<<std::min(grid, nitems[0]), kEnsColThreads, smem, st>>>(dmem, ditems[0], nitems[0], par);
    } else {
      const size_t smem = ens_col_smem<T, 16>();
      TARA_TRY(grid_of(k_ens_col_inv<T, 16>, kEnsColThreads, smem, tuning[3], grid));
      k_ens_col_inv<T, 16><<<std::min(grid, nitems[0]), kEnsColThreads, smem, st>>>(dmem, ditems[0], nitems[0], par);
    }
    return TARA_OK;
  }
  int launch_row() {
    if (!nitems[1]) return TARA_OK;
    int grid = 0;
    if (tuning[1] == 8) {
      const size_t smem = ens_row_smem<T, 8>();
      TARA_TRY(grid_of(k_ens_row<T, 8>, kEnsRowThreads, smem, tuning[4], grid));
      k_ens_row<T, 8><<<std::min(grid, nitems[1]), kEnsRowThreads, smem, st>>>(dmem, ditems[1], nitems[1]);
    } else {
      const size_t smem = ens_row_smem<T, 16>();
      TARA_TRY(grid_of(k_ens_row<T, 16>, kEnsRowThreads, smem, tuning[4], grid));
      k_ens_row<T, 16><<<std::min(grid, nitems[1]), kEnsRowThreads, smem, st>>>(dmem, ditems[1], nitems[1]);
    }
    return TARA_OK;
  }
  int launch_fwd(int par) {
    if (!nitems[2]) return TARA_OK;
    int grid = 0;
    if (tuning[2] == 8) {
      const size_t smem = ens_col_smem<T, 8>();
      TARA_TRY(grid_of(k_ens_col_fwd<T, 8>, kEnsColThreads, smem, tuning[5], grid));
      k_ens_col_fwd<T, 8><<<std::min(grid, nitems[2]), kEnsColThreads, smem, st>>>(dmem, ditems[2], nitems[2], par);
    } else {
      const size_t smem = ens_col_smem<T, 16>();
      TARA_TRY(grid_of(k_ens_col_fwd<T, 16>, kEnsColThreads, smem, tuning[5], grid));
      k_ens_col_fwd<T, 16><<<std::min(grid, nitems[2]), kEnsColThreads, smem, st>>>(dmem, ditems[2], nitems[2], par);
    }
    return TARA_OK;
  }
  // MHD phase ph (0 column inverse, 1 row pass 1, 2 d(uy)/dy, 3 row pass 2,
  // 4 column forward + update) over every MHD member
  int launch_com(int ph, int par) {
    if (!ncitems[ph]) return TARA_OK;
    int grid = 0;
    const int ni = ncitems[ph];
    switch (ph) {
      case 0: {
        const size_t smem = ens_com_col_smem<T>();
        TARA_TRY(grid_of(k_ens_com_inv<T>, kEnsComThreads, smem, 0, grid));
        k_ens_com_inv<T><<<std::min(grid, ni), kEnsComThreads, smem, st>>>(dcom, citems[0], ni, par);
        break;
      }
      case 1: {
        const size_t smem = ens_com_row_smem<T>(1);
        TARA_TRY(grid_of(k_ens_com_row1<T>, kEnsComThreads, smem, 0, grid));
        k_ens_com_row1<T><<<std::min(grid, ni), kEnsComThreads, smem, st>>>(dcom, citems[1], ni);
        break;
      }
      case 2: {
        const size_t smem = ens_com_col_smem<T>();
        TARA_TRY(grid_of(k_ens_com_rt<T>, kEnsComThreads, smem, 0, grid));
        k_ens_com_rt<T><<<std::min(grid, ni), kEnsComThreads, smem, st>>>(dcom, citems[2], ni);
        break;
      }
      case 3: {
        const size_t smem = ens_com_row_smem<T>(2);
        TARA_TRY(grid_of(k_ens_com_row2<T>, kEnsComThreads, smem, 0, grid));
        k_ens_com_row2<T><<<std::min(grid, ni), kEnsComThreads, smem, st>>>(dcom, citems[3], ni);
        break;
      }
      default: {
        const size_t smem = ens_com_col_smem<T>();
        TARA_TRY(grid_of(k_ens_com_fwd<T>, kEnsComThreads, smem, 0, grid));
        k_ens_com_fwd<T><<<std::min(grid, ni), kEnsComThreads, smem, st>>>(dcom, citems[4], ni, par);
        break;
      }
    }
    return TARA_OK;
  }
  // the MHD phases of one step in one cooperative launch: as many CTAs as are
  // resident at once (the grid barriers need all of them)
  int launch_com_step(int par, bool first) {
    const size_t smem =
        std::max(ens_com_col_smem<T>(), std::max(ens_com_row_smem<T>(1), ens_com_row_smem<T>(2)));
    int grid = 0;
    TARA_TRY(grid_of(k_ens_com_step<T>, kEnsComThreads, smem, 0, grid));
    const Tables<T>& tb = grids.begin()->second->tb;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kEnsComThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    TARA_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_ens_com_step<T>, (const EnsComMember<T>*)dcom, (const int4*)citems[0],
                                     ncitems[0], (const int4*)citems[1], ncitems[1], (const int4*)citems[2],
                                     ncitems[2], (const int4*)citems[3], ncitems[3], (const int4*)citems[4],
                                     ncitems[4], par, first ? 1 : 0, dbar, tb.status, tb.wait_ns));
    return TARA_OK;
  }
  int launch_steps(int n_) {
    for (int s = 0; s < n_; s++) {
      TARA_TRY(launch_inv(parity));
      TARA_TRY(launch_row());
      TARA_TRY(launch_fwd(parity));
      if (ncom) {
        if (com_coop) {
          TARA_TRY(launch_com_step(parity, !com_h_valid));
        } else {
          for (int ph = com_h_valid ? 1 : 0; ph < 5; ph++) TARA_TRY(launch_com(ph, parity));
        }
        com_h_valid = true;  // the column forward pass wrote the y-inverse of the new state
      }
      TARA_CUDA_TRY(cudaGetLastError());
      parity ^= 1;
    }
    return TARA_OK;
  }
  int step(int stepper, int nsteps) override {
    if (stepper != TARA_STEP_AB2 && stepper != TARA_STEP_EULER) {
      set_error("ensembles step with AB2 or Euler");
      return TARA_EINVAL;
    }
    const int mode = stepper == TARA_STEP_AB2 ? STEP_AB2 : STEP_EULER;
    if (mode != built_mode) {
      drop_graph();
      TARA_TRY(set_mode(mode));
    }
    int done = 0;
    if (ncom && !com_h_valid && nsteps > 0) {
      // the MHD members' first step includes their column inverse; captured
      // step pairs start from half-real fields written by a step
      TARA_TRY(launch_steps(1));
      done = 1;
    }
    if (nsteps - done >= 2) {
      if (!graph || graph_mode != mode || graph_parity != parity) {
        drop_graph();
        const int p0 = parity;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
          const int r = launch_steps(2);
          const cudaError_t e = cudaStreamEndCapture(st, &g);
          if (r == TARA_OK && e == cudaSuccess && g && cudaGraphInstantiate(&graph, g, 0) != cudaSuccess) graph = nullptr;
          if (g) cudaGraphDestroy(g);
          cudaGetLastError();
        }
        parity = p0;  // nothing ran while capturing
        if (graph) {
          graph_mode = mode;
          graph_parity = parity;
        }
      }
      if (graph)
        for (; done + 2 <= nsteps; done += 2) TARA_CUDA_TRY(cudaGraphLaunch(graph, st));
    }
    return launch_steps(nsteps - done);
  }

  int set_tuning(const int* t) override {
    for (int k = 0; k < 3; k++)
      if (t[k] != 8 && t[k] != 16) { set_error("values per thread must be 8 or 16"); return TARA_EINVAL; }
    for (int k = 3; k < 6; k++)
      if (t[k] < 0) { set_error("CTAs per SM must be >= 0"); return TARA_EINVAL; }
    const bool items_change = t[0] != tuning[0] || t[1] != tuning[1] || t[2] != tuning[2];
    std::memcpy(tuning, t, sizeof(tuning));
    drop_graph();
    if (items_change) TARA_TRY(build_items());
    return TARA_OK;
  }
  void get_tuning(int* t) const override { std::memcpy(t, tuning, sizeof(tuning)); }

  // device time of each phase summed over `reps` steps (host launches)
  int time_phases(int stepper, int reps, float* ms3) override {
    const int mode = stepper == TARA_STEP_AB2 ? STEP_AB2 : STEP_EULER;
    drop_graph();
    TARA_TRY(set_mode(mode));
    for (int k = 0; k < 3; k++) ms3[k] = 0;
    for (auto& e : ev)
      if (!e) TARA_CUDA_TRY(cudaEventCreate(&e));
    for (int r = 0; r < reps; r++) {
      TARA_CUDA_TRY(cudaEventRecord(ev[0], st));
      TARA_TRY(launch_inv(parity));
      TARA_CUDA_TRY(cudaEventRecord(ev[1], st));
      TARA_TRY(launch_row());
      TARA_CUDA_TRY(cudaEventRecord(ev[2], st));
      TARA_TRY(launch_fwd(parity));
      TARA_CUDA_TRY(cudaEventRecord(ev[3], st));
      TARA_CUDA_TRY(cudaEventSynchronize(ev[3]));
      for (int k = 0; k < 3; k++) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
        ms3[k] += t;
      }
      parity ^= 1;
    }
    return device_status();
  }
  // copy of every member's state and AB2 history (restore = true puts it back)
  int save_state(bool restore) override {
    size_t need = 0;
    for (int m = 0; m < n; m++) need += 3 * nfields(m) * elems[m];
    if (!restore) {
      if (!backup) {
        if (cudaMalloc(&backup, need * sizeof(Cx<T>)) != cudaSuccess) {
          backup = nullptr;
          set_error("cudaMalloc of the tuning backup failed");
          return TARA_ENOMEM;
        }
        backup_elems = need;
      }
      saved_parity = parity;
    } else if (!backup) {
      set_error("no saved state");
      return TARA_EINVAL;
    }
    size_t o = 0;
    for (int m = 0; m < n; m++) {  // u_A, u_B, history: the first 3 nf fields of the member's block
      const size_t b = 3 * nfields(m) * elems[m] * sizeof(Cx<T>);
      if (restore) TARA_CUDA_TRY(cudaMemcpyAsync(field(m, 0), backup + o, b, cudaMemcpyDeviceToDevice, st));
      else TARA_CUDA_TRY(cudaMemcpyAsync(backup + o, field(m, 0), b, cudaMemcpyDeviceToDevice, st));
      o += 3 * nfields(m) * elems[m];
    }
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    if (restore) {
      cudaFree(backup);
      backup = nullptr;
      parity = saved_parity;
      com_h_valid = false;
      drop_graph();
    }
    return TARA_OK;
  }

  int device_status() override {
    int v = 0;
    for (auto& g : grids) {
      int s = 0;
      TARA_CUDA_TRY(cudaMemcpyAsync(&s, g.second->tb.status, sizeof(int), cudaMemcpyDeviceToHost, st));
      TARA_CUDA_TRY(cudaStreamSynchronize(st));
      if (s != TARA_OK) {
        const int zero = 0;
        cudaMemcpyAsync(g.second->tb.status, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
        v = s;
      }
    }
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    if (v) set_error("a bounded wait ran out in a kernel");
    return v;
  }

  // which: 0 state, 1 AB2 history
  Cx<T>* fptr(int m, int which, int q) {
    if (model[m] == TARA_MODEL_COM) return field(m, which ? EC_DOLD + q : (parity ? EC_UB : EC_UA) + q);
    return field(m, which ? EF_DOLD + q : (parity ? EF_UB : EF_UA) + q);
  }
  int set_state(int m, const double* const* h, int which) override {
    if (m < 0 || m >= n || !h) { set_error("bad member or null field array"); return TARA_EINVAL; }
    const int Nh = N[m] / 2 + 1, ld = grids[N[m]]->ld;
    if (which == 0 && model[m] == TARA_MODEL_COM) com_h_valid = false;
    for (int q = 0; q < nfields(m); q++) {
      if (!h[q]) { set_error("null host field pointer"); return TARA_EINVAL; }
      if constexpr (sizeof(T) == sizeof(double)) {
        TARA_CUDA_TRY(cudaMemcpy2DAsync(fptr(m, which, q), ld * sizeof(Cx<T>), h[q], Nh * sizeof(Cx<double>),
                                        Nh * sizeof(Cx<double>), N[m], cudaMemcpyHostToDevice, st));
      } else {
        TARA_CUDA_TRY(cudaMemcpyAsync(stage, h[q], (size_t)Nh * N[m] * sizeof(Cx<double>), cudaMemcpyHostToDevice, st));
        k_ens_f64_to_f32<<<256, 256, 0, st>>>(reinterpret_cast<const double2*>(stage),
                                              reinterpret_cast<Cx<float>*>(fptr(m, which, q)), Nh, ld, N[m]);
        TARA_CUDA_TRY(cudaGetLastError());
      }
    }
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }
  int get_state(int m, double* const* h, int which) override {
    if (m < 0 || m >= n || !h) { set_error("bad member or null field array"); return TARA_EINVAL; }
    const int Nh = N[m] / 2 + 1, ld = grids[N[m]]->ld;
    for (int q = 0; q < nfields(m); q++) {
      if (!h[q]) { set_error("null host field pointer"); return TARA_EINVAL; }
      if constexpr (sizeof(T) == sizeof(double)) {
        TARA_CUDA_TRY(cudaMemcpy2DAsync(h[q], Nh * sizeof(Cx<double>), fptr(m, which, q), ld * sizeof(Cx<T>),
                                        Nh * sizeof(Cx<double>), N[m], cudaMemcpyDeviceToHost, st));
      } else {
        k_ens_f32_to_f64<<<256, 256, 0, st>>>(reinterpret_cast<const Cx<float>*>(fptr(m, which, q)),
                                              reinterpret_cast<double2*>(stage), Nh, ld, N[m]);
        TARA_CUDA_TRY(cudaGetLastError());
        TARA_CUDA_TRY(cudaMemcpyAsync(h[q], stage, (size_t)Nh * N[m] * sizeof(Cx<double>), cudaMemcpyDeviceToHost, st));
      }
      TARA_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return device_status();
  }

  int num_shells(int m) override {
    if (m < 0 || m >= n) return 0;
    return diag_num_shells(N[m], N[m], prm[m].Lx, prm[m].Ly, prm[m].pi);
  }
  int diagnostics(int m, double* out, int nout, double* Ek, int nbins) override {
    if (m < 0 || m >= n) { set_error("bad member"); return TARA_EINVAL; }
    const int ns = num_shells(m);
    if (nout > kDiagOut || nbins > ns || ns > 1024) { set_error("more values requested than computed"); return TARA_EINVAL; }
    Grid<T>& g = *grids[N[m]];
    auto& dw = diags[N[m]];
    if (!dw) {
      dw.reset(new DiagWork<T>());
      TARA_TRY(dw->alloc(g, st));
    }
    if (model[m] == TARA_MODEL_COM) {
      // the half-real and x-transformed work fields are the diagnostics' scratch
      FieldPool<T> H{field(m, EC_H), elems[m], 7}, X{field(m, EC_X), elems[m], 13};
      FieldPool<T> spec{field(m, EC_X + 2), elems[m], 2};
      Cx<T>* state[6];
      for (int q = 0; q < 6; q++) state[q] = fptr(m, 0, q);
      com_h_valid = false;
      TARA_TRY(diag_record(TARA_MODEL_COM, g, *dw, state, H, X, spec, drec, st));
    } else {
      FieldPool<T> H{field(m, EF_H), elems[m], 8}, X{field(m, EF_X), elems[m], 3};
      Cx<T>* state[3] = {fptr(m, 0, 0), fptr(m, 0, 1), fptr(m, 0, 2)};
      TARA_TRY(diag_record(TARA_MODEL_COH, g, *dw, state, H, X, X, drec, st));
    }
    std::vector<double> rec(kDiagOut + ns);
    TARA_CUDA_TRY(cudaMemcpyAsync(rec.data(), drec, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    for (int k = 0; k < nout; k++) out[k] = rec[k];
    for (int k = 0; k < nbins; k++) Ek[k] = rec[kDiagOut + k];
    return device_status();
  }
};

}  // namespace

namespace tara {
int ens_member_state(tara_ensemble* e, int m, const Grid<double>** g, Cx<double>** state6, cudaStream_t* st) {
  const void* gp = nullptr;
  void* sp[6];
  const int r = e->member_state(m, &gp, sp);
  if (r != TARA_OK) return r;
  *g = static_cast<const Grid<double>*>(gp);
  for (int q = 0; q < 6; q++) state6[q] = static_cast<Cx<double>*>(sp[q]);
  *st = e->st;
  return TARA_OK;
}
}  // namespace tara

extern "C" {

int tara_ens_open_mixed(tara_ensemble** out, int n, const int* models, const int* N, const tara_params* params,
                        int precision) {
  if (!out || !models || !N || !params || n < 1) { set_error("null argument or empty ensemble"); return TARA_EINVAL; }
  *out = nullptr;
  if (precision != TARA_FP32 && precision != TARA_FP64) { set_error("unknown precision"); return TARA_EINVAL; }
  std::unique_ptr<tara_ensemble> e(precision == TARA_FP32 ? (tara_ensemble*)new EnsembleT<float>()
                                                          : (tara_ensemble*)new EnsembleT<double>());
  e->precision = precision;
  e->n = n;
  if (cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("cudaStreamCreate failed");
    return TARA_ECUDA;
  }
  const int r = e->init(models, N, params);
  if (r != TARA_OK) return r;
  *out = e.release();
  return TARA_OK;
}
int tara_ens_open(tara_ensemble** out, int model, int n, const int* N, const tara_params* params, int precision) {
  if (!out || n < 1) { set_error("null argument or empty ensemble"); return TARA_EINVAL; }
  *out = nullptr;
  if (model != TARA_MODEL_COH && model != TARA_MODEL_COM) {
    set_error("ensembles run the hydro or the MHD model");
    return TARA_EUNSUPPORTED;
  }
  std::vector<int> models(n, model);
  return tara_ens_open_mixed(out, n, models.data(), N, params, precision);
}
int tara_ens_num_fields(const tara_ensemble* e, int member) { return e ? e->num_fields(member) : 0; }
int tara_ens_close(tara_ensemble* e) {
  if (!e) return TARA_EINVAL;
  delete e;
  return TARA_OK;
}
int tara_ens_size(const tara_ensemble* e) { return e ? e->n : 0; }
int tara_ens_set_state(tara_ensemble* e, int m, const double* const* f) { return e ? e->set_state(m, f, 0) : TARA_EINVAL; }
int tara_ens_get_state(tara_ensemble* e, int m, double* const* f) { return e ? e->get_state(m, f, 0) : TARA_EINVAL; }
int tara_ens_get_history(tara_ensemble* e, int m, double* const* f) { return e ? e->get_state(m, f, 1) : TARA_EINVAL; }
int tara_ens_step(tara_ensemble* e, int stepper, int nsteps) {
  if (!e || nsteps < 0) return TARA_EINVAL;
  return e->step(stepper, nsteps);
}
int tara_ens_time_steps(tara_ensemble* e, int stepper, int nsteps, float* ms) {
  if (!e || !ms || nsteps < 0) return TARA_EINVAL;
  if (cudaStreamSynchronize(e->st) != cudaSuccess) return TARA_ECUDA;
  for (int k = 0; k < 2; k++)
    if (!e->ev[4 + k] && cudaEventCreate(&e->ev[4 + k]) != cudaSuccess) return TARA_ECUDA;
  cudaEventRecord(e->ev[4], e->st);
  int r = e->step(stepper, nsteps);
  if (r != TARA_OK) return r;
  cudaEventRecord(e->ev[5], e->st);
  if (cudaEventSynchronize(e->ev[5]) != cudaSuccess) {
    set_error("cudaEventSynchronize failed");
    return TARA_ECUDA;
  }
  cudaEventElapsedTime(ms, e->ev[4], e->ev[5]);
  return e->device_status();
}
int tara_ens_set_tuning(tara_ensemble* e, const int* t) { return e && t ? e->set_tuning(t) : TARA_EINVAL; }
int tara_ens_get_tuning(const tara_ensemble* e, int* t) {
  if (!e || !t) return TARA_EINVAL;
  e->get_tuning(t);
  return TARA_OK;
}

// Times each phase kernel under every candidate (values per thread 8/16,
// 1, 2 or all CTAs per SM that fit) on the ensemble's own members and keeps
// the fastest per phase.  The state and AB2 history are restored afterwards.
int tara_ens_autotune(tara_ensemble* e, int stepper, int reps, int* chosen, float* best_ms) {
  if (!e || reps < 1) return TARA_EINVAL;
  int r = e->save_state(false);
  if (r != TARA_OK) return r;
  int t[6];
  e->get_tuning(t);
  const int pvals[2] = {8, 16}, occ[3] = {1, 2, 0};
  float best[3] = {1e30f, 1e30f, 1e30f};
  int bestp[3] = {t[0], t[1], t[2]}, besto[3] = {t[3], t[4], t[5]};
  for (int pi = 0; pi < 2 && r == TARA_OK; pi++)
    for (int oi = 0; oi < 3 && r == TARA_OK; oi++) {
      int c[6] = {pvals[pi], pvals[pi], pvals[pi], occ[oi], occ[oi], occ[oi]};
      r = e->set_tuning(c);
      float ms[3];
      if (r == TARA_OK) r = e->time_phases(stepper, 1, ms);     // warm-up
      if (r == TARA_OK) r = e->time_phases(stepper, reps, ms);
      if (r != TARA_OK) break;
      for (int k = 0; k < 3; k++)
        if (ms[k] < best[k]) {
          best[k] = ms[k];
          bestp[k] = pvals[pi];
          besto[k] = occ[oi];
        }
    }
  const int fin[6] = {bestp[0], bestp[1], bestp[2], besto[0], besto[1], besto[2]};
  if (r == TARA_OK) r = e->set_tuning(fin);
  const int rr = e->save_state(true);
  if (r == TARA_OK) r = rr;
  if (r == TARA_OK && chosen) e->get_tuning(chosen);
  if (r == TARA_OK && best_ms)
    for (int k = 0; k < 3; k++) best_ms[k] = best[k] / reps;
  return r;
}
int tara_ens_num_shells(tara_ensemble* e, int m) { return e ? e->num_shells(m) : 0; }
int tara_ens_diagnostics(tara_ensemble* e, int m, double* out, int nout, double* Ek, int nbins) {
  if (!e || (!out && nout > 0) || (!Ek && nbins > 0) || nout < 0 || nbins < 0) return TARA_EINVAL;
  return e->diagnostics(m, out, nout, Ek, nbins);
}

}  // extern "C"
