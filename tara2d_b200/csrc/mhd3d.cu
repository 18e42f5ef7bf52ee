// 3D compressible MHD on the device, FP64: the RHS of src/derive3com.f95:5-1047
// and the AB2 step of src/ab3com.f95:6-66.
//
// Layout: spectral fields [Nz][Ny][Nh] Cx<double>, unpadded (the reference's
// Fortran (Nh,Ny,Nz) complex(8) arrays, so host buffers copy as they are);
// real fields [Nz][Ny][Nx] double.
//
// 3D c2r (FFTW's rank-3 c2r): complex inverse DFT along z of every (kx, ky)
// line, along y of every (kx, z) line, then the real inverse along x of every
// row (the imaginary parts of the kx = 0 and kx = Nx/2 bins ignored).  3D r2c
// is the reverse.  The z and y passes are one kernel (k_lines3): CB adjacent
// lines per CTA, so every global load and store of a tile moves CB * 16
// contiguous bytes; the x pass is one thread group per row.  Both run the
// Stockham engine of fft_core.cuh.
//
// One RHS (derive3com):
//   state c2r       8 fields, normalised by Nx Ny Nz             (:78-135, :160-177)
//   k3_velocity     u = (rho u)/rho                                  (:179-182)
//   velocity r2c    3 fields                                         (:198-215)
//   derivative c2r  9 fields; i kx / i ky / i kz applied as the z pass loads
//                   its lines                                       (:244-340)
//   k_rows3_flux    per row: the reference's 19 flux arrays, of which 15
//                   differ (as written, Mom_y_1 = Mom_x_2, Mag_y_1 = Mag_x_1,
//                   Mag_z_1 = Mag_x_2, Mag_z_2 = Mag_y_2)   (:347-414),
//                   and their r2c along x, in shared memory        (:416-500)
//   flux y, z       forward passes of the 15 flux fields
//   k3_assemble     i k multiplies, the k^2 terms, the spherical 2/3 mask and
//                   the sums (:502-1043); while stepping, also ab3com's update
//                   and the history shift of src/main3com.f95:572-600.
// The forcing arrays of :184-188 and their transforms (:217-230) do not enter
// the result (the forcing terms are commented out at :1028-1033) and are not
// formed.
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>
#include "plan.h"
#include "kernels.cuh"

using namespace tara;

namespace tara {
void set_legacy_status(int s);
}

namespace {

constexpr int NSTATE = 8, NDER = 9, NFLUX = 15, MAXJOB = 16;
enum : int { M3_NONE = 0, M3_IKX = 1, M3_IKY = 2, M3_IKZ = 3 };

bool len3_ok(int n) { return n == 16 || n == 32 || n == 64 || n == 128 || n == 256 || n == 512; }

#define TARA3_DISPATCH(n, FN, ...)        \
  switch (n) {                            \
    case 16: FN<16>(__VA_ARGS__); break;  \
    case 32: FN<32>(__VA_ARGS__); break;  \
    case 64: FN<64>(__VA_ARGS__); break;  \
    case 128: FN<128>(__VA_ARGS__); break; \
    case 256: FN<256>(__VA_ARGS__); break; \
    case 512: FN<512>(__VA_ARGS__); break; \
    default: break;                       \
  }

// ------------------------------------------------------------ z and y passes
struct Line3Job {
  const Cx<double>* src;
  Cx<double>* dst;  // may equal src (each CTA reads its whole tile before it writes)
};
struct Line3Args {
  Line3Job job[MAXJOB];
  const Cx<double>* tw;  // e^{-2 pi i m/L}, m < L
  const double *kx, *ky, *kz;
  long long es;          // element stride along a line (complex elements)
  long long ps;          // stride between planes
  int ncol;              // lines per plane, adjacent (stride 1)
  int tiles;             // tiles of CB lines per plane
  int Nh;                // z pass: line c is (kx index c % Nh, ky index c / Nh)
  double thr;            // masked z forward pass: the 2/3-rule threshold
  double dkz;            // 2 pi / Lz (first guess of the cut-off)
};

// shared memory of k_lines3: the exchange tile, the kz table, then per line a
// multiplier and a mask cut-off
template <int L, int CB, int P> constexpr size_t lines3_smem() {
  return (size_t)FFTB<L, CB, P>::SMEM_ELEMS * sizeof(Cx<double>) + (L + CB) * sizeof(double) + CB * sizeof(int);
}

// dsqrt(kx*kx + ky*ky + kz*kz) .ge. thr with kxy = kx*kx + ky*ky, each
// product and sum rounded as written                    (src/derive3com.f95:850)
__device__ __forceinline__ bool masked3(double kxy, double kz, double thr) {
  return __dsqrt_rn(__dadd_rn(kxy, __dmul_rn(kz, kz))) >= thr;
}

// blockIdx.x: (plane, tile of CB lines), blockIdx.y: job.  MUL: i kx / i ky /
// i kz applied as the z pass loads (c2r of a derivative); MASK: the forward z
// pass leaves the modes of the 2/3 rule unwritten.
template <int L, int CB, int P, int DIR, int MUL, bool MASK>
__global__ void __launch_bounds__(CB * L / P, TARA_MINB(CB * L / P)) k_lines3(const Line3Args a) {
  using F = FFTB<L, CB, P>;
  extern __shared__ __align__(16) unsigned char smraw[];
  Cx<double>* sm = reinterpret_cast<Cx<double>*>(smraw);
  double* kzs = reinterpret_cast<double*>(sm + F::SMEM_ELEMS);  // kz(i), i < L
  double* kline = kzs + L;                                       // kx or ky of each line
  int* cut = reinterpret_cast<int*>(kline + CB);                 // first masked |kz| index of each line
  const Line3Job jb = a.job[blockIdx.y];
  const int plane = blockIdx.x / a.tiles;
  const int c0 = (blockIdx.x - plane * a.tiles) * CB;
  const size_t base = (size_t)plane * (size_t)a.ps;
  const int tid = threadIdx.x;
  if constexpr (MUL == M3_IKZ) {
    for (int i = tid; i < L; i += CB * L / P) kzs[i] = __ldg(a.kz + i);
    __syncthreads();
  }
  if constexpr (MUL == M3_IKX || MUL == M3_IKY || MASK) {
    if (tid < CB) {
      const int c = c0 + tid;
      double km = 0.0;
      int ct = L;
      if (c < a.ncol) {
        const double kx = __ldg(a.kx + c % a.Nh), ky = __ldg(a.ky + c / a.Nh);
        km = MUL == M3_IKX ? kx : ky;
        if constexpr (MASK) {
          // first m in 0..L/2 with the line's mode at |kz index| m masked (the test
          // is monotone in m, and kz(-m)^2 == kz(m)^2 bit for bit): a guess from
          // the threshold, then exact tests up and down
          const double kxy = __dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky));
          const double rem = a.thr * a.thr - kxy;
          int m = rem > 0.0 ? (int)(sqrt(rem) / a.dkz) : 0;
          m = m < 0 ? 0 : (m > L / 2 + 1 ? L / 2 + 1 : m);
          while (m <= L / 2 && !masked3(kxy, __ldg(a.kz + m), a.thr)) m++;
          while (m > 0 && masked3(kxy, __ldg(a.kz + m - 1), a.thr)) m--;
          ct = m;
        }
      }
      kline[tid] = km;
      cut[tid] = ct;
    }
    __syncthreads();
  }
  Cx<double> v[P];
  fft_run<F, DIR>(sm, tid, v, TwGlobal<double>{a.tw}, [&](int t, int i) -> Cx<double> {
    const int c = c0 + t;
    if (c >= a.ncol) return cx<double>(0, 0);
    const Cx<double> x = ldg(jb.src + base + (size_t)i * (size_t)a.es + c);
    if constexpr (MUL == M3_IKX || MUL == M3_IKY) return ikmul(kline[t], x);
    if constexpr (MUL == M3_IKZ) return ikmul(kzs[i], x);
    return x;
  }, SyncBlock{});
  fft_emit<F>(tid, v, [&](int t, int i, Cx<double> x) {
    const int c = c0 + t;
    if (c >= a.ncol) return;
    if constexpr (MASK) {
      if ((i <= L / 2 ? i : L - i) >= cut[t]) return;  // masked: never read
    }
    st(jb.dst + base + (size_t)i * (size_t)a.es + c, x);
  });
}

template <int L, int DIR, int MUL, bool MASK>
void launch_lines3(const Line3Args& a0, int njobs, int nplanes, cudaStream_t st) {
  constexpr int CB = ColCfg<double, L>::CB, P = ColCfg<double, L>::P;
  Line3Args a = a0;
  a.tiles = (a.ncol + CB - 1) / CB;
  const size_t smem = lines3_smem<L, CB, P>();
  auto kern = k_lines3<L, CB, P, DIR, MUL, MASK>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<dim3((unsigned)(a.tiles * nplanes), (unsigned)njobs), CB * L / P, smem, st>>>(a);
}
template <int L> void lines3_inv(const Line3Args& a, int nj, int np, cudaStream_t st, int mul) {
  switch (mul) {
    case M3_IKX: launch_lines3<L, +1, M3_IKX, false>(a, nj, np, st); break;
    case M3_IKY: launch_lines3<L, +1, M3_IKY, false>(a, nj, np, st); break;
    case M3_IKZ: launch_lines3<L, +1, M3_IKZ, false>(a, nj, np, st); break;
    default: launch_lines3<L, +1, M3_NONE, false>(a, nj, np, st); break;
  }
}
template <int L> void lines3_fwd(const Line3Args& a, int nj, int np, cudaStream_t st, bool masked) {
  if (masked) launch_lines3<L, -1, M3_NONE, true>(a, nj, np, st);
  else launch_lines3<L, -1, M3_NONE, false>(a, nj, np, st);
}

// ------------------------------------------------------------------ x pass
struct Row3Args {
  Tables<double> tb;  // tw_row, tw_real, ld = Nh, nn = Nx Ny Nz
  const Cx<double>* src[MAXJOB];
  Cx<double>* dst[MAXJOB];
  int rb;
};

// c2r along x of half-real rows (pitch Nh) into real rows (Nx/2 pairs),
// normalised by Nx Ny Nz
// five CTAs per SM (at most 96 registers) in both x-pass kernels
template <int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(M / P), 5) k_rows3_c2r(const Row3Args a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, 1> th;
  const auto sync = th.sync();
  const Tables<double>& tb = a.tb;
  Cx<double>* xs = reinterpret_cast<Cx<double>*>(smraw) + (size_t)th.row * RF::SMEM_ELEMS;
  const size_t y = (size_t)blockIdx.x * a.rb + th.row;
  const Cx<double>* h = a.src[blockIdx.y] + y * tb.ld;
  Cx<double>* out = a.dst[blockIdx.y] + y * M;
  Cx<double> v[P];
  row_c2r<RF>(xs, th.lane, v, tb, [&](int k) { return ldg(h + k); }, sync);
  fft_emit<RF>(th.lane, v, [&](int, int n, Cx<double> z) {
    st(out + n, cx<double>(normalise(z.x, tb), normalise(z.y, tb)));
  });
}

// r2c along x of real rows into x-transformed rows (pitch Nh)
template <int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(M / P), 5) k_rows3_r2c(const Row3Args a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, 1> th;
  const auto sync = th.sync();
  const Tables<double>& tb = a.tb;
  Cx<double>* xs = reinterpret_cast<Cx<double>*>(smraw) + (size_t)th.row * RF::SMEM_ELEMS;
  const size_t y = (size_t)blockIdx.x * a.rb + th.row;
  const Cx<double>* in = a.src[blockIdx.y] + y * M;
  Cx<double>* xo = a.dst[blockIdx.y] + y * tb.ld;
  Cx<double> v[P];
  row_r2c_begin<RF>(th.lane, v, tb, [&](int n) { return ldg(in + n); });
  row_r2c_finish<RF>(xs, th.lane, NTR, v, tb, [&](int k, Cx<double> X) { st(xo + k, X); }, sync);
}

template <int Nx>
void launch_rows3(bool inverse, const Row3Args& a0, int nf, int rows, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  Row3Args a = a0;
  const size_t per_row = (size_t)RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<double>);
  a.rb = 1;
  while (a.rb * 2 * NTR <= 128 && rows % (a.rb * 2) == 0 && (a.rb * 2) * per_row <= 96 * 1024) a.rb *= 2;
  const size_t smem = per_row * a.rb;
  const dim3 grid((unsigned)(rows / a.rb), (unsigned)nf);
  if (inverse) {
    auto kern = k_rows3_c2r<M, P>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<grid, NTR * a.rb, smem, st>>>(a);
  } else {
    auto kern = k_rows3_r2c<M, P>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<grid, NTR * a.rb, smem, st>>>(a);
  }
}

// ------------------------------------------------------------ point kernels
struct Vel3Args {
  const double *rho, *mx, *my, *mz;
  double *ux, *uy, *uz;
  size_t n;
};
// ux = rho_ux/rho ...                                         (src/derive3com.f95:179-182)
__global__ void k3_velocity(const Vel3Args a) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < a.n; p += (size_t)gridDim.x * blockDim.x) {
    const double r = a.rho[p];
    a.ux[p] = a.mx[p] / r;
    a.uy[p] = a.my[p] / r;
    a.uz[p] = a.mz[p] / r;
  }
}

// The 15 distinct fluxes of one point from its 8 state and 9 derivative
// values (real space, normalised).  Order: 0 Mom_x_1, 1 Mom_x_2 (= Mom_y_1),
// 2 Mom_x_3, 3 Mom_y_2, 4 Mom_y_3, 5 Mom_z_1, 6 Mom_z_2, 7 Mom_z_3,
// 8 Energy_x, 9 Energy_y, 10 Energy_z, 11 E_Visc, 12 Mag_x_1 (= Mag_y_1),
// 13 Mag_x_2 (= Mag_z_1), 14 Mag_y_2 (= Mag_z_2)
__device__ __forceinline__ void fluxes15(const double* s, const double* d, double cs, double eta, double* f) {
  const double rho = s[0], mx = s[1], my = s[2], mz = s[3], E = s[4], Bx = s[5], By = s[6], Bz = s[7];
  const double ux = mx / rho, uy = my / rho, uz = mz / rho;  // as k3_velocity: the same values
  const double B2 = Bx * Bx + By * By + Bz * Bz;
  // curl as the reference defines it                                 (:370-373)
  const double cx_ = d[8] - d[6], cy_ = d[7] - d[4], cz_ = d[5] - d[3];
  const double P = cs * cs * rho;                                    // (:375)
  const double hB2 = B2 / 2.0;
  f[0] = mx * ux + P + hB2 - Bx * Bx;                                // (:380-388)
  f[1] = mx * uy - Bx * By;
  f[2] = mx * uz - Bx * Bz;
  f[3] = my * uy + P + hB2 - By * By;
  f[4] = my * uz - By * Bz;
  f[5] = mz * ux - Bz * Bx;
  f[6] = mz * uy - Bz * By;
  f[7] = mz * uz + P + hB2 - Bz * Bz;
  const double H = E + P + hB2;                                      // (:391-399)
  f[8] = H * ux - ux * Bx * Bx - uy * Bx * By - uz * Bx * Bz - eta * (By * cz_ + Bz * cy_);
  f[9] = H * uy - ux * Bx * By - uy * By * By - uz * By * Bz + eta * (Bx * cz_ - Bz * cx_);
  f[10] = H * uz - ux * Bz * Bx - uy * Bz * By - uz * Bz * Bz + eta * (Bx * cy_ + By * cx_);
  const double dv = d[0] + d[1] + d[2];                              // (:402)
  f[11] = dv * dv;
  f[12] = ux * By - uy * Bx;                                         // (:405-410)
  f[13] = ux * Bz - uz * Bx;
  f[14] = uy * Bz - uz * By;
}

// Fluxes and their r2c along x in one row kernel: per row, every thread of
// the row forms the 15 fluxes of its point pairs (x[2n], x[2n+1]) into 15
// shared-memory rows, then 15 thread groups run one r2c each, using their own
// row as exchange buffer.  The real flux fields never reach HBM.
struct FluxRowArgs {
  Tables<double> tb;
  const double* s[NSTATE];  // rho, rho ux, rho uy, rho uz, E, Bx, By, Bz (real, normalised)
  const double* d[NDER];    // dux/dx duy/dy duz/dz dBx/dy dBx/dz dBy/dx dBy/dz dBz/dx dBz/dy
  Cx<double>* x[NFLUX];     // x-transformed flux rows (pitch Nh)
  double cs, eta;
  int rb;
};
// Five CTAs per SM where a CTA has at most 128 threads (92 registers, no
// spills; 20 instead of 15 warps per SM at Nx = 256)
template <int M, int P>
__global__ void __launch_bounds__(TARA_ROW_LB(NFLUX * (M / P)), (NFLUX * (M / P) <= 128 ? 5 : 1))
    k_rows3_flux(const FluxRowArgs a) {
  using RF = RowFFT<M, P>;
  constexpr int NTR = M / P, G = NFLUX, ARR = RF::SMEM_ELEMS;
  extern __shared__ __align__(16) unsigned char smraw[];
  const RowThread<NTR, G> th;
  const auto sync = th.sync();
  const Tables<double>& tb = a.tb;
  Cx<double>* base = reinterpret_cast<Cx<double>*>(smraw) + (size_t)th.row * G * ARR;
  const size_t y = (size_t)blockIdx.x * a.rb + th.row;
  const size_t ro = y * (size_t)(2 * M);
  // phase 1: fluxes of the point pairs n (x = 2n, 2n+1)                (:343-414)
  // one point at a time (x = 2n + h into component h of the pair), which keeps
  // few values live
  double* basd = reinterpret_cast<double*>(base);
  for (int e = th.g * NTR + th.lane; e < 2 * M; e += G * NTR) {
    double sv[NSTATE], dv[NDER], f[NFLUX];
#pragma unroll
    for (int q = 0; q < NSTATE; q++) sv[q] = __ldg(a.s[q] + ro + e);
#pragma unroll
    for (int q = 0; q < NDER; q++) dv[q] = __ldg(a.d[q] + ro + e);
    fluxes15(sv, dv, a.cs, a.eta, f);
#pragma unroll
    for (int q = 0; q < NFLUX; q++) basd[2 * q * ARR + e] = f[q];
  }
  __syncthreads();
  // phase 2: r2c along x of flux g, exchanges in its own row (every value of
  // the row is in registers before the first exchange store)     (:416-500)
  Cx<double>* arr = base + th.g * ARR;
  Cx<double> v[P];
  row_r2c_begin<RF>(th.lane, v, tb, [&](int n) { return arr[n]; });
  Cx<double>* xo = a.x[th.g] + y * tb.ld;
  row_r2c_finish<RF>(arr, th.lane, NTR, v, tb, [&](int k, Cx<double> X) { st(xo + k, X); }, sync);
}

template <int Nx>
void launch_rows3_flux(const FluxRowArgs& a0, int rows, cudaStream_t st) {
  constexpr int M = Nx / 2;
  constexpr int P = RowCfg<M>::P;
  constexpr int NTR = M / P;
  FluxRowArgs a = a0;
  const size_t per_row = (size_t)NFLUX * RowFFT<M, P>::SMEM_ELEMS * sizeof(Cx<double>);
  a.rb = 1;
  // rows per CTA within the kernel's launch bound
  while ((a.rb * 2) * NFLUX * NTR <= TARA_ROW_LB(NFLUX * NTR) && rows % (a.rb * 2) == 0 &&
         (a.rb * 2) * per_row <= 100 * 1024)
    a.rb *= 2;
  const size_t smem = per_row * a.rb;
  auto kern = k_rows3_flux<M, P>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<(unsigned)(rows / a.rb), NFLUX * NTR * a.rb, smem, st>>>(a);
}

struct Asm3Args {
  const Cx<double>* f[NFLUX];  // flux spectra
  const Cx<double>* u[3];      // ux_k, uy_k, uz_k
  Cx<double>* s[NSTATE];       // state (read; updated in place while stepping)
  Cx<double>* h[NSTATE];       // history d_old (read, then replaced by d_new) while stepping
  Cx<double>* out[NSTATE];     // d_new (RHS only)
  const double *kx, *ky, *kz;
  double mu, dt, thr;
  int Nh, Ny, Nz, step;
};

__device__ __forceinline__ Cx<double> div450(Cx<double> z) { return cx<double>(z.x / 450.0, z.y / 450.0); }

// u + ((3/2) dn - (1/2) dold) dt, every product and sum rounded as written
// (src/ab3com.f95:47)
__device__ __forceinline__ double ab2_rn(double u, double dn, double dold, double dt) {
  return __dadd_rn(u, __dmul_rn(__dsub_rn(__dmul_rn(1.5, dn), __dmul_rn(0.5, dold)), dt));
}
__device__ __forceinline__ Cx<double> ab2_rn(Cx<double> u, Cx<double> dn, Cx<double> dold, double dt) {
  return cx<double>(ab2_rn(u.x, dn.x, dold.x, dt), ab2_rn(u.y, dn.y, dold.y, dt));
}

// i k multiplies, k^2 terms, mask and sums    (src/derive3com.f95:502-1043);
// with a.step, ab3com (src/ab3com.f95:44-61) and the history shift
__global__ void __launch_bounds__(256, 3) k3_assemble(const Asm3Args a) {
  const size_t n = (size_t)a.Nh * a.Ny * a.Nz;
  for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < n; m += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(m % a.Nh);
    const size_t r = m / a.Nh;
    const int j = (int)(r % a.Ny), k = (int)(r / a.Ny);
    const double kx = __ldg(a.kx + i), ky = __ldg(a.ky + j), kz = __ldg(a.kz + k);
    // dsqrt(kx*kx + ky*ky + kz*kz) .ge. (dfloat(Nx+Ny+Nz)/3.0)/3.0, each
    // product and sum rounded as written                                  (:850)
    const double k2s = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    const bool masked = __dsqrt_rn(k2s) >= a.thr;
    Cx<double> d[NSTATE];
    if (masked) {
#pragma unroll
      for (int q = 0; q < NSTATE; q++) d[q] = cx<double>(0, 0);
    } else {
      const double kx2 = kx * kx, ky2 = ky * ky, kz2 = kz * kz;
      auto visc = [&](Cx<double> z) { return div450(rmul(kx2, z) + rmul(ky2, z) + rmul(kz2, z)); };
      auto F = [&](int q) { return ldg(a.f[q] + m); };
      const Cx<double> rux = ldg(a.s[1] + m), ruy = ldg(a.s[2] + m), ruz = ldg(a.s[3] + m);
      d[0] = -(ikmul(kx, rux) + ikmul(ky, ruy) + ikmul(kz, ruz));                       // (:1024)
      d[1] = -(ikmul(kx, F(0)) + ikmul(ky, F(1)) + ikmul(kz, F(2))) - visc(ldg(a.u[0] + m));
      d[2] = -(ikmul(kx, F(1)) + ikmul(ky, F(3)) + ikmul(kz, F(4))) - visc(ldg(a.u[1] + m));
      d[3] = -(ikmul(kx, F(5)) + ikmul(ky, F(6)) + ikmul(kz, F(7))) - visc(ldg(a.u[2] + m));
      d[4] = -(ikmul(kx, F(8)) + ikmul(ky, F(9)) + ikmul(kz, F(10))) + rmul(a.mu, F(11)); // (:1035-1036)
      d[5] = (ikmul(ky, F(12)) + ikmul(kz, F(13))) - visc(ldg(a.s[5] + m));              // (:1038-1043)
      d[6] = -(ikmul(kx, F(12)) - ikmul(kz, F(14))) - visc(ldg(a.s[6] + m));
      d[7] = -(ikmul(kx, F(13)) + ikmul(ky, F(14))) - visc(ldg(a.s[7] + m));
    }
    if (!a.step) {
#pragma unroll
      for (int q = 0; q < NSTATE; q++) st(a.out[q] + m, d[q]);
      continue;
    }
    // u_new = u + ((3/2) d_new - (1/2) d_old) dt; E unchanged; d_old = d_new
#pragma unroll
    for (int q = 0; q < NSTATE; q++) {
      const Cx<double> old = ld(a.h[q] + m);
      if (q != 4) {
        const Cx<double> u = ld(a.s[q] + m);
        st(a.s[q] + m, ab2_rn(u, d[q], old, a.dt));
      }
      st(a.h[q] + m, d[q]);
    }
  }
}

// ab3com alone (the drop-in entry point): out = u + ((3/2) dn - (1/2) dold) dt, E copied
struct Ab3Args {
  const Cx<double>* u[NSTATE];
  const Cx<double>* dn[NSTATE];
  const Cx<double>* dold[NSTATE];
  Cx<double>* out[NSTATE];
  double dt;
  size_t n;
};
__global__ void k3_ab2(const Ab3Args a) {
  for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < a.n; m += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < NSTATE; q++) {
      const Cx<double> u = ldg(a.u[q] + m);
      st(a.out[q] + m, q == 4 ? u : ab2_rn(u, ldg(a.dn[q] + m), ldg(a.dold[q] + m), a.dt));
    }
  }
}

}  // namespace

// ======================================================================
// session
// ======================================================================
struct tara3d {
  int Nx = 0, Ny = 0, Nz = 0, Nh = 0;
  size_t ns = 0, nr = 0;  // spectral / real elements per field
  tara3d_params p{};
  cudaStream_t st = nullptr;
  void* tables = nullptr;
  Tables<double> tb{};
  const Cx<double>* twy = nullptr;
  const Cx<double>* twz = nullptr;
  const double *kx = nullptr, *ky = nullptr, *kz = nullptr;
  Cx<double>* spec = nullptr;  // one block: state, history, d_new, flux spectra, velocity spectra
  double* real = nullptr;      // one block: state, velocity and derivative fields
  Cx<double>* S[NSTATE]{};
  Cx<double>* H[NSTATE]{};
  Cx<double>* D[NSTATE]{};
  Cx<double>* T[NFLUX]{};
  Cx<double>* U[3]{};
  double* R[NSTATE]{};
  double* V[3]{};
  double* G[NDER]{};
  int grid_pts = 0;
  cudaGraphExec_t graph = nullptr;

  // 3D c2r of nf fields (src -> real), through the spectral scratch T; mul[q]
  // multiplies field q as the z pass loads it (one z launch per multiplier)
  int c2r(int nf, const Cx<double>* const* src, const int* mul, double* const* dst) {
    for (int m = M3_NONE; m <= M3_IKZ; m++) {
      Line3Args z{};
      int nj = 0;
      for (int q = 0; q < nf; q++)
        if ((mul ? mul[q] : M3_NONE) == m) z.job[nj++] = Line3Job{src[q], T[q]};
      if (nj == 0) continue;
      z.tw = twz; z.kx = kx; z.ky = ky; z.kz = kz;
      z.es = (long long)Ny * Nh; z.ps = 0; z.ncol = Ny * Nh; z.Nh = Nh;
      TARA3_DISPATCH(Nz, lines3_inv, z, nj, 1, st, m)
    }
    Line3Args y{};
    for (int q = 0; q < nf; q++) y.job[q] = Line3Job{T[q], T[q]};
    y.tw = twy; y.es = Nh; y.ps = (long long)Ny * Nh; y.ncol = Nh; y.Nh = Nh;
    TARA3_DISPATCH(Ny, lines3_inv, y, nf, Nz, st, M3_NONE)
    Row3Args x{};
    x.tb = tb;
    for (int q = 0; q < nf; q++) { x.src[q] = T[q]; x.dst[q] = reinterpret_cast<Cx<double>*>(dst[q]); }
    TARA3_DISPATCH(Nx, launch_rows3, true, x, nf, Ny * Nz, st)
    return TARA_OK;
  }
  // 3D r2c of nf real fields into dst (x pass writes dst, y and z in place);
  // masked: the z pass leaves the modes of the 2/3 rule unwritten
  int r2c(int nf, const double* const* src, Cx<double>* const* dst, bool masked) {
    Row3Args x{};
    x.tb = tb;
    for (int q = 0; q < nf; q++) { x.src[q] = reinterpret_cast<const Cx<double>*>(src[q]); x.dst[q] = dst[q]; }
    TARA3_DISPATCH(Nx, launch_rows3, false, x, nf, Ny * Nz, st)
    return fwd_yz(nf, dst, masked);
  }
  // forward y and z passes in place of nf x-transformed fields
  int fwd_yz(int nf, Cx<double>* const* dst, bool masked) {
    Line3Args y{};
    for (int q = 0; q < nf; q++) y.job[q] = Line3Job{dst[q], dst[q]};
    y.tw = twy; y.es = Nh; y.ps = (long long)Ny * Nh; y.ncol = Nh; y.Nh = Nh;
    TARA3_DISPATCH(Ny, lines3_fwd, y, nf, Nz, st, false)
    Line3Args z{};
    for (int q = 0; q < nf; q++) z.job[q] = Line3Job{dst[q], dst[q]};
    z.tw = twz; z.kx = kx; z.ky = ky; z.kz = kz;
    z.es = (long long)Ny * Nh; z.ps = 0; z.ncol = Ny * Nh; z.Nh = Nh;
    z.thr = mask_thr();
    z.dkz = 2.0 * p.pi / p.Lz;
    TARA3_DISPATCH(Nz, lines3_fwd, z, nf, 1, st, masked)
    return TARA_OK;
  }

  // One RHS; step = 0: d_new into D, step = 1: AB2 update of S and H.
  int rhs(int step) {
    const Cx<double>* s8[NSTATE];
    for (int q = 0; q < NSTATE; q++) s8[q] = S[q];
    TARA_TRY(c2r(NSTATE, s8, nullptr, R));
    Vel3Args va{R[0], R[1], R[2], R[3], V[0], V[1], V[2], nr};
    k3_velocity<<<grid_pts, 256, 0, st>>>(va);
    const double* v3[3] = {V[0], V[1], V[2]};
    TARA_TRY(r2c(3, v3, U, false));  // every mode: the derivatives below use them all
    // i kx ux, i ky uy, i kz uz, i ky Bx, i kz Bx, i kx By, i kz By, i kx Bz, i ky Bz   (:232-340)
    const Cx<double>* dsrc[NDER] = {U[0], U[1], U[2], S[5], S[5], S[6], S[6], S[7], S[7]};
    const int dmul[NDER] = {M3_IKX, M3_IKY, M3_IKZ, M3_IKY, M3_IKZ, M3_IKX, M3_IKZ, M3_IKX, M3_IKY};
    TARA_TRY(c2r(NDER, dsrc, dmul, G));
    FluxRowArgs fa{};
    fa.tb = tb;
    for (int q = 0; q < NSTATE; q++) fa.s[q] = R[q];
    for (int q = 0; q < NDER; q++) fa.d[q] = G[q];
    for (int q = 0; q < NFLUX; q++) fa.x[q] = T[q];
    fa.cs = p.CS; fa.eta = p.eta;
    TARA3_DISPATCH(Nx, launch_rows3_flux, fa, Ny * Nz, st)
    TARA_TRY(fwd_yz(NFLUX, T, true));  // k3_assemble reads unmasked modes only
    Asm3Args aa{};
    for (int q = 0; q < NFLUX; q++) aa.f[q] = T[q];
    for (int q = 0; q < 3; q++) aa.u[q] = U[q];
    for (int q = 0; q < NSTATE; q++) { aa.s[q] = S[q]; aa.h[q] = H[q]; aa.out[q] = D[q]; }
    aa.kx = kx; aa.ky = ky; aa.kz = kz;
    aa.mu = p.mu; aa.dt = p.dt;
    aa.thr = mask_thr();
    aa.Nh = Nh; aa.Ny = Ny; aa.Nz = Nz; aa.step = step;
    k3_assemble<<<grid_pts, 256, 0, st>>>(aa);
    TARA_CUDA_TRY(cudaGetLastError());
    return TARA_OK;
  }

  // (dfloat(Nx+Ny+Nz)/3.0)/3.0 + 0                                  (src/derive3com.f95:850)
  double mask_thr() const { return ((double)(Nx + Ny + Nz) / 3.0) / 3.0 + 0; }

  int launches_per_step() const { return 3 + 1 + 3 + 5 + 1 + 2 + 1; }

  int steps(int n) {
    if (n <= 0) return TARA_OK;
    if (!graph) {
      // eager first step (sets kernel attributes), then capture one step
      TARA_TRY(rhs(1));
      n--;
      cudaGraph_t g = nullptr;
      TARA_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const int r = rhs(1);
      const cudaError_t e = cudaStreamEndCapture(st, &g);
      if (r != TARA_OK) { if (g) cudaGraphDestroy(g); return r; }
      TARA_CUDA_TRY(e);
      const cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
      cudaGraphDestroy(g);
      TARA_CUDA_TRY(ie);
    }
    for (int k = 0; k < n; k++) TARA_CUDA_TRY(cudaGraphLaunch(graph, st));
    TARA_CUDA_TRY(cudaGetLastError());
    return TARA_OK;
  }

  int init(int nx, int ny, int nz, const tara3d_params& prm) {
    if (!len3_ok(nx) || !len3_ok(ny) || !len3_ok(nz)) {
      set_error("3D grid sizes must be 16, 32, 64, 128, 256 or 512");
      return TARA_EUNSUPPORTED;
    }
    Nx = nx; Ny = ny; Nz = nz; Nh = nx / 2 + 1;
    ns = (size_t)Nh * Ny * Nz;
    nr = (size_t)Nx * Ny * Nz;
    p = prm;
    TARA_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int dev = 0, sms = 148;
    TARA_CUDA_TRY(cudaGetDevice(&dev));
    TARA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    grid_pts = sms * 8;
    TARA_TRY(make_tables(sms));
    // spectral: S, H, D (8 each), T (15), U (3); real: R (8), V (3), G (9)
    const size_t nspec = 3 * NSTATE + NFLUX + 3, nreal = NSTATE + 3 + NDER;
    if (cudaMalloc(&spec, nspec * ns * sizeof(Cx<double>)) != cudaSuccess) {
      spec = nullptr;
      set_error("cudaMalloc of the 3D spectral fields failed");
      return TARA_ENOMEM;
    }
    if (cudaMalloc(&real, nreal * nr * sizeof(double)) != cudaSuccess) {
      real = nullptr;
      set_error("cudaMalloc of the 3D real fields failed");
      return TARA_ENOMEM;
    }
    Cx<double>* c = spec;
    for (int q = 0; q < NSTATE; q++, c += ns) S[q] = c;
    for (int q = 0; q < NSTATE; q++, c += ns) H[q] = c;
    for (int q = 0; q < NSTATE; q++, c += ns) D[q] = c;
    for (int q = 0; q < NFLUX; q++, c += ns) T[q] = c;
    for (int q = 0; q < 3; q++, c += ns) U[q] = c;
    double* r = real;
    for (int q = 0; q < NSTATE; q++, r += nr) R[q] = r;
    for (int q = 0; q < 3; q++, r += nr) V[q] = r;
    for (int q = 0; q < NDER; q++, r += nr) G[q] = r;
    TARA_CUDA_TRY(cudaMemsetAsync(spec, 0, nspec * ns * sizeof(Cx<double>), st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }

  int make_tables(int sms) {
    const int M = Nx / 2;
    auto tw = [](int L, int count, std::vector<Cx<double>>& out) {
      out.resize(count);
      for (int m = 0; m < count; m++) {
        long double c, s;
        twiddle(m, L, c, s);
        out[m] = cx<double>((double)c, (double)s);
      }
    };
    std::vector<Cx<double>> ty, tz, tr, tre;
    tw(Ny, Ny, ty);
    tw(Nz, Nz, tz);
    tw(M, M, tr);
    tw(Nx, M + 1, tre);
    // kx = 2.0d0*pi*dfloat(i-1)/Lx; ky, kz negative above N/2   (src/derive3com.f95:237-246)
    std::vector<double> vkx(Nh), vky(Ny), vkz(Nz);
    for (int i = 0; i < Nh; i++) vkx[i] = 2.0 * p.pi * (double)i / p.Lx;
    for (int j = 0; j < Ny; j++) vky[j] = 2.0 * p.pi * (double)(j < Ny / 2 ? j : j - Ny) / p.Ly;
    for (int k = 0; k < Nz; k++) vkz[k] = 2.0 * p.pi * (double)(k < Nz / 2 ? k : k - Nz) / p.Lz;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t o_ty = 0, o_tz = o_ty + al(ty.size() * 16), o_tr = o_tz + al(tz.size() * 16),
                 o_tre = o_tr + al(tr.size() * 16), o_kx = o_tre + al(tre.size() * 16),
                 o_ky = o_kx + al(vkx.size() * 8), o_kz = o_ky + al(vky.size() * 8),
                 o_status = o_kz + al(vkz.size() * 8), total = o_status + 256;
    std::vector<char> h(total, 0);
    std::memcpy(h.data() + o_ty, ty.data(), ty.size() * 16);
    std::memcpy(h.data() + o_tz, tz.data(), tz.size() * 16);
    std::memcpy(h.data() + o_tr, tr.data(), tr.size() * 16);
    std::memcpy(h.data() + o_tre, tre.data(), tre.size() * 16);
    std::memcpy(h.data() + o_kx, vkx.data(), vkx.size() * 8);
    std::memcpy(h.data() + o_ky, vky.data(), vky.size() * 8);
    std::memcpy(h.data() + o_kz, vkz.data(), vkz.size() * 8);
    if (cudaMalloc(&tables, total) != cudaSuccess) {
      tables = nullptr;
      set_error("cudaMalloc of the 3D tables failed");
      return TARA_ENOMEM;
    }
    // on the session's (non-blocking) stream and waited for: a plain copy from
    // pageable memory may return before the data reaches the device and is
    // not ordered with that stream's kernels
    TARA_CUDA_TRY(cudaMemcpyAsync(tables, h.data(), total, cudaMemcpyHostToDevice, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    char* b = (char*)tables;
    twy = (const Cx<double>*)(b + o_ty);
    twz = (const Cx<double>*)(b + o_tz);
    kx = (const double*)(b + o_kx);
    ky = (const double*)(b + o_ky);
    kz = (const double*)(b + o_kz);
    tb = Tables<double>{};
    tb.tw_col = twy;
    tb.tw_row = (const Cx<double>*)(b + o_tr);
    tb.tw_real = (const Cx<double>*)(b + o_tre);
    tb.kx = kx;
    tb.ky = ky;
    tb.cut = nullptr;
    tb.Nx = Nx; tb.Ny = Ny * Nz; tb.Nh = Nh; tb.ld = Nh;
    const double nn = (double)Nx * (double)Ny * (double)Nz;  // dfloat(Nx)*dfloat(Ny)*dfloat(Nz)
    tb.nn = nn;
    tb.inv_nn = 1.0 / nn;
    tb.nn_pow2 = 1;  // every supported size is a power of two
    tb.status = (int*)(b + o_status);
    tb.sm_count = sms;
    tb.no_tma = 0;
    tb.wait_ns = 1000000000ull;
    return TARA_OK;
  }

  void release() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    if (st) cudaStreamSynchronize(st);
    if (spec) cudaFree(spec);
    if (real) cudaFree(real);
    if (tables) cudaFree(tables);
    if (st) cudaStreamDestroy(st);
    spec = nullptr; real = nullptr; tables = nullptr; st = nullptr;
  }

  int upload(Cx<double>* const* dst, const double* const* src) {
    for (int q = 0; q < NSTATE; q++) {
      if (!src[q]) { set_error("null field pointer"); return TARA_EINVAL; }
      TARA_CUDA_TRY(cudaMemcpyAsync(dst[q], src[q], ns * sizeof(Cx<double>), cudaMemcpyHostToDevice, st));
    }
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }
  int download(double* const* dst, Cx<double>* const* src) {
    for (int q = 0; q < NSTATE; q++) {
      if (!dst[q]) { set_error("null field pointer"); return TARA_EINVAL; }
      TARA_CUDA_TRY(cudaMemcpyAsync(dst[q], src[q], ns * sizeof(Cx<double>), cudaMemcpyDeviceToHost, st));
    }
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }
};

namespace {

bool params_ok(const tara3d_params* p) {
  if (!p) { set_error("null parameters"); return false; }
  if (!(p->Lx > 0 && p->Ly > 0 && p->Lz > 0)) { set_error("box lengths must be positive"); return false; }
  return true;
}

std::mutex g3_mu;
std::unique_ptr<tara3d> g3_legacy;  // cached session of the drop-in entry points

tara3d_params params_from_comm(double pi) {
  // COMMON /comm/ iret,thread_num,time_max,Lx,Ly,Lz,dx,dy,dz,spheat,mu,ms,CS,
  //               mu_0,eta,dt,kf                               (src/main3com.f95:56)
  tara3d_params p{};
  p.pi = pi;
  p.Lx = comm_[2]; p.Ly = comm_[3]; p.Lz = comm_[4];
  p.mu = comm_[9]; p.CS = comm_[11]; p.eta = comm_[13]; p.dt = comm_[14];
  return p;
}

// Caller holds g3_mu.
tara3d* legacy3(int Nx, int Ny, int Nz, int Nh, const tara3d_params& p, int& status) {
  if (Nh != Nx / 2 + 1) { set_error("inconsistent Nx/Nh"); status = TARA_EINVAL; return nullptr; }
  tara3d* s = g3_legacy.get();
  const bool same = s && s->Nx == Nx && s->Ny == Ny && s->Nz == Nz && s->p.pi == p.pi && s->p.Lx == p.Lx &&
                    s->p.Ly == p.Ly && s->p.Lz == p.Lz;
  if (!same) {
    if (s) s->release();
    g3_legacy.reset(new tara3d());
    s = g3_legacy.get();
    status = s->init(Nx, Ny, Nz, p);
    if (status != TARA_OK) { s->release(); g3_legacy.reset(); return nullptr; }
  }
  s->p = p;
  if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }  // parameters are baked into a graph
  status = TARA_OK;
  return s;
}

}  // namespace

// ======================================================================
// C ABI
// ======================================================================
extern "C" {

int tara3d_open(tara3d** out, int Nx, int Ny, int Nz, const tara3d_params* p) {
  if (!out || !params_ok(p)) { if (!out) set_error("null argument"); return TARA_EINVAL; }
  *out = nullptr;
  auto s = std::make_unique<tara3d>();
  const int r = s->init(Nx, Ny, Nz, *p);
  if (r != TARA_OK) { s->release(); return r; }
  *out = s.release();
  return TARA_OK;
}

int tara3d_close(tara3d* s) {
  if (!s) return TARA_EINVAL;
  s->release();
  delete s;
  return TARA_OK;
}

int tara3d_set_params(tara3d* s, const tara3d_params* p) {
  if (!s || !params_ok(p)) return TARA_EINVAL;
  if (p->pi != s->p.pi || p->Lx != s->p.Lx || p->Ly != s->p.Ly || p->Lz != s->p.Lz) {
    set_error("pi and the box lengths are fixed when the session opens");
    return TARA_EINVAL;
  }
  s->p = *p;
  if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
  return TARA_OK;
}

int tara3d_set_state(tara3d* s, const double* const fields[8]) {
  if (!s || !fields) { set_error("null argument"); return TARA_EINVAL; }
  return s->upload(s->S, fields);
}
int tara3d_get_state(tara3d* s, double* const fields[8]) {
  if (!s || !fields) { set_error("null argument"); return TARA_EINVAL; }
  return s->download(fields, s->S);
}
int tara3d_set_history(tara3d* s, const double* const d_old[8]) {
  if (!s || !d_old) { set_error("null argument"); return TARA_EINVAL; }
  return s->upload(s->H, d_old);
}
int tara3d_rhs(tara3d* s, double* const d_new[8]) {
  if (!s || !d_new) { set_error("null argument"); return TARA_EINVAL; }
  TARA_TRY(s->rhs(0));
  return s->download(d_new, s->D);
}
int tara3d_step(tara3d* s, int nsteps) {
  if (!s || nsteps < 0) { set_error("bad argument"); return TARA_EINVAL; }
  TARA_TRY(s->steps(nsteps));
  TARA_CUDA_TRY(cudaStreamSynchronize(s->st));
  return TARA_OK;
}
int tara3d_time_steps(tara3d* s, int nsteps, float* ms) {
  if (!s || nsteps < 1 || !ms) { set_error("bad argument"); return TARA_EINVAL; }
  TARA_TRY(s->steps(1));  // builds the graph outside the timed region
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // the events are released on every path
  auto timed = [&]() -> int {
    TARA_CUDA_TRY(cudaEventCreate(&e0));
    TARA_CUDA_TRY(cudaEventCreate(&e1));
    TARA_CUDA_TRY(cudaStreamSynchronize(s->st));
    TARA_CUDA_TRY(cudaEventRecord(e0, s->st));
    const int r = s->steps(nsteps);
    TARA_CUDA_TRY(cudaEventRecord(e1, s->st));
    TARA_CUDA_TRY(cudaEventSynchronize(e1));
    TARA_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
    return r;
  };
  const int r = timed();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return r;
}
int tara3d_launches_per_step(tara3d* s) { return s ? s->launches_per_step() : 0; }

void derive3com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nz, const int32_t* Nh,
                 const double* pi, const double* time, double* rho_k, double* rho_ux_k,
                 double* rho_uy_k, double* rho_uz_k, double* E_k, double* Bx_k, double* By_k,
                 double* Bz_k, double* d_rho_k_dt_old, double* d_rho_k_dt_new,
                 double* d_rho_ux_k_dt_old, double* d_rho_ux_k_dt_new, double* d_rho_uy_k_dt_old,
                 double* d_rho_uy_k_dt_new, double* d_rho_uz_k_dt_old, double* d_rho_uz_k_dt_new,
                 double* d_E_k_dt_old, double* d_E_k_dt_new, double* d_Bx_k_dt_old,
                 double* d_Bx_k_dt_new, double* d_By_k_dt_old, double* d_By_k_dt_new,
                 double* d_Bz_k_dt_old, double* d_Bz_k_dt_new) {
  (void)time; (void)d_rho_k_dt_old; (void)d_rho_ux_k_dt_old; (void)d_rho_uy_k_dt_old;
  (void)d_rho_uz_k_dt_old; (void)d_E_k_dt_old; (void)d_Bx_k_dt_old; (void)d_By_k_dt_old;
  (void)d_Bz_k_dt_old;
  if (!Nx || !Ny || !Nz || !Nh || !pi) { set_error("null argument"); set_legacy_status(TARA_EINVAL); return; }
  std::lock_guard<std::mutex> lk(g3_mu);
  int st = TARA_OK;
  tara3d* s = legacy3(*Nx, *Ny, *Nz, *Nh, params_from_comm(*pi), st);
  if (s) {
    const double* in[8] = {rho_k, rho_ux_k, rho_uy_k, rho_uz_k, E_k, Bx_k, By_k, Bz_k};
    double* out[8] = {d_rho_k_dt_new, d_rho_ux_k_dt_new, d_rho_uy_k_dt_new, d_rho_uz_k_dt_new,
                      d_E_k_dt_new, d_Bx_k_dt_new, d_By_k_dt_new, d_Bz_k_dt_new};
    st = s->upload(s->S, in);
    if (st == TARA_OK) st = s->rhs(0);
    if (st == TARA_OK) st = s->download(out, s->D);
  }
  set_legacy_status(st);
}

void ab3com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nz, const int32_t* Nh,
             const double* pi, const double* time, double* rho_k, double* rho_ux_k, double* rho_uy_k,
             double* rho_uz_k, double* E_k, double* Bx_k, double* By_k, double* Bz_k,
             double* rho_k_new, double* rho_ux_k_new, double* rho_uy_k_new, double* rho_uz_k_new,
             double* E_k_new, double* Bx_k_new, double* By_k_new, double* Bz_k_new,
             double* d_rho_k_dt_old, double* d_rho_k_dt_new, double* d_rho_ux_k_dt_old,
             double* d_rho_ux_k_dt_new, double* d_rho_uy_k_dt_old, double* d_rho_uy_k_dt_new,
             double* d_rho_uz_k_dt_old, double* d_rho_uz_k_dt_new, double* d_E_k_dt_old,
             double* d_E_k_dt_new, double* d_Bx_k_dt_old, double* d_Bx_k_dt_new,
             double* d_By_k_dt_old, double* d_By_k_dt_new, double* d_Bz_k_dt_old,
             double* d_Bz_k_dt_new) {
  (void)time;
  if (!Nx || !Ny || !Nz || !Nh || !pi) { set_error("null argument"); set_legacy_status(TARA_EINVAL); return; }
  std::lock_guard<std::mutex> lk(g3_mu);
  int st = TARA_OK;
  tara3d* s = legacy3(*Nx, *Ny, *Nz, *Nh, params_from_comm(*pi), st);
  if (s) {
    const double* u[8] = {rho_k, rho_ux_k, rho_uy_k, rho_uz_k, E_k, Bx_k, By_k, Bz_k};
    const double* dn[8] = {d_rho_k_dt_new, d_rho_ux_k_dt_new, d_rho_uy_k_dt_new, d_rho_uz_k_dt_new,
                           d_E_k_dt_new, d_Bx_k_dt_new, d_By_k_dt_new, d_Bz_k_dt_new};
    const double* dol[8] = {d_rho_k_dt_old, d_rho_ux_k_dt_old, d_rho_uy_k_dt_old, d_rho_uz_k_dt_old,
                            d_E_k_dt_old, d_Bx_k_dt_old, d_By_k_dt_old, d_Bz_k_dt_old};
    double* out[8] = {rho_k_new, rho_ux_k_new, rho_uy_k_new, rho_uz_k_new, E_k_new, Bx_k_new, By_k_new, Bz_k_new};
    st = s->upload(s->S, u);
    if (st == TARA_OK) st = s->upload(s->D, dn);
    if (st == TARA_OK) st = s->upload(s->H, dol);
    if (st == TARA_OK) {
      Ab3Args a{};
      for (int q = 0; q < 8; q++) { a.u[q] = s->S[q]; a.dn[q] = s->D[q]; a.dold[q] = s->H[q]; a.out[q] = s->T[q]; }
      a.dt = s->p.dt;
      a.n = s->ns;
      k3_ab2<<<s->grid_pts, 256, 0, s->st>>>(a);
      st = cudaGetLastError() == cudaSuccess ? TARA_OK : TARA_ECUDA;
      if (st != TARA_OK) set_error("ab3com kernel launch failed");
    }
    if (st == TARA_OK) st = s->download(out, s->T);
  }
  set_legacy_status(st);
}

}  // extern "C"
