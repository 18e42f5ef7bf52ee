// Hydro right-hand side (derive2coh) that allocates nothing.
//
// Why this exists: the regular entry points create a cached grid context and
// allocate their device workspace with cudaMalloc on first use.  Some hosts
// must not do that from the solver -- for example a program that has already
// handed all device memory to its own pool allocator (a raw cudaMalloc would
// fail there, or bypass the pool's accounting), or a time-critical loop in
// which an allocation's latency and implicit device synchronisation are not
// acceptable.  tara_derive2coh_noalloc takes device buffers the caller already
// owns and keeps every temporary (the eight half-real fields, the three
// x-transformed rows and the grid tables) in one statically sized device
// array that the library reserves when it is loaded.
//
// Limits and behaviour:
//   * Nx, Ny in {16, 32, 64, 128, 256}; larger grids are rejected with
//     TARA_EINVAL (the static workspace is sized for 256 x 256, about 6 MB,
//     held on every device that loads the library until the process exits).
//   * FP64 only; inputs and outputs are the reference's complex(8) (Nh,Ny)
//     arrays (no row padding) in device memory.
//   * Every call uses the same workspace.  Two calls whose kernels overlap on
//     the GPU (different streams without ordering) race and give wrong
//     results; calls on one stream are ordered and safe.  Each call writes
//     every workspace element it later reads, so nothing needs clearing.
//   * The grid tables (twiddles, wavenumbers, dealiasing cut-offs) are built
//     on the host into one fixed-size static structure, rebuilt only when
//     (Nx, Ny, Lx, Ly, pi) change, and reach the workspace as the by-value
//     parameter of a small copy kernel (no host-to-device memcpy).  A mutex
//     serialises that host-side preparation, so calls from several host
//     threads do not corrupt each other's tables on the host.
//   * The column passes run the register-staged kernels (no TMA tile loads,
//     hence no bounded waits and no device status word to read back): every
//     failure of a call is reported by its return value.
//   * The first call on a device looks up the workspace's device address
//     (cudaGetSymbolAddress) for that device; make that first call before
//     any stream capture begins.
#include <cmath>
#include <cstring>
#include <mutex>
#include "models.h"

namespace {

using tara::Cx;

constexpr int kMaxN = 256;                 // largest Nx and Ny accepted
constexpr int kMaxNh = kMaxN / 2 + 1;
constexpr size_t kField = (size_t)kMaxN * kMaxNh;  // complex elements of one field at the maximum size
constexpr size_t kTableBytes = 64 * 1024;           // twiddles, wavenumbers and cut-offs
constexpr size_t kScratchBytes = 11 * kField * sizeof(Cx<double>) + kTableBytes;

// The whole workspace: 11 fields of kField complex values, then the tables.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
static void* g_scratch_addr[kMaxDevices] = {nullptr};

// Grid tables of one call, built on the host.  Fixed size, so that building
// them allocates nothing; passed by value to k_noalloc_tables (about 12 KB of
// kernel parameters).
struct NoallocTables {
  Cx<double> tw_col[kMaxN];
  Cx<double> tw_row[kMaxN / 2];
  Cx<double> tw_real[kMaxN / 2 + 1];
  double kx[kMaxNh];
  double ky[kMaxN];
  int cut[kMaxN];
};
// Byte offsets of the tables inside the workspace's table region (each on a
// 256-byte boundary).
constexpr size_t al256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffTwCol = 0;
constexpr size_t kOffTwRow = al256(kOffTwCol + sizeof(Cx<double>) * kMaxN);
constexpr size_t kOffTwReal = al256(kOffTwRow + sizeof(Cx<double>) * (kMaxN / 2));
constexpr size_t kOffKx = al256(kOffTwReal + sizeof(Cx<double>) * (kMaxN / 2 + 1));
constexpr size_t kOffKy = al256(kOffKx + sizeof(double) * kMaxNh);
constexpr size_t kOffCut = al256(kOffKy + sizeof(double) * kMaxN);
constexpr size_t kOffStatus = kTableBytes - 256;
static_assert(kOffCut + sizeof(int) * kMaxN <= kOffStatus, "tables exceed the workspace's table region");

// Host cache of the last tables built and the lock that serialises the
// host-side preparation (workspace lookup, table build, table upload).
static std::mutex g_mu;
static NoallocTables g_tab;
static int g_key_n[2] = {0, 0};
static double g_key_d[3] = {0, 0, 0};

__global__ void k_noalloc_tables(const NoallocTables t, unsigned char* dtab, int Ny, int M, int Nh) {
  Cx<double>* twc = reinterpret_cast<Cx<double>*>(dtab + kOffTwCol);
  Cx<double>* twr = reinterpret_cast<Cx<double>*>(dtab + kOffTwRow);
  Cx<double>* twre = reinterpret_cast<Cx<double>*>(dtab + kOffTwReal);
  double* kx = reinterpret_cast<double*>(dtab + kOffKx);
  double* ky = reinterpret_cast<double*>(dtab + kOffKy);
  int* cut = reinterpret_cast<int*>(dtab + kOffCut);
  for (int m = threadIdx.x; m < Ny; m += blockDim.x) {
    twc[m] = t.tw_col[m];
    ky[m] = t.ky[m];
    cut[m] = t.cut[m];
  }
  for (int m = threadIdx.x; m <= M; m += blockDim.x) {
    if (m < M) twr[m] = t.tw_row[m];
    twre[m] = t.tw_real[m];
  }
  for (int i = threadIdx.x; i < Nh; i += blockDim.x) kx[i] = t.kx[i];
  if (threadIdx.x == 0) *reinterpret_cast<int*>(dtab + kOffStatus) = TARA_OK;
}

// Builds the tables of (Nx, Ny, Lx, Ly, pi) into g_tab with the reference
// formulas (kx, ky: src/derive2coh.f95:58-86; 2/3 rule: :208-212), unless
// g_tab holds them already.  Called with g_mu held.
void build_tables(int Nx, int Ny, const tara_params* p) {
  if (g_key_n[0] == Nx && g_key_n[1] == Ny && g_key_d[0] == p->Lx && g_key_d[1] == p->Ly && g_key_d[2] == p->pi)
    return;
  const int Nh = Nx / 2 + 1, M = Nx / 2;
  NoallocTables& t = g_tab;
  for (int m = 0; m < Ny; m++) {
    long double c, s;
    tara::twiddle(m, Ny, c, s);
    t.tw_col[m] = tara::cx<double>((double)c, (double)s);
  }
  for (int m = 0; m < M; m++) {
    long double c, s;
    tara::twiddle(m, M, c, s);
    t.tw_row[m] = tara::cx<double>((double)c, (double)s);
  }
  for (int m = 0; m <= M; m++) {
    long double c, s;
    tara::twiddle(m, Nx, c, s);
    t.tw_real[m] = tara::cx<double>((double)c, (double)s);
  }
  for (int i = 0; i < Nh; i++) t.kx[i] = 2.0 * p->pi * (double)i / p->Lx;
  for (int j = 0; j < Ny; j++)
    t.ky[j] = (j < Ny / 2) ? 2.0 * p->pi * (double)j / p->Ly : 2.0 * p->pi * (double)(j - Ny) / p->Ly;
  const double thr = ((double)(Nx + Ny) / 2.0) / 3.0 + 0;
  for (int j = 0; j < Ny; j++) {
    int c = Nh;
    for (int i = 0; i < Nh; i++) {
      volatile double a = t.kx[i] * t.kx[i];
      volatile double b = t.ky[j] * t.ky[j];
      volatile double sum = a + b;
      if (std::sqrt((double)sum) >= thr) { c = i; break; }
    }
    t.cut[j] = c;
  }
  g_key_n[0] = Nx;
  g_key_n[1] = Ny;
  g_key_d[0] = p->Lx;
  g_key_d[1] = p->Ly;
  g_key_d[2] = p->pi;
}

// Device address of the workspace on the current device.  Called with g_mu held.
int scratch_address(int dev, void** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    tara::set_error("device index out of range for the static workspace table");
    return TARA_EINVAL;
  }
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      tara::set_error(std::string("cudaGetSymbolAddress(workspace): ") + cudaGetErrorString(e));
      return TARA_ECUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return TARA_OK;
}

bool size_ok(int n) { return n == 16 || n == 32 || n == 64 || n == 128 || n == 256; }

}  // namespace

extern "C" int tara_derive2coh_noalloc(const tara_params* p, int Nx, int Ny, const double* nk,
                                       const double* ukx, const double* uky, double* dn_dt,
                                       double* dux_dt, double* duy_dt, void* stream) {
  using namespace tara;
  if (!p || !nk || !ukx || !uky || !dn_dt || !dux_dt || !duy_dt) {
    set_error("tara_derive2coh_noalloc: null argument");
    return TARA_EINVAL;
  }
  if (!size_ok(Nx) || !size_ok(Ny)) {
    set_error("tara_derive2coh_noalloc: Nx and Ny must be one of 16, 32, 64, 128, 256 (static workspace limit)");
    return TARA_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int Nh = Nx / 2 + 1, M = Nx / 2;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    set_error("tara_derive2coh_noalloc: device query failed");
    return TARA_ECUDA;
  }
  void* base = nullptr;
  unsigned char* dtab = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    const int r = scratch_address(dev, &base);
    if (r != TARA_OK) return r;
    build_tables(Nx, Ny, p);
    dtab = static_cast<unsigned char*>(base) + 11 * kField * sizeof(Cx<double>);
    // the launch copies g_tab into its parameters, so the lock may end after it
    k_noalloc_tables<<<1, 256, 0, st>>>(g_tab, dtab, Ny, M, Nh);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("tara_derive2coh_noalloc: table upload: ") + cudaGetErrorString(e));
      return TARA_ECUDA;
    }
  }

  Grid<double> g;  // describes the static workspace; init()/release() are never called
  g.Nx = Nx; g.Ny = Ny; g.Nh = Nh; g.ld = Nh;
  g.Lx = p->Lx; g.Ly = p->Ly; g.pi = p->pi;
  g.tb.tw_col = reinterpret_cast<const Cx<double>*>(dtab + kOffTwCol);
  g.tb.tw_row = reinterpret_cast<const Cx<double>*>(dtab + kOffTwRow);
  g.tb.tw_real = reinterpret_cast<const Cx<double>*>(dtab + kOffTwReal);
  g.tb.kx = reinterpret_cast<const double*>(dtab + kOffKx);
  g.tb.ky = reinterpret_cast<const double*>(dtab + kOffKy);
  g.tb.cut = reinterpret_cast<const int*>(dtab + kOffCut);
  g.tb.Nx = Nx; g.tb.Ny = Ny; g.tb.Nh = Nh; g.tb.ld = Nh;
  const double nn = (double)Nx * (double)Ny;
  g.tb.nn = nn;
  g.tb.inv_nn = 1.0 / nn;
  g.tb.nn_pow2 = 1;  // every accepted size is a power of two
  g.tb.status = reinterpret_cast<int*>(dtab + kOffStatus);  // written by no kernel of this path
  g.tb.sm_count = sms;
  g.tb.no_tma = 1;  // register-staged column passes: no TMA loads, no bounded waits
  g.tb.wait_ns = 0;

  // fields of this grid packed back to back in the workspace
  const size_t fe = (size_t)Ny * Nh;
  CohWork<double> w;
  w.H.base = static_cast<Cx<double>*>(base);
  w.H.elems = fe;
  w.H.count = 8;
  w.X.base = static_cast<Cx<double>*>(base) + 8 * fe;
  w.X.elems = fe;
  w.X.count = 3;

  CohParamsT<double> cp{p->mux, p->muy, p->CS * p->CS};
  Cx<double>* in[3] = {reinterpret_cast<Cx<double>*>(const_cast<double*>(nk)),
                       reinterpret_cast<Cx<double>*>(const_cast<double*>(ukx)),
                       reinterpret_cast<Cx<double>*>(const_cast<double*>(uky))};
  StepArgs<double> s{};
  s.mode = STEP_RHS;
  s.out[0] = reinterpret_cast<Cx<double>*>(dn_dt);
  s.out[1] = reinterpret_cast<Cx<double>*>(dux_dt);
  s.out[2] = reinterpret_cast<Cx<double>*>(duy_dt);
  return coh_rhs(g, w, cp, in, s, st);
}
