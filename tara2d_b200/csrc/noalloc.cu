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
//   * The first call on a device looks up the workspace's device address
//     (cudaGetSymbolAddress) for that device; make that first call before
//     any stream capture begins.
#include <cmath>
#include <cstring>
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

// Host staging of the tables: fixed-size, so that building them allocates nothing.
static Cx<double> h_tw_col[kMaxN];
static Cx<double> h_tw_row[kMaxN / 2];
static Cx<double> h_tw_real[kMaxN / 2 + 1];
static double h_kx[kMaxNh];
static double h_ky[kMaxN];
static int h_cut[kMaxN];
static unsigned char h_tables[kTableBytes];

int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    tara::set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return TARA_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    tara::set_error("device index out of range for the static workspace table");
    return TARA_EINVAL;
  }
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
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
  void* base = nullptr;
  int r = scratch_address(&base);
  if (r != TARA_OK) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int Nh = Nx / 2 + 1, M = Nx / 2;

  // Tables, built on the host into fixed buffers with the reference formulas
  // (kx, ky: src/derive2coh.f95:58-86; 2/3 rule: :208-212).
  for (int m = 0; m < Ny; m++) { long double c, s; twiddle(m, Ny, c, s); h_tw_col[m] = cx<double>((double)c, (double)s); }
  for (int m = 0; m < M; m++) { long double c, s; twiddle(m, M, c, s); h_tw_row[m] = cx<double>((double)c, (double)s); }
  for (int m = 0; m <= M; m++) { long double c, s; twiddle(m, Nx, c, s); h_tw_real[m] = cx<double>((double)c, (double)s); }
  for (int i = 0; i < Nh; i++) h_kx[i] = 2.0 * p->pi * (double)i / p->Lx;
  for (int j = 0; j < Ny; j++)
    h_ky[j] = (j < Ny / 2) ? 2.0 * p->pi * (double)j / p->Ly : 2.0 * p->pi * (double)(j - Ny) / p->Ly;
  const double thr = ((double)(Nx + Ny) / 2.0) / 3.0 + 0;
  for (int j = 0; j < Ny; j++) {
    int c = Nh;
    for (int i = 0; i < Nh; i++) {
      volatile double a = h_kx[i] * h_kx[i];
      volatile double b = h_ky[j] * h_ky[j];
      volatile double sum = a + b;
      if (std::sqrt((double)sum) >= thr) { c = i; break; }
    }
    h_cut[j] = c;
  }
  size_t off[6], o = 0;
  const size_t bytes[6] = {Ny * sizeof(Cx<double>), M * sizeof(Cx<double>), (M + 1) * sizeof(Cx<double>),
                           Nh * sizeof(double), Ny * sizeof(double), Ny * sizeof(int)};
  const void* src[6] = {h_tw_col, h_tw_row, h_tw_real, h_kx, h_ky, h_cut};
  for (int q = 0; q < 6; q++) {
    off[q] = o;
    std::memcpy(h_tables + o, src[q], bytes[q]);
    o += (bytes[q] + 255) / 256 * 256;
  }
  unsigned char* dtab = static_cast<unsigned char*>(base) + 11 * kField * sizeof(Cx<double>);
  cudaError_t e = cudaMemcpyAsync(dtab, h_tables, o, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    set_error(std::string("tara_derive2coh_noalloc: table upload: ") + cudaGetErrorString(e));
    return TARA_ECUDA;
  }

  Grid<double> g;  // describes the static workspace; init()/release() are never called
  g.Nx = Nx; g.Ny = Ny; g.Nh = Nh; g.ld = Nh;
  g.Lx = p->Lx; g.Ly = p->Ly; g.pi = p->pi;
  g.tb.tw_col = reinterpret_cast<const Cx<double>*>(dtab + off[0]);
  g.tb.tw_row = reinterpret_cast<const Cx<double>*>(dtab + off[1]);
  g.tb.tw_real = reinterpret_cast<const Cx<double>*>(dtab + off[2]);
  g.tb.kx = reinterpret_cast<const double*>(dtab + off[3]);
  g.tb.ky = reinterpret_cast<const double*>(dtab + off[4]);
  g.tb.cut = reinterpret_cast<const int*>(dtab + off[5]);
  g.tb.Nx = Nx; g.tb.Ny = Ny; g.tb.Nh = Nh; g.tb.ld = Nh;
  const double nn = (double)Nx * (double)Ny;
  g.tb.nn = nn;
  g.tb.inv_nn = 1.0 / nn;
  g.tb.nn_pow2 = 1;  // every accepted size is a power of two
  // status word of the kernels' bounded waits: the last 256 bytes of the table region
  g.tb.status = reinterpret_cast<int*>(dtab + kTableBytes - 256);
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    set_error("tara_derive2coh_noalloc: device query failed");
    return TARA_ECUDA;
  }
  g.tb.sm_count = sms;
  const int zero = 0;
  e = cudaMemcpyAsync(g.tb.status, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    set_error(std::string("tara_derive2coh_noalloc: status reset: ") + cudaGetErrorString(e));
    return TARA_ECUDA;
  }

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
