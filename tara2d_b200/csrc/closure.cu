// Learned subgrid closure for the MHD path (no counterpart in the reference).
//
// Training pairs come from a fine FP64 MHD session on Nf^2 (a DNS), filtered
// to the closure's Nc^2 grid by a sharp spectral cut (modes with
// |kx|, |ky| < Nc/2 kept, scaled by (Nc/Nf)^2 for the unnormalised transform):
//   input  (Nc^2, 5 channels): rho - 1, ux, uy, Bx, By of the filtered state
//   target (Nc^2, 4 channels): tau_xx, tau_xy, tau_yy, EMF with
//          tau_ij = filter(F_ij(fine)) - F_ij(filtered state) and F the
//          nonlinear momentum fluxes rho u_i u_j + B^2/2 d_ij - B_i B_j and the
//          EMF uy Bx - ux By of the reference's flux assembly
//          (src/derive2com.f95:193-213; the pressure CS^2 rho is linear and
//          has no subgrid part).
// Everything stays on the device: the dataset lives in HBM, batches are
// gathered with random periodic shifts and the point reflection
// (x, y) -> (-x, -y) (u, B change sign, tau and EMF do not), the CNN
// (cnn.cuh) trains with Adam on the MSE of the normalised targets.
// In a coarse run the session adds -(i kx tau_x. + i ky tau_.y) to the
// momentum derivatives and -i ky EMF / +i kx EMF to Bx / By, masked like the
// resolved fluxes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>
#include "closure.h"
#include "cnn.cuh"
#include "realspace.cuh"
#include "session.h"

using namespace tara;

namespace {

constexpr int kIn = kCnnIn, kOut = kCnnOut;

// sharp spectral filter: fine [Nf][ldf] -> coarse [Nc][ldc], scaled
__global__ void k_filter(const Cx<double>* __restrict__ f, int Nf, int ldf, Cx<double>* __restrict__ c, int Nc,
                         int ldc, double scale) {
  const int Nhc = Nc / 2 + 1;
  const size_t n = (size_t)Nhc * Nc;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int jc = (int)(q / Nhc), ic = (int)(q % Nhc);
    Cx<double> v = cx<double>(0.0, 0.0);
    if (ic < Nc / 2 && jc != Nc / 2) {
      const int jf = jc < Nc / 2 ? jc : jc + (Nf - Nc);
      const Cx<double> s = f[(size_t)jf * ldf + ic];
      v = cx<double>(s.x * scale, s.y * scale);
    }
    c[(size_t)jc * ldc + ic] = v;
  }
}

// nonlinear fluxes of real fields rho, mx, my, bx, by (src/derive2com.f95:193-213, no pressure)
__device__ __forceinline__ void fluxes(double rho, double mx, double my, double bx, double by, double* F) {
  const double ux = mx / rho, uy = my / rho;
  const double B2 = bx * bx + by * by;
  F[0] = mx * ux + B2 / 2.0 - bx * bx;
  F[1] = mx * uy - bx * by;
  F[2] = my * uy + B2 / 2.0 - by * by;
  F[3] = uy * bx - by * ux;
}

struct Real5 { const double* r[5]; };   // rho, mx, my, bx, by
struct Real4 { double* r[4]; };

__global__ void k_fine_fluxes(Real5 s, Real4 o, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    double F[4];
    fluxes(s.r[0][q], s.r[1][q], s.r[2][q], s.r[3][q], s.r[4][q], F);
    for (int k = 0; k < 4; k++) o.r[k][q] = F[k];
  }
}

// pair = (inputs, filtered flux - flux of the filtered state), FP32
__global__ void k_make_pair(Real5 s, Real4 filt, size_t n, float* __restrict__ in, float* __restrict__ out) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const double rho = s.r[0][q], mx = s.r[1][q], my = s.r[2][q], bx = s.r[3][q], by = s.r[4][q];
    double F[4];
    fluxes(rho, mx, my, bx, by, F);
    in[q] = (float)(rho - 1.0);
    in[n + q] = (float)(mx / rho);
    in[2 * n + q] = (float)(my / rho);
    in[3 * n + q] = (float)bx;
    in[4 * n + q] = (float)by;
    for (int k = 0; k < 4; k++) out[k * n + q] = (float)(filt.r[k][q] - F[k]);
  }
}

struct Norm { float mi[kIn], si[kIn], mo[kOut], so[kOut]; };

// network input of a coarse state (B = 1)
__global__ void k_cnn_input(Real5 s, size_t n, Norm nm, float* __restrict__ in) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const double rho = s.r[0][q];
    const float v[kIn] = {(float)(rho - 1.0), (float)(s.r[1][q] / rho), (float)(s.r[2][q] / rho), (float)s.r[3][q],
                          (float)s.r[4][q]};
    for (int c = 0; c < kIn; c++) in[c * n + q] = (v[c] - nm.mi[c]) / nm.si[c];
  }
}
__global__ void k_cnn_output(const float* __restrict__ out, size_t n, Norm nm, Real4 o) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    for (int c = 0; c < kOut; c++) o.r[c][q] = (double)(out[c * n + q] * nm.so[c] + nm.mo[c]);
}

// one batch: sample idx[b] shifted by (sx, sy), point-reflected if flip,
// normalised
__global__ void k_gather(const float* __restrict__ din, const float* __restrict__ dout, const int4* __restrict__ pick,
                         int N, Norm nm, float* __restrict__ bin, float* __restrict__ bout) {
  const size_t plane = (size_t)N * N;
  const int b = blockIdx.y;
  const int4 p = pick[b];  // x: sample, y: sx, z: sy, w: flip
  const float* si = din + (size_t)p.x * kIn * plane;
  const float* so = dout + (size_t)p.x * kOut * plane;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < plane; q += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(q / N), x = (int)(q % N);
    int ys = p.w ? -y : y, xs = p.w ? -x : x;
    ys = ((ys + p.z) % N + N) % N;
    xs = ((xs + p.y) % N + N) % N;
    const size_t src = (size_t)ys * N + xs;
    for (int c = 0; c < kIn; c++) {
      const float sg = (p.w && c > 0) ? -1.0f : 1.0f;  // u and B reverse under the reflection
      bin[((size_t)b * kIn + c) * plane + q] = (sg * si[c * plane + src] - nm.mi[c]) / nm.si[c];
    }
    for (int c = 0; c < kOut; c++) bout[((size_t)b * kOut + c) * plane + q] = (so[c * plane + src] - nm.mo[c]) / nm.so[c];
  }
}

__global__ void k_channel_stats(const float* __restrict__ d, int first, int count, int C, size_t plane,
                                double* __restrict__ acc /* [C][2] */) {
  const int c = blockIdx.y;
  double s = 0.0, s2 = 0.0;
  const size_t n = (size_t)count * plane;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t smp = first + q / plane;
    const double v = d[(smp * C + c) * plane + q % plane];
    s += v;
    s2 += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 2 * c, s);
    atomicAdd(acc + 2 * c + 1, s2);
  }
}

}  // namespace

struct tara_closure {
  int Nc = 0, cap = 0, count = 0, Bmax = 0;
  cudaStream_t st = nullptr;
  Cnn net;
  Norm norm{};
  float* din = nullptr;    // [cap][5][Nc][Nc]
  float* dout = nullptr;   // [cap][4][Nc][Nc]
  float* bin = nullptr;    // [Bmax][5][Nc][Nc]
  float* bout = nullptr;   // [Bmax][4][Nc][Nc]
  int4* pick = nullptr;
  double* stats = nullptr;
  double* rc = nullptr;    // coarse real FP64 fields [9][Nc*Nc]
  FieldPool<double> cs;    // coarse spectral fields (9): filtered state (5) and fluxes (4)
  FieldPool<double> cw;    // coarse work fields (9)
  Grid<double> cg;
  // fine-grid buffers of the last Nf used
  int Nf = 0;
  double* rf = nullptr;    // [10][Nf*Nf]: 6 state + 4 fluxes
  FieldPool<double> fs, fw;  // fine spectral fluxes (4), fine work (6)
  Grid<double> fg;
  std::mt19937_64 rng;
  ~tara_closure() {
    if (st) cudaStreamSynchronize(st);
    net.release();
    for (void* p : {(void*)din, (void*)dout, (void*)bin, (void*)bout, (void*)pick, (void*)stats, (void*)rc, (void*)rf})
      if (p) cudaFree(p);
    cs.release(); cw.release(); fs.release(); fw.release(); cg.release(); fg.release();
    if (st) cudaStreamDestroy(st);
  }
};

namespace tara {
int closure_grid(const tara_closure* c) { return c ? c->Nc : 0; }

int closure_terms(tara_closure* c, const Grid<double>& g, Cx<double>* const* in, Cx<double>* const* out4,
                  cudaStream_t st) {
  const size_t n = (size_t)c->Nc * c->Nc;
  const Cx<double>* src[5] = {in[0], in[1], in[2], in[4], in[5]};
  double* r[9];
  for (int k = 0; k < 9; k++) r[k] = c->rc + k * n;
  Cx<double>* wk[8];
  for (int k = 0; k < 8; k++) wk[k] = c->cw[k];
  TARA_TRY(c2r_fields(g, 5, src, r, wk, true, st));
  Real5 s{{r[0], r[1], r[2], r[3], r[4]}};
  k_cnn_input<<<256, 256, 0, st>>>(s, n, c->norm, c->bin);
  TARA_TRY(c->net.forward(c->bin, 1, false, st));
  Real4 o{{r[5], r[6], r[7], r[8]}};
  k_cnn_output<<<256, 256, 0, st>>>(c->net.out(), n, c->norm, o);
  const double* ro[4] = {r[5], r[6], r[7], r[8]};
  return r2c_fields(g, 4, ro, out4, wk, st);
}
}  // namespace tara

namespace {

// One training pair from an FP64 MHD state on the fine grid fg (six
// spectral fields, last written on stream src).
int add_pair_from(tara_closure* c, const Grid<double>& fg, Cx<double>* const* fstate, cudaStream_t src) {
  if (fg.Nx != fg.Ny || fg.Nx % c->Nc != 0) {
    set_error("training pairs come from an FP64 MHD state on a square grid that the closure grid divides");
    return TARA_EINVAL;
  }
  if (c->count >= c->cap) { set_error("the closure's dataset is full"); return TARA_EINVAL; }
  const int Nf = fg.Nx, Nc = c->Nc;
  if (c->Nf != Nf) {
    if (c->rf) cudaFree(c->rf);
    c->rf = nullptr;
    c->fs.release();
    c->fw.release();
    c->Nf = Nf;
    TARA_CUDA_TRY(cudaMalloc(&c->rf, (size_t)10 * Nf * Nf * sizeof(double)));
    TARA_TRY(c->fs.alloc(fg, 4, c->st));
    TARA_TRY(c->fw.alloc(fg, 6, c->st));
  }
  TARA_CUDA_TRY(cudaStreamSynchronize(src));
  cudaStream_t st = c->st;
  const size_t nf = (size_t)Nf * Nf, nc = (size_t)Nc * Nc;
  // fine state in real space, its nonlinear fluxes, their spectra
  Cx<double>* state[6];
  double* rf[10];
  Cx<double>* fw[6];
  for (int k = 0; k < 6; k++) {
    state[k] = fstate[k];
    fw[k] = c->fw[k];
  }
  for (int k = 0; k < 10; k++) rf[k] = c->rf + k * nf;
  TARA_TRY(state_to_real(fg, 6, state, rf, fw, st));
  k_fine_fluxes<<<592, 256, 0, st>>>(Real5{{rf[0], rf[1], rf[2], rf[4], rf[5]}}, Real4{{rf[6], rf[7], rf[8], rf[9]}},
                                     nf);
  const double* fl[4] = {rf[6], rf[7], rf[8], rf[9]};
  Cx<double>* fsp[4] = {c->fs[0], c->fs[1], c->fs[2], c->fs[3]};
  TARA_TRY(r2c_fields(fg, 4, fl, fsp, fw, st));
  // sharp filter of the state (rho, mx, my, bx, by) and of the flux spectra
  const double scale = ((double)Nc * Nc) / ((double)Nf * Nf);
  const Cx<double>* fsrc[9] = {state[0], state[1], state[2], state[4], state[5], c->fs[0], c->fs[1], c->fs[2], c->fs[3]};
  for (int k = 0; k < 9; k++)
    k_filter<<<256, 256, 0, st>>>(fsrc[k], Nf, fg.ld, c->cs[k], Nc, c->cg.ld, scale);
  double* rc[9];
  const Cx<double>* csrc[9];
  Cx<double>* cw[9];
  for (int k = 0; k < 9; k++) {
    rc[k] = c->rc + k * nc;
    csrc[k] = c->cs[k];
    cw[k] = c->cw[k];
  }
  TARA_TRY(c2r_fields(c->cg, 5, csrc, rc, cw, true, st));
  TARA_TRY(c2r_fields(c->cg, 4, csrc + 5, rc + 5, cw, true, st));
  float* pin = c->din + (size_t)c->count * kIn * nc;
  float* pout = c->dout + (size_t)c->count * kOut * nc;
  k_make_pair<<<256, 256, 0, st>>>(Real5{{rc[0], rc[1], rc[2], rc[3], rc[4]}}, Real4{{rc[5], rc[6], rc[7], rc[8]}}, nc,
                                   pin, pout);
  TARA_CUDA_TRY(cudaGetLastError());
  TARA_CUDA_TRY(cudaStreamSynchronize(st));
  c->count++;
  return TARA_OK;
}
int add_pair(tara_closure* c, tara_session* fine) {
  if (fine->model != TARA_MODEL_COM || fine->precision != TARA_FP64) {
    set_error("training pairs come from an FP64 MHD session on a square grid that the closure grid divides");
    return TARA_EINVAL;
  }
  Cx<double>* state[6];
  for (int k = 0; k < 6; k++) state[k] = static_cast<Cx<double>*>(fine->state_ptr(k));
  return add_pair_from(c, *static_cast<const Grid<double>*>(fine->grid_ptr()), state, fine->st);
}

// one pass over samples [first, first + count) in batches; train: shuffled,
// augmented, one Adam step per batch.  Returns the mean loss per element.
int run_epoch(tara_closure* c, int first, int count, int batch, bool train, float lr, double* loss) {
  const int N = c->Nc;
  std::vector<int> order(count);
  for (int k = 0; k < count; k++) order[k] = first + k;
  if (train) std::shuffle(order.begin(), order.end(), c->rng);
  TARA_CUDA_TRY(cudaMemsetAsync(c->net.lossacc, 0, sizeof(double), c->st));
  std::vector<int4> pk(batch);
  for (int s = 0; s < count; s += batch) {
    const int B = std::min(batch, count - s);
    for (int b = 0; b < B; b++) {
      if (train) {
        pk[b] = make_int4(order[s + b], (int)(c->rng() % N), (int)(c->rng() % N), (int)(c->rng() & 1));
      } else {
        pk[b] = make_int4(order[s + b], 0, 0, 0);
      }
    }
    TARA_CUDA_TRY(cudaMemcpyAsync(c->pick, pk.data(), B * sizeof(int4), cudaMemcpyHostToDevice, c->st));
    k_gather<<<dim3(64, B), 256, 0, c->st>>>(c->din, c->dout, c->pick, N, c->norm, c->bin, c->bout);
    TARA_TRY(c->net.forward(c->bin, B, train, c->st));
    TARA_TRY(c->net.mse(c->bout, B, c->st));
    if (train) {
      TARA_TRY(c->net.backward(c->bin, c->net.dz[1], B, c->st));
      TARA_TRY(c->net.adam(lr, 0.9f, 0.999f, 1e-8f, c->st));
    }
    TARA_CUDA_TRY(cudaStreamSynchronize(c->st));  // pick[] is reused by the next batch
  }
  double acc = 0.0;
  TARA_CUDA_TRY(cudaMemcpyAsync(&acc, c->net.lossacc, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  // k_mse sums squared errors of each batch; report the mean over all elements
  *loss = acc / ((double)count * kOut * N * N);
  return TARA_OK;
}

}  // namespace

extern "C" {

int tara_closure_open(tara_closure** out, int Nc, int capacity, int batch_max, unsigned long long seed) {
  if (!out || capacity < 1 || batch_max < 1 || Nc < 16 || Nc % 16 || !supported_length(Nc)) {
    set_error("closure grid must be a supported size and a multiple of 16; capacity, batch >= 1");
    return TARA_EINVAL;
  }
  *out = nullptr;
  std::unique_ptr<tara_closure> c(new tara_closure());
  c->Nc = Nc;
  c->cap = capacity;
  c->Bmax = batch_max;
  c->rng.seed(seed);
  TARA_CUDA_TRY(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  const double pi = 3.14159265358979323846;
  TARA_TRY(c->cg.init(Nc, Nc, 2 * pi, 2 * pi, pi, c->st));
  const size_t nc = (size_t)Nc * Nc;
  auto am = [&](void** p, size_t b) { return cudaMalloc(p, b) == cudaSuccess; };
  if (!am((void**)&c->din, (size_t)capacity * kIn * nc * 4) || !am((void**)&c->dout, (size_t)capacity * kOut * nc * 4) ||
      !am((void**)&c->bin, (size_t)batch_max * kIn * nc * 4) || !am((void**)&c->bout, (size_t)batch_max * kOut * nc * 4) ||
      !am((void**)&c->pick, (size_t)batch_max * sizeof(int4)) || !am((void**)&c->stats, 2 * 9 * sizeof(double)) ||
      !am((void**)&c->rc, 9 * nc * sizeof(double))) {
    set_error("cudaMalloc of the closure dataset and buffers failed");
    return TARA_ENOMEM;
  }
  TARA_TRY(c->cs.alloc(c->cg, 9, c->st));
  TARA_TRY(c->cw.alloc(c->cg, 9, c->st));
  TARA_TRY(c->net.alloc(Nc, Nc, batch_max));
  // He-style initialisation, seeded; biases zero
  const int np = cnn_num_params();
  std::vector<float> w(np, 0.0f);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  int off = 0;
  for (int l = 0; l < kCnnLayers; l++) {
    const CnnLayerDims d = cnn_layer(l);
    const float sd = std::sqrt(2.0f / (9.0f * d.cin)) * (l == kCnnLayers - 1 ? 0.1f : 1.0f);
    for (int k = 0; k < d.cout * d.cin * 9; k++) w[off + k] = sd * nd(c->rng);
    off += d.cout * d.cin * 9 + d.cout;
  }
  // every copy of the closure is ordered on its (non-blocking) stream: a plain
  // cudaMemcpy from pageable memory may return before the data has reached
  // the device, and the weight packing on c->st could then read old weights
  TARA_CUDA_TRY(cudaMemcpyAsync(c->net.master, w.data(), np * 4, cudaMemcpyHostToDevice, c->st));
  TARA_TRY(c->net.refresh(c->st));
  for (int k = 0; k < kIn; k++) { c->norm.mi[k] = 0.0f; c->norm.si[k] = 1.0f; }
  for (int k = 0; k < kOut; k++) { c->norm.mo[k] = 0.0f; c->norm.so[k] = 1.0f; }
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  *out = c.release();
  return TARA_OK;
}
int tara_closure_close(tara_closure* c) {
  if (!c) return TARA_EINVAL;
  delete c;
  return TARA_OK;
}
int tara_closure_num_params(void) { return cnn_num_params(); }
int tara_closure_count(const tara_closure* c) { return c ? c->count : 0; }
int tara_closure_add_pair(tara_closure* c, tara_session* fine) {
  if (!c || !fine) return TARA_EINVAL;
  return add_pair(c, fine);
}
// a training pair from the current state of FP64 MHD ensemble member m
int tara_closure_add_pair_member(tara_closure* c, tara_ensemble* e, int member) {
  if (!c || !e) return TARA_EINVAL;
  const Grid<double>* g = nullptr;
  Cx<double>* state[6];
  cudaStream_t st = nullptr;
  TARA_TRY(ens_member_state(e, member, &g, state, &st));
  return add_pair_from(c, *g, state, st);
}
int tara_closure_get_pair(tara_closure* c, int idx, float* in5, float* out4) {
  if (!c || idx < 0 || idx >= c->count || !in5 || !out4) return TARA_EINVAL;
  const size_t nc = (size_t)c->Nc * c->Nc;
  TARA_CUDA_TRY(cudaMemcpyAsync(in5, c->din + (size_t)idx * kIn * nc, kIn * nc * 4, cudaMemcpyDeviceToHost, c->st));
  TARA_CUDA_TRY(
      cudaMemcpyAsync(out4, c->dout + (size_t)idx * kOut * nc, kOut * nc * 4, cudaMemcpyDeviceToHost, c->st));
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  return TARA_OK;
}
// norm: mean_in[5], std_in[5], mean_out[4], std_out[4]
int tara_closure_get_norm(const tara_closure* c, float* norm18) {
  if (!c || !norm18) return TARA_EINVAL;
  std::memcpy(norm18, &c->norm, sizeof(Norm));
  return TARA_OK;
}
int tara_closure_set_norm(tara_closure* c, const float* norm18) {
  if (!c || !norm18) return TARA_EINVAL;
  Norm n;
  std::memcpy(&n, norm18, sizeof(Norm));
  for (int k = 0; k < kIn; k++)
    if (!(n.si[k] > 0)) { set_error("scales must be positive"); return TARA_EINVAL; }
  for (int k = 0; k < kOut; k++)
    if (!(n.so[k] > 0)) { set_error("scales must be positive"); return TARA_EINVAL; }
  c->norm = n;
  return TARA_OK;
}
int tara_closure_fit_norm(tara_closure* c, int first, int count) {
  if (!c || first < 0 || count < 1 || first + count > c->count) return TARA_EINVAL;
  const size_t plane = (size_t)c->Nc * c->Nc;
  double h[18];
  TARA_CUDA_TRY(cudaMemsetAsync(c->stats, 0, 18 * sizeof(double), c->st));
  k_channel_stats<<<dim3(256, kIn), 256, 0, c->st>>>(c->din, first, count, kIn, plane, c->stats);
  k_channel_stats<<<dim3(256, kOut), 256, 0, c->st>>>(c->dout, first, count, kOut, plane, c->stats + 2 * kIn);
  TARA_CUDA_TRY(cudaMemcpyAsync(h, c->stats, 18 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  const double n = (double)count * plane;
  for (int k = 0; k < kIn + kOut; k++) {
    const double m = h[2 * k] / n, v = std::max(h[2 * k + 1] / n - m * m, 0.0);
    const float sd = (float)std::sqrt(v);
    const bool in = k < kIn;
    const int i = in ? k : k - kIn;
    // u and B are odd under the reflection used for augmentation: centre them at 0
    const float mean = (in && k > 0) ? 0.0f : (float)m;
    (in ? c->norm.mi : c->norm.mo)[i] = mean;
    (in ? c->norm.si : c->norm.so)[i] = sd > 1e-30f ? sd : 1.0f;
  }
  return TARA_OK;
}
int tara_closure_train(tara_closure* c, int first, int count, int epochs, int batch, float lr, float* epoch_loss) {
  if (!c || first < 0 || count < 1 || first + count > c->count || epochs < 0 || batch < 1 || batch > c->Bmax)
    return TARA_EINVAL;
  for (int e = 0; e < epochs; e++) {
    double l = 0;
    TARA_TRY(run_epoch(c, first, count, batch, true, lr, &l));
    if (epoch_loss) epoch_loss[e] = (float)l;
  }
  return c->net.check(c->st);
}
int tara_closure_eval_loss(tara_closure* c, int first, int count, float* loss) {
  if (!c || !loss || first < 0 || count < 1 || first + count > c->count) return TARA_EINVAL;
  double l = 0;
  TARA_TRY(run_epoch(c, first, count, c->Bmax, false, 0.0f, &l));
  *loss = (float)l;
  return c->net.check(c->st);
}
int tara_closure_set_tensor_cores(tara_closure* c, int on) {
  if (!c) return TARA_EINVAL;
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  c->net.tensor_cores = on ? 1 : 0;
  return TARA_OK;
}
int tara_closure_status(tara_closure* c) { return c ? c->net.check(c->st) : TARA_EINVAL; }
// device time of `reps` network evaluations on the batch buffer (B samples of
// whatever it holds): forward alone, and forward + backward with the output
// gradient in the other batch buffer
int tara_closure_time_cnn(tara_closure* c, int B, int reps, float* ms_forward, float* ms_backward) {
  if (!c || !ms_forward || !ms_backward || B < 1 || B > c->Bmax || reps < 1) return TARA_EINVAL;
  cudaEvent_t e[3];
  for (auto& x : e) TARA_CUDA_TRY(cudaEventCreate(&x));
  int r = TARA_OK;
  r = c->net.forward(c->bin, B, true, c->st);  // warm-up
  if (r == TARA_OK) r = c->net.backward(c->bin, c->bout, B, c->st);
  cudaEventRecord(e[0], c->st);
  for (int k = 0; k < reps && r == TARA_OK; k++) r = c->net.forward(c->bin, B, true, c->st);
  cudaEventRecord(e[1], c->st);
  for (int k = 0; k < reps && r == TARA_OK; k++) {
    r = c->net.forward(c->bin, B, true, c->st);
    if (r == TARA_OK) r = c->net.backward(c->bin, c->bout, B, c->st);
  }
  cudaEventRecord(e[2], c->st);
  if (cudaEventSynchronize(e[2]) != cudaSuccess && r == TARA_OK) {
    set_error("cudaEventSynchronize failed");
    r = TARA_ECUDA;
  }
  if (r == TARA_OK) {
    cudaEventElapsedTime(ms_forward, e[0], e[1]);
    cudaEventElapsedTime(ms_backward, e[1], e[2]);
    *ms_forward /= reps;
    *ms_backward /= reps;
  }
  for (auto& x : e) cudaEventDestroy(x);
  return r == TARA_OK ? c->net.check(c->st) : r;
}
int tara_closure_get_params(tara_closure* c, float* w) {
  if (!c || !w) return TARA_EINVAL;
  TARA_CUDA_TRY(cudaMemcpyAsync(w, c->net.master, cnn_num_params() * 4, cudaMemcpyDeviceToHost, c->st));
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  return TARA_OK;
}
int tara_closure_set_params(tara_closure* c, const float* w) {
  if (!c || !w) return TARA_EINVAL;
  TARA_CUDA_TRY(cudaMemcpyAsync(c->net.master, w, cnn_num_params() * 4, cudaMemcpyHostToDevice, c->st));
  TARA_TRY(c->net.refresh(c->st));
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  return TARA_OK;
}
// network on normalised inputs: in [B][5][Nc][Nc] -> out [B][4][Nc][Nc]
int tara_closure_forward(tara_closure* c, const float* in, int B, float* out) {
  if (!c || !in || !out || B < 1 || B > c->Bmax) return TARA_EINVAL;
  const size_t nc = (size_t)c->Nc * c->Nc;
  TARA_CUDA_TRY(cudaMemcpyAsync(c->bin, in, (size_t)B * kIn * nc * 4, cudaMemcpyHostToDevice, c->st));
  TARA_TRY(c->net.forward(c->bin, B, true, c->st));
  TARA_CUDA_TRY(cudaMemcpyAsync(out, c->net.out(), (size_t)B * kOut * nc * 4, cudaMemcpyDeviceToHost, c->st));
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  return c->net.check(c->st);
}
// gradient of sum(dout * net(in)) with respect to the parameters
int tara_closure_backward(tara_closure* c, const float* in, const float* dout, int B, float* grad) {
  if (!c || !in || !dout || !grad || B < 1 || B > c->Bmax) return TARA_EINVAL;
  const size_t nc = (size_t)c->Nc * c->Nc;
  TARA_CUDA_TRY(cudaMemcpyAsync(c->bin, in, (size_t)B * kIn * nc * 4, cudaMemcpyHostToDevice, c->st));
  TARA_TRY(c->net.forward(c->bin, B, true, c->st));
  TARA_CUDA_TRY(cudaMemcpyAsync(c->bout, dout, (size_t)B * kOut * nc * 4, cudaMemcpyHostToDevice, c->st));
  TARA_TRY(c->net.backward(c->bin, c->bout, B, c->st));
  TARA_CUDA_TRY(cudaMemcpyAsync(grad, c->net.grad, cnn_num_params() * 4, cudaMemcpyDeviceToHost, c->st));
  TARA_CUDA_TRY(cudaStreamSynchronize(c->st));
  return c->net.check(c->st);
}
int tara_session_attach_closure(tara_session* s, tara_closure* c) {
  if (!s) return TARA_EINVAL;
  return s->fail_if(s->attach_closure(c));
}
int tara_session_set_closure_mode(tara_session* s, int mode) {
  if (!s) return TARA_EINVAL;
  return s->fail_if(s->set_closure_mode(mode));
}
// coarse state = sharp spectral filter of the fine state (both MHD FP64)
int tara_filter_state(tara_session* fine, tara_session* coarse) {
  if (!fine || !coarse) return TARA_EINVAL;
  if (fine->model != coarse->model || fine->precision != TARA_FP64 || coarse->precision != TARA_FP64 ||
      fine->Nx != fine->Ny || coarse->Nx != coarse->Ny || fine->Nx % coarse->Nx != 0) {
    set_error("filtering needs FP64 sessions of one model on square grids, the coarse size dividing the fine");
    return TARA_EINVAL;
  }
  const Grid<double>& fg = *static_cast<const Grid<double>*>(fine->grid_ptr());
  const Grid<double>& cg = *static_cast<const Grid<double>*>(coarse->grid_ptr());
  TARA_CUDA_TRY(cudaStreamSynchronize(fine->st));
  const double scale = ((double)coarse->Nx * coarse->Nx) / ((double)fine->Nx * fine->Nx);
  for (int k = 0; k < fine->nf; k++)
    k_filter<<<256, 256, 0, coarse->st>>>(static_cast<Cx<double>*>(fine->state_ptr(k)), fine->Nx, fg.ld,
                                          static_cast<Cx<double>*>(coarse->state_ptr(k)), coarse->Nx, cg.ld, scale);
  TARA_CUDA_TRY(cudaGetLastError());
  TARA_CUDA_TRY(cudaStreamSynchronize(coarse->st));
  coarse->invalidate_derived();
  return TARA_OK;
}

}  // extern "C"
