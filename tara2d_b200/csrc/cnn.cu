// Closure CNN kernels and their host driver (see cnn.cuh).
//
//   k_conv      3x3 periodic convolution of a 16x16 pixel tile for every
//               output channel: the input tile with its one-pixel halo
//               (wrapped around the periodic box) and the layer's weights
//               (BF16, widened to FP32) are staged in shared memory; each
//               thread accumulates one pixel's COUT outputs in FP32.  The
//               epilogue adds the bias and applies GELU (keeping the
//               pre-activation), nothing, or the GELU derivative of the
//               previous layer (input-gradient pass with mirrored weights).
//   k_conv_dw   weight and bias gradients of one tile: each thread owns
//               (cout, cin) pairs and all 9 taps; per-CTA partials are then
//               summed in a fixed order by k_sum_parts.
//   k_mse, k_adam, k_pack_weights: loss/gradient, optimiser, BF16 layouts.
#include <algorithm>
#include <cmath>
#include <cstring>
#include "cnn.cuh"
#include "plan.h"
#include "umma.cuh"

namespace tara {

namespace {

constexpr int kTile = 16, kHalo = 18, kPlane = kHalo * kHalo;

enum { EPI_GELU = 0, EPI_LINEAR = 1, EPI_GELUGRAD = 2 };

__device__ __forceinline__ float gelu(float v) { return 0.5f * v * (1.0f + erff(v * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float v) {
  return 0.5f * (1.0f + erff(v * 0.70710678118654752f)) + v * 0.39894228040143268f * expf(-0.5f * v * v);
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// COUTT output channels in all, COUT of them (from blockIdx.z % (COUTT/COUT))
// per CTA: small batches split the channels over more CTAs.
template <int CIN, int COUTT, int COUT, int EPI>
__global__ void __launch_bounds__(256) k_conv(const float* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                              const float* __restrict__ bias, float* __restrict__ z,
                                              float* __restrict__ out, const float* __restrict__ zprev, int H,
                                              int W) {
  static_assert(COUT % 4 == 0 && COUTT % COUT == 0, "output channels in groups of four");
  constexpr int S = COUTT / COUT;
  extern __shared__ __align__(16) float sm[];
  float* xs = sm;                  // [CIN][18][18]
  float* ws = sm + CIN * kPlane;   // [CIN*9][COUT]
  const int b = blockIdx.z / S, c0 = (blockIdx.z % S) * COUT;
  const int y0 = blockIdx.y * kTile, x0 = blockIdx.x * kTile;
  const int tid = threadIdx.x, ty = tid / kTile, tx = tid % kTile;
  const size_t plane = (size_t)H * W;
  const float* inb = in + (size_t)b * CIN * plane;
  for (int q = tid; q < CIN * kPlane; q += 256) {
    const int c = q / kPlane, r = q % kPlane;
    const int gy = wrap(y0 + r / kHalo - 1, H), gx = wrap(x0 + r % kHalo - 1, W);
    xs[q] = __ldg(inb + c * plane + (size_t)gy * W + gx);
  }
  for (int q = tid; q < CIN * 9 * COUT; q += 256) ws[q] = __bfloat162float(w[(q / COUT) * COUTT + c0 + q % COUT]);
  __syncthreads();
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; co++) acc[co] = 0.0f;
#pragma unroll 1
  for (int ci = 0; ci < CIN; ci++) {
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
      const float xv = xs[ci * kPlane + (ty + tap / 3) * kHalo + tx + tap % 3];
      const float4* wr = reinterpret_cast<const float4*>(ws + (ci * 9 + tap) * COUT);
#pragma unroll
      for (int k = 0; k < COUT / 4; k++) {
        const float4 w4 = wr[k];
        acc[4 * k] = fmaf(xv, w4.x, acc[4 * k]);
        acc[4 * k + 1] = fmaf(xv, w4.y, acc[4 * k + 1]);
        acc[4 * k + 2] = fmaf(xv, w4.z, acc[4 * k + 2]);
        acc[4 * k + 3] = fmaf(xv, w4.w, acc[4 * k + 3]);
      }
    }
  }
  const size_t po = (size_t)(y0 + ty) * W + x0 + tx;
#pragma unroll
  for (int co = 0; co < COUT; co++) {
    const float v = acc[co] + (bias ? __ldg(bias + c0 + co) : 0.0f);
    const size_t idx = ((size_t)b * COUTT + c0 + co) * plane + po;
    if constexpr (EPI == EPI_GELU) {
      z[idx] = v;
      out[idx] = gelu(v);
    } else if constexpr (EPI == EPI_LINEAR) {
      out[idx] = v;
    } else {
      out[idx] = v * gelu_d(__ldg(zprev + idx));
    }
  }
}

// ---------------------------------------------------------------------------
// Tensor-core path of the convolutions (all four layers forward and the
// three input-gradient convolutions), as an implicit GEMM on tcgen05
// (kind::tf32, FP32 accumulation in TMEM).
//
// A CTA (four warps) computes one image row y0 of kTcPix pixels x0.. for
// all output channels of a layer: one M = 128 (pixels) x N accumulator,
// K = (input channels) x 9 taps, issued as 9 taps x CG/2 MMAs of K = 8.  The
// input row with its one-pixel periodic halo (three image rows) is staged in
// shared memory as [channel group of 4][halo row][halo pixel][4] (TF32,
// rounded to nearest): in the canonical no-swizzle K-major layout every pixel
// is one 16-byte core-matrix row, so the A operand of tap (dy, dx) is the
// same buffer with its start shifted by dy halo rows and dx pixels; no
// im2col copy is made.  Weights are packed once per update as
// [tap][channel group][N][4] (the B operand, K-major), zero where a layer has
// fewer channels than the padded shape: 5 input channels are two groups
// (channels 5..7 zero), 4 input channels are two groups (one zero), 4 output
// channels are an N = 16 tile.  Weights are BF16 values, exact in TF32;
// activations are rounded to TF32 (10-bit mantissa).
constexpr int kTcPix = 128;                             // pixels per tile (the MMA's M)
constexpr int kTcXW = kTcPix + 2;                       // halo row width
constexpr int kTcAPlane = 3 * kTcXW;                    // halo pixels per channel group (3 rows)
constexpr unsigned kTcCols = 32;                        // TMEM columns (N <= 32)

// Shared-memory geometry of a layer shape: CG channel groups of four
// (even: one MMA covers two), N accumulator columns.
template <int CG, int NN> struct TcGeom {
  static_assert(CG % 2 == 0 && (NN == 16 || NN == 32), "padded layer shape");
  static constexpr size_t A_BYTES = (size_t)CG * kTcAPlane * 16;
  static constexpr size_t B_BYTES = (size_t)9 * CG * NN * 16;
  static constexpr size_t SMEM = A_BYTES + B_BYTES + 32;  // + 2 mbarriers, TMEM address, issue flag
};

// Input [B][CINR][H][W] -> output [B][COUT][H][W] (and z for GELU); wtc: the
// packed B operand [9][CG][NN][4].
template <int CG, int NN, int COUT, int CINR, int EPI>
__global__ void __launch_bounds__(128, 1)
    k_conv_tc(const float* __restrict__ in, const float* __restrict__ wtc, const float* __restrict__ bias,
              float* __restrict__ z, float* __restrict__ out, const float* __restrict__ zprev, int B, int H, int W,
              int* __restrict__ status, unsigned long long wait_ns) {
  using G = TcGeom<CG, NN>;
  static_assert(CINR <= 4 * CG && COUT <= NN, "layer does not fit the padded shape");
  extern __shared__ __align__(128) unsigned char smraw[];
  float4* As = reinterpret_cast<float4*>(smraw);
  float4* Bs = reinterpret_cast<float4*>(smraw + G::A_BYTES);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smraw + G::A_BYTES + G::B_BYTES);  // [0] weights, [1] MMAs
  unsigned* slot = reinterpret_cast<unsigned*>(smraw + G::A_BYTES + G::B_BYTES + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t plane = (size_t)H * W;
  const int tx = W / kTcPix, ntiles = tx * H * B;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init_fence();
    // the weights (B operand) once per CTA: one bulk copy, overlapping the first tile's staging
    mbar_expect_tx(&bars[0], (unsigned)G::B_BYTES);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(Bs)),
                 "l"(wtc), "r"((unsigned)G::B_BYTES), "r"(smem_u32(&bars[0]))
                 : "memory");
  }
  if (warp == 0) umma::tmem_alloc(slot, kTcCols);
  // channel c of a group: 4 values of one pixel (zero past the layer's channels)
  auto chan = [&](const float* src, int c0, int j) -> float {
    if constexpr (CINR == 4 * CG) return umma::to_tf32(__ldg(src + (size_t)j * plane));
    else return c0 + j < CINR ? umma::to_tf32(__ldg(src + (size_t)j * plane)) : 0.0f;
  };
  bool ok = true;
  int it = 0;
#pragma unroll 1
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, it++) {
    const int b = tile / (tx * H), rem_t = tile % (tx * H);
    const int y0 = rem_t / tx, x0 = (rem_t % tx) * kTcPix;
    const float* inb = in + (size_t)b * CINR * plane;
    // A: halo tile [cg][halo row][halo pixel][4 channels]; the 128 interior
    // pixels of a row by 16-byte loads along x (4 pixels of each channel)
    for (int q = tid; q < CG * 3 * (kTcPix / 4); q += 128) {
      const int k4 = q % (kTcPix / 4), rr = q / (kTcPix / 4), r = rr % 3, cg = rr / 3;
      const float* src = inb + (size_t)(4 * cg) * plane + (size_t)wrap(y0 + r - 1, H) * W + x0 + 4 * k4;
      float4 c[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        if (CINR == 4 * CG || 4 * cg + j < CINR) {
          const float4 v = __ldg(reinterpret_cast<const float4*>(src + (size_t)j * plane));
          c[j] = make_float4(umma::to_tf32(v.x), umma::to_tf32(v.y), umma::to_tf32(v.z), umma::to_tf32(v.w));
        } else {
          c[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
      }
      float4* dst = As + (size_t)(cg * 3 + r) * kTcXW + 1 + 4 * k4;
      dst[0] = make_float4(c[0].x, c[1].x, c[2].x, c[3].x);
      dst[1] = make_float4(c[0].y, c[1].y, c[2].y, c[3].y);
      dst[2] = make_float4(c[0].z, c[1].z, c[2].z, c[3].z);
      dst[3] = make_float4(c[0].w, c[1].w, c[2].w, c[3].w);
    }
    // the two halo pixels of every row (periodic wrap in x)
    for (int q = tid; q < CG * 3 * 2; q += 128) {
      const int side = q & 1, rr = q >> 1, r = rr % 3, cg = rr / 3;
      const int px = side ? kTcXW - 1 : 0;
      const float* src = inb + (size_t)(4 * cg) * plane + (size_t)wrap(y0 + r - 1, H) * W + wrap(x0 + px - 1, W);
      As[(size_t)(cg * 3 + r) * kTcXW + px] =
          make_float4(chan(src, 4 * cg, 0), chan(src, 4 * cg, 1), chan(src, 4 * cg, 2), chan(src, 4 * cg, 3));
    }
    fence_proxy_async_smem();  // the operands are read by the tensor cores (async proxy)
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const unsigned tmem = *slot;
    if (tid == 0) {
      const bool wok = it > 0 || mbar_wait_bounded(&bars[0], 0, wait_ns);
      if (wok) {
        constexpr uint32_t idesc = umma::instr_desc(umma::kFmtTF32, kTcPix, NN);
        const unsigned a0 = smem_u32(As), b0 = smem_u32(Bs);
#pragma unroll 1
        for (int tap = 0; tap < 9; tap++) {
          const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
          for (int s = 0; s < CG / 2; s++) {  // channel groups 2s, 2s+1: K = 8
            const unsigned aoff = (unsigned)((2 * s * kTcAPlane + (1 + dy) * kTcXW + 1 + dx) * 16);
            const unsigned boff = (unsigned)((tap * CG + 2 * s) * NN * 16);
            umma::mma_tf32(tmem, umma::smem_desc(a0 + aoff, kTcAPlane * 16, 128),
                           umma::smem_desc(b0 + boff, NN * 16, 128), idesc, tap > 0 || s > 0);
          }
        }
        umma::commit(&bars[1]);
      } else {
        atomicExch(status, TARA_ETIMEOUT);
      }
      slot[1] = wok ? 1u : 0u;
    }
    __syncthreads();
    ok = slot[1] != 0;
    if (ok) ok = __syncthreads_and(mbar_wait_bounded(&bars[1], it & 1, wait_ns));
    umma::fence_after_sync();
    if (ok) {
      float acc[32];  // columns NN..31 are not written by the MMAs and are not used
      umma::ld_32x32b_x32(tmem + ((unsigned)(32 * warp) << 16), acc);
      const size_t po = (size_t)y0 * W + x0 + 32 * warp + lane;
#pragma unroll
      for (int co = 0; co < COUT; co++) {
        const float v = acc[co] + (bias ? __ldg(bias + co) : 0.0f);
        const size_t idx = ((size_t)b * COUT + co) * plane + po;
        if constexpr (EPI == EPI_GELU) {
          z[idx] = v;
          out[idx] = gelu(v);
        } else if constexpr (EPI == EPI_LINEAR) {
          out[idx] = v;
        } else {
          out[idx] = v * gelu_d(__ldg(zprev + idx));
        }
      }
    } else if (slot[1]) {
      // the MMAs were issued but did not complete in time: record it and give
      // them a bounded time to finish before their accumulator is released
      if (tid == 0) atomicExch(status, TARA_ETIMEOUT);
      mbar_wait_bounded(&bars[1], it & 1, wait_ns);
    }
    umma::fence_before_sync();
    __syncthreads();  // the accumulator and the A tile are free again
  }
  if (it == 0 || !ok) {
    // the weight copy may still be in flight (no tile, or a failed wait):
    // let it land before the CTA's shared memory is released
    if (tid == 0) mbar_wait_bounded(&bars[0], 0, wait_ns);
    __syncthreads();
  }
  if (warp == 0) umma::tmem_dealloc(*slot, kTcCols);
}

// Tensor-core B operand of a layer W[cout][cin][3][3] (BF16-rounded values
// as FP32), padded to cg channel groups of four and nn columns:
//   forward:        [tap][ci/4][co][ci%4]          (inputs ci, outputs co)
//   input gradient: [8 - tap][co/4][ci][co%4]      (inputs co, outputs ci)
// Every entry of the padded shape is written (zero outside the layer).
__global__ void k_pack_weights_tc(const float* __restrict__ m, int cin, int cout, int cg, int nn, int grad,
                                  float* __restrict__ dst) {
  const int n = 9 * cg * nn * 4;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i % 4, col = (i / 4) % nn, g = (i / (4 * nn)) % cg, t = i / (4 * nn * cg);
    const int k = 4 * g + c;  // input channel of the convolution
    const int ci = grad ? col : k, co = grad ? k : col, tap = grad ? 8 - t : t;
    dst[i] = (ci < cin && co < cout) ? __bfloat162float(__float2bfloat16_rn(m[(co * cin + ci) * 9 + tap])) : 0.0f;
  }
}

// weight (and bias) gradient partials of one 16x16 tile of one sample
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) k_conv_dw(const float* __restrict__ in, const float* __restrict__ dz,
                                                 float* __restrict__ part, int H, int W) {
  constexpr int XS = kPlane + 1;  // odd plane stride: lanes with consecutive cin hit distinct banks
  constexpr int NP = COUT * CIN, NPT = (NP + 255) / 256, NWL = COUT * CIN * 9 + COUT;
  extern __shared__ __align__(16) float sm[];
  float* xs = sm;              // [CIN][18*18 + 1]
  float* ds = sm + CIN * XS;   // [COUT][256]
  const int b = blockIdx.z, y0 = blockIdx.y * kTile, x0 = blockIdx.x * kTile;
  const int tid = threadIdx.x;
  const size_t plane = (size_t)H * W;
  for (int q = tid; q < CIN * kPlane; q += 256) {
    const int c = q / kPlane, r = q % kPlane;
    const int gy = wrap(y0 + r / kHalo - 1, H), gx = wrap(x0 + r % kHalo - 1, W);
    xs[c * XS + r] = __ldg(in + ((size_t)b * CIN + c) * plane + (size_t)gy * W + gx);
  }
  for (int q = tid; q < COUT * 256; q += 256) {
    const int c = q / 256, p = q % 256;
    ds[q] = __ldg(dz + ((size_t)b * COUT + c) * plane + (size_t)(y0 + p / kTile) * W + x0 + p % kTile);
  }
  __syncthreads();
  float acc[NPT][9];
#pragma unroll
  for (int k = 0; k < NPT; k++)
#pragma unroll
    for (int t = 0; t < 9; t++) acc[k][t] = 0.0f;
#pragma unroll 1
  for (int p = 0; p < 256; p++) {
    const int py = p / kTile, px = p % kTile;
#pragma unroll
    for (int k = 0; k < NPT; k++) {
      const int q = tid + k * 256;
      if (q < NP) {
        const int co = q / CIN, ci = q % CIN;
        const float d = ds[co * 256 + p];
        const float* xb = xs + ci * XS + py * kHalo + px;
#pragma unroll
        for (int t = 0; t < 9; t++) acc[k][t] = fmaf(d, xb[(t / 3) * kHalo + t % 3], acc[k][t]);
      }
    }
  }
  const size_t cta = ((size_t)b * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  float* pp = part + cta * NWL;
#pragma unroll
  for (int k = 0; k < NPT; k++) {
    const int q = tid + k * 256;
    if (q < NP)
#pragma unroll
      for (int t = 0; t < 9; t++) pp[q * 9 + t] = acc[k][t];  // (co*CIN + ci)*9 + tap
  }
  if (tid < COUT) {
    float s = 0.0f;
    for (int p = 0; p < 256; p++) s += ds[tid * 256 + p];
    pp[COUT * CIN * 9 + tid] = s;
  }
}

__global__ void k_sum_parts(const float* __restrict__ part, int nct, int nw, float* __restrict__ g) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw; i += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int c = 0; c < nct; c++) s += part[(size_t)c * nw + i];
    g[i] = s;
  }
}

// master W[cout][cin][3][3], b[cout] -> BF16 [cin][9][cout] and mirrored
// [cout][9][cin]; bias rounded to BF16 (kept as FP32)
__global__ void k_pack_weights(const float* __restrict__ m, int cin, int cout, __nv_bfloat16* wf,
                               __nv_bfloat16* wb, float* bias) {
  const int nw = cout * cin * 9;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw + cout; i += gridDim.x * blockDim.x) {
    if (i < nw) {
      const int co = i / (cin * 9), ci = (i / 9) % cin, tap = i % 9;
      const __nv_bfloat16 v = __float2bfloat16_rn(m[i]);
      wf[(ci * 9 + tap) * cout + co] = v;
      wb[(co * 9 + (8 - tap)) * cin + ci] = v;
    } else {
      bias[i] = __bfloat162float(__float2bfloat16_rn(m[i]));  // same offset as in the master vector
    }
  }
}

__global__ void k_mse(const float* __restrict__ o, const float* __restrict__ t, size_t n, float* __restrict__ d,
                      double* __restrict__ acc) {
  __shared__ double red[8];
  double s = 0.0;
  const float sc = 2.0f / (float)n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float e = o[i] - t[i];
    d[i] = sc * e;
    s += (double)e * e;
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) r += red[w];
    atomicAdd(acc, r);
  }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

int layer_params(int l) {
  const CnnLayerDims d = cnn_layer(l);
  return d.cout * d.cin * 9 + d.cout;
}
int layer_offset(int l) {
  int o = 0;
  for (int k = 0; k < l; k++) o += layer_params(k);
  return o;
}

template <int CIN, int COUTT, int COUT, int EPI>
void launch_conv_split(const float* in, const __nv_bfloat16* w, const float* bias, float* z, float* out,
                       const float* zprev, int B, int H, int W, cudaStream_t st) {
  const size_t smem = (size_t)(CIN * kPlane + CIN * 9 * COUT) * sizeof(float);
  auto kern = k_conv<CIN, COUTT, COUT, EPI>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<dim3(W / kTile, H / kTile, B * (COUTT / COUT)), 256, smem, st>>>(in, w, bias, z, out, zprev, H, W);
}
// fewer than ~4 tiles per SM: a quarter of the output channels per CTA
template <int CIN, int COUT, int EPI>
void launch_conv(const float* in, const __nv_bfloat16* w, const float* bias, float* z, float* out,
                 const float* zprev, int B, int H, int W, cudaStream_t st) {
  const int tiles = B * (H / kTile) * (W / kTile);
  if constexpr (COUT == kCnnHid) {
    if (tiles < 600) {
      launch_conv_split<CIN, COUT, COUT / 4, EPI>(in, w, bias, z, out, zprev, B, H, W, st);
      return;
    }
  }
  launch_conv_split<CIN, COUT, COUT, EPI>(in, w, bias, z, out, zprev, B, H, W, st);
}
// Padded tensor-core shape of a convolution with cin inputs and cout
// outputs: channel groups of four (an even number) and accumulator columns.
inline int tc_groups(int cin) { return ((cin + 3) / 4 + 1) / 2 * 2; }
inline int tc_cols(int cout) { return cout <= 16 ? 16 : 32; }

template <int CG, int NN, int COUT, int CINR, int EPI>
void launch_conv_tc(const float* in, const float* wtc, const float* bias, float* z, float* out, const float* zprev,
                    int B, int H, int W, int* status, unsigned long long wait_ns, cudaStream_t st) {
  using G = TcGeom<CG, NN>;
  auto kern = k_conv_tc<CG, NN, COUT, CINR, EPI>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
  // persistent: at most as many CTAs as fit (by shared memory; the kernel's
  // 128 threads leave registers for two), each loading the weights once
  int dev = 0, sms = 148, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  const int per_sm = std::max(1, std::min(2, optin / (int)(G::SMEM + 1024)));
  const int ntiles = (W / kTcPix) * H * B;
  const int grid = std::min(ntiles, per_sm * sms);
  kern<<<grid, 128, G::SMEM, st>>>(in, wtc, bias, z, out, zprev, B, H, W, status, wait_ns);
}
template <int CIN, int COUT>
void launch_dw(const float* in, const float* dz, float* part, float* g, int B, int H, int W, cudaStream_t st) {
  const size_t smem = (size_t)(CIN * (kPlane + 1) + COUT * 256) * sizeof(float);
  auto kern = k_conv_dw<CIN, COUT>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<dim3(W / kTile, H / kTile, B), 256, smem, st>>>(in, dz, part, H, W);
  const int nct = B * (H / kTile) * (W / kTile), nw = COUT * CIN * 9 + COUT;
  k_sum_parts<<<(nw + 255) / 256, 256, 0, st>>>(part, nct, nw, g);
}

}  // namespace

int cnn_num_params() { return layer_offset(kCnnLayers); }

bool Cnn::tc_layer(int) const { return tensor_cores && W % kTcPix == 0; }

int Cnn::alloc(int H_, int W_, int Bmax_) {
  if (H_ % kTile || W_ % kTile || H_ < kTile || W_ < kTile || Bmax_ < 1) {
    set_error("CNN planes must be multiples of 16");
    return TARA_EINVAL;
  }
  H = H_; W = W_; Bmax = Bmax_;
  const size_t np = cnn_num_params(), plane = (size_t)H * W;
  auto am = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
  bool ok = am((void**)&master, np * 4) && am((void**)&grad, np * 4) && am((void**)&adam_m, np * 4) &&
            am((void**)&adam_v, np * 4) && am((void**)&biasbuf, np * 4) && am((void**)&lossacc, sizeof(double));
  for (int l = 0; l < kCnnLayers && ok; l++) {
    const CnnLayerDims d = cnn_layer(l);
    ok = am((void**)&wfwd[l], (size_t)d.cin * 9 * d.cout * 2) && am((void**)&wbwd[l], (size_t)d.cin * 9 * d.cout * 2);
    if (ok && d.gelu) ok = am((void**)&z[l], (size_t)Bmax * d.cout * plane * 4);
    if (ok) ok = am((void**)&a[l], (size_t)Bmax * d.cout * plane * 4);
    bias[l] = biasbuf + layer_offset(l) + d.cout * d.cin * 9;
    if (ok) ok = am((void**)&wtcf[l], (size_t)9 * tc_groups(d.cin) * tc_cols(d.cout) * 16);
    if (ok && l > 0) ok = am((void**)&wtcb[l], (size_t)9 * tc_groups(d.cout) * tc_cols(d.cin) * 16);
  }
  if (ok) ok = am((void**)&status, sizeof(int));
  if (ok) ok = cudaMemset(status, 0, sizeof(int)) == cudaSuccess;
  for (int k = 0; k < 2 && ok; k++) ok = am((void**)&dz[k], (size_t)Bmax * kCnnHid * plane * 4);
  part_elems = (size_t)Bmax * (H / kTile) * (W / kTile) * (kCnnHid * kCnnHid * 9 + kCnnHid);
  if (ok) ok = am((void**)&part, part_elems * 4);
  if (!ok) {
    set_error("cudaMalloc of CNN buffers failed");
    return TARA_ENOMEM;
  }
  cudaMemset(adam_m, 0, np * 4);
  cudaMemset(adam_v, 0, np * 4);
  // the memsets run on the legacy stream, which the closure's non-blocking
  // stream does not wait for: finish them here
  TARA_CUDA_TRY(cudaDeviceSynchronize());
  return TARA_OK;
}

void Cnn::release() {
  for (void* p : {(void*)master, (void*)grad, (void*)adam_m, (void*)adam_v, (void*)biasbuf, (void*)lossacc,
                  (void*)part, (void*)dz[0], (void*)dz[1]})
    if (p) cudaFree(p);
  for (int l = 0; l < kCnnLayers; l++)
    for (void* p : {(void*)wfwd[l], (void*)wbwd[l], (void*)z[l], (void*)a[l], (void*)wtcf[l], (void*)wtcb[l]})
      if (p) cudaFree(p);
  if (status) cudaFree(status);
  *this = Cnn{};
}

int Cnn::refresh(cudaStream_t st) {
  for (int l = 0; l < kCnnLayers; l++) {
    const CnnLayerDims d = cnn_layer(l);
    k_pack_weights<<<64, 256, 0, st>>>(master + layer_offset(l), d.cin, d.cout, wfwd[l], wbwd[l],
                                       biasbuf + layer_offset(l));
    if (wtcf[l])
      k_pack_weights_tc<<<36, 256, 0, st>>>(master + layer_offset(l), d.cin, d.cout, tc_groups(d.cin),
                                            tc_cols(d.cout), 0, wtcf[l]);
    if (wtcb[l])
      k_pack_weights_tc<<<36, 256, 0, st>>>(master + layer_offset(l), d.cin, d.cout, tc_groups(d.cout),
                                            tc_cols(d.cin), 1, wtcb[l]);
  }
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

int Cnn::forward(const float* in, int B, bool, cudaStream_t st) {
  if (B < 1 || B > Bmax) { set_error("batch larger than the CNN buffers"); return TARA_EINVAL; }
  if (tc_layer(0)) {
    // all four layers on the tensor cores (padded shapes: 5 inputs in two
    // channel groups, 4 outputs in an N = 16 tile)
    launch_conv_tc<2, 32, kCnnHid, kCnnIn, EPI_GELU>(in, wtcf[0], bias[0], z[0], a[0], nullptr, B, H, W, status,
                                                      wait_ns, st);
    for (int l = 1; l <= 2; l++)
      launch_conv_tc<8, 32, kCnnHid, kCnnHid, EPI_GELU>(a[l - 1], wtcf[l], bias[l], z[l], a[l], nullptr, B, H, W,
                                                         status, wait_ns, st);
    launch_conv_tc<8, 16, kCnnOut, kCnnHid, EPI_LINEAR>(a[2], wtcf[3], bias[3], nullptr, a[3], nullptr, B, H, W,
                                                         status, wait_ns, st);
  } else {
    launch_conv<kCnnIn, kCnnHid, EPI_GELU>(in, wfwd[0], bias[0], z[0], a[0], nullptr, B, H, W, st);
    for (int l = 1; l <= 2; l++)
      launch_conv<kCnnHid, kCnnHid, EPI_GELU>(a[l - 1], wfwd[l], bias[l], z[l], a[l], nullptr, B, H, W, st);
    launch_conv<kCnnHid, kCnnOut, EPI_LINEAR>(a[2], wfwd[3], bias[3], nullptr, a[3], nullptr, B, H, W, st);
  }
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

int Cnn::backward(const float* in, const float* dout, int B, cudaStream_t st) {
  if (B < 1 || B > Bmax) { set_error("batch larger than the CNN buffers"); return TARA_EINVAL; }
  const bool tc = tc_layer(0);
  // layer 3 (linear): dout is the gradient of its pre-activation
  launch_dw<kCnnHid, kCnnOut>(a[2], dout, part, grad + layer_offset(3), B, H, W, st);
  if (tc)
    launch_conv_tc<2, 32, kCnnHid, kCnnOut, EPI_GELUGRAD>(dout, wtcb[3], nullptr, nullptr, dz[0], z[2], B, H, W,
                                                           status, wait_ns, st);
  else
    launch_conv<kCnnOut, kCnnHid, EPI_GELUGRAD>(dout, wbwd[3], nullptr, nullptr, dz[0], z[2], B, H, W, st);
  launch_dw<kCnnHid, kCnnHid>(a[1], dz[0], part, grad + layer_offset(2), B, H, W, st);
  if (tc)
    launch_conv_tc<8, 32, kCnnHid, kCnnHid, EPI_GELUGRAD>(dz[0], wtcb[2], nullptr, nullptr, dz[1], z[1], B, H, W,
                                                           status, wait_ns, st);
  else
    launch_conv<kCnnHid, kCnnHid, EPI_GELUGRAD>(dz[0], wbwd[2], nullptr, nullptr, dz[1], z[1], B, H, W, st);
  launch_dw<kCnnHid, kCnnHid>(a[0], dz[1], part, grad + layer_offset(1), B, H, W, st);
  if (tc)
    launch_conv_tc<8, 32, kCnnHid, kCnnHid, EPI_GELUGRAD>(dz[1], wtcb[1], nullptr, nullptr, dz[0], z[0], B, H, W,
                                                           status, wait_ns, st);
  else
    launch_conv<kCnnHid, kCnnHid, EPI_GELUGRAD>(dz[1], wbwd[1], nullptr, nullptr, dz[0], z[0], B, H, W, st);
  launch_dw<kCnnIn, kCnnHid>(in, dz[0], part, grad + layer_offset(0), B, H, W, st);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

int Cnn::check(cudaStream_t st) {
  int v = 0;
  TARA_CUDA_TRY(cudaMemcpyAsync(&v, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  TARA_CUDA_TRY(cudaStreamSynchronize(st));
  if (v != TARA_OK) {
    TARA_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), st));
    set_error("a bounded wait of a tensor-core convolution ran out");
  }
  return v;
}

int Cnn::mse(const float* target, int B, cudaStream_t st) {
  const size_t n = (size_t)B * kCnnOut * H * W;
  k_mse<<<296, 256, 0, st>>>(a[3], target, n, dz[1], lossacc);
  TARA_CUDA_TRY(cudaGetLastError());
  return TARA_OK;
}

int Cnn::adam(float lr, float b1, float b2, float eps, cudaStream_t st) {
  adam_t++;
  const float c1 = 1.0f - (float)std::pow((double)b1, (double)adam_t);
  const float c2 = 1.0f - (float)std::pow((double)b2, (double)adam_t);
  const int n = cnn_num_params();
  k_adam<<<(n + 255) / 256, 256, 0, st>>>(master, grad, adam_m, adam_v, n, lr, b1, b2, eps, c1, c2);
  TARA_CUDA_TRY(cudaGetLastError());
  return refresh(st);
}

}  // namespace tara
