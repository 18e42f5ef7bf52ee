// The closure CNN: 4 periodic 3x3 convolutions, channels
// 5 -> 32 -> 32 -> 32 -> 4, GELU after the first three.  Weights are kept as
// FP32 masters (the optimiser's copy) and used rounded to BF16; accumulation
// is FP32.  Every convolution (forward and input gradient) runs on the
// tensor cores (tcgen05 MMAs, TF32 activations) when the plane width is a
// multiple of 128, unless tensor_cores is 0; then, and for the weight
// gradients, CUDA cores with FP32 activations.  Hand-written forward, input-gradient and weight-gradient
// kernels; Adam on the masters.
//
// Tensors are [B][C][H][W] FP32 (H, W multiples of 16).  Flat parameter
// vector: per layer W[cout][cin][3][3] then b[cout].
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <vector>

namespace tara {

constexpr int kCnnLayers = 4;
constexpr int kCnnIn = 5, kCnnHid = 32, kCnnOut = 4;

struct CnnLayerDims { int cin, cout; bool gelu; };
inline CnnLayerDims cnn_layer(int l) {
  const int ci[kCnnLayers] = {kCnnIn, kCnnHid, kCnnHid, kCnnHid};
  const int co[kCnnLayers] = {kCnnHid, kCnnHid, kCnnHid, kCnnOut};
  return CnnLayerDims{ci[l], co[l], l < kCnnLayers - 1};
}
int cnn_num_params();

struct Cnn {
  int H = 0, W = 0, Bmax = 0;
  float* master = nullptr;          // flat FP32 parameters
  float* grad = nullptr;            // flat FP32 gradient
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  __nv_bfloat16* wfwd[kCnnLayers] = {};   // [cin][9][cout]
  __nv_bfloat16* wbwd[kCnnLayers] = {};   // [cout][9][cin], taps mirrored
  float* bias[kCnnLayers] = {};           // views into a BF16-rounded FP32 copy
  float* biasbuf = nullptr;
  float* z[kCnnLayers] = {};              // pre-activations (training)
  float* a[kCnnLayers] = {};              // layer outputs
  float* dz[2] = {};                      // ping-pong gradients w.r.t. pre-activations
  float* part = nullptr;                  // per-CTA weight-gradient partials
  size_t part_elems = 0;
  // tensor cores (tcgen05, TF32 activations) for the convolutions; 0: every
  // convolution on CUDA cores with FP32 activations (the reference of the
  // tensor-core path)
  int tensor_cores = 1;
  float* wtcf[kCnnLayers] = {};           // tensor-core B operands of the forward convolutions
  float* wtcb[kCnnLayers] = {};           // and of the input-gradient convolutions (layers 1..3)
  int* status = nullptr;                  // device word: TARA_ETIMEOUT when a bounded wait ran out
  unsigned long long wait_ns = 1000000000ull;
  bool tc_layer(int l) const;             // the convolutions run on the tensor cores
  double* lossacc = nullptr;
  long long adam_t = 0;
  int alloc(int H, int W, int Bmax);
  void release();
  // master -> BF16 forward/backward layouts (after every change of the masters)
  int refresh(cudaStream_t st);
  // out = net(in), in [B][5][H][W] -> a[3] = [B][4][H][W]
  int forward(const float* in, int B, bool keep, cudaStream_t st);
  // gradient of sum over out of dout*out w.r.t. the parameters into grad
  int backward(const float* in, const float* dout, int B, cudaStream_t st);
  // MSE of a[3] against target: dout = 2 (out - target)/n into dz[1] (reused
  // as the output gradient), the loss sum accumulated in lossacc
  int mse(const float* target, int B, cudaStream_t st);
  int adam(float lr, float b1, float b2, float eps, cudaStream_t st);
  // TARA_ETIMEOUT if a tensor-core kernel's bounded wait ran out since the
  // last call (synchronises st; clears the word)
  int check(cudaStream_t st);
  float* out() const { return a[kCnnLayers - 1]; }
};

}  // namespace tara
