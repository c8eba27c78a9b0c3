// hg_mlp.cu -- training and batched inference of the learned shock sensor (no reference counterpart).
//
// The network of hg_sensor.cuh (16 -> 32 -> 32 -> 1, tanh hidden layers, sigmoid output) is
// trained on the GPU by these kernels: weighted binary cross-entropy on the logit,
//   L = sum_i w_i [softplus(z_i) - t_i z_i] / B,
// gradients by back-propagation (one thread per sample for the forward/backward sweep, then one
// thread per parameter reducing over the block's samples from shared memory), and Adam.
#include "../../include/horses_gpu.h"
#include "hg_sensor.cuh"

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

using namespace hg;
static_assert(MLP_PARAMS == HG_MLP_PARAMS && MLP_IN == HG_SENSOR_FEATURES, "network layout and C ABI agree");

namespace {

constexpr int TB = 128;            // samples per block in the gradient kernel
constexpr int LD = TB + 1;         // padded leading dimension of the [feature][sample] tiles
constexpr size_t GRAD_SMEM = sizeof(float) * (size_t(MLP_IN + 4 * MLP_H) * LD + TB);

__device__ __forceinline__ void mlp_forward_one(const float* __restrict__ W, const float* x, float* h1, float* h2,
                                                float& z) {
#pragma unroll 4
  for (int o = 0; o < MLP_H; ++o) {
    float a = __ldg(W + MLP_B1 + o);
#pragma unroll
    for (int q = 0; q < MLP_IN; ++q) a += __ldg(W + MLP_W1 + o * MLP_IN + q) * x[q];
    h1[o] = tanhf(a);
  }
#pragma unroll 4
  for (int o = 0; o < MLP_H; ++o) {
    float a = __ldg(W + MLP_B2 + o);
#pragma unroll
    for (int q = 0; q < MLP_H; ++q) a += __ldg(W + MLP_W2 + o * MLP_H + q) * h1[q];
    h2[o] = tanhf(a);
  }
  float a = __ldg(W + MLP_B3);
#pragma unroll
  for (int q = 0; q < MLP_H; ++q) a += __ldg(W + MLP_W3 + q) * h2[q];
  z = a;
}

__global__ void mlp_forward_kernel(const float* __restrict__ W, const float* __restrict__ X, int64_t n, float* y) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[MLP_IN], h1[MLP_H], h2[MLP_H], z;
#pragma unroll
  for (int q = 0; q < MLP_IN; ++q) x[q] = X[i * MLP_IN + q];
  mlp_forward_one(W, x, h1, h2, z);
  y[i] = 1.0f / (1.0f + expf(-z));
}

// Block b: samples k in [b*TB, b*TB + TB) of the (optionally permuted) sample list.  Writes its share
// of the gradient (scaled by inv_batch) to gpart[b][MLP_PARAMS] and of the loss (unscaled) to lpart[b];
// the sums over blocks run in block order afterwards (mlp_adam_kernel, mlp_reduce_kernel), so that
// training gives the same bits on every run (atomic adds would sum in arrival order).
__global__ void __launch_bounds__(TB) mlp_grad_kernel(const float* __restrict__ W, const float* __restrict__ X,
                                                      const float* __restrict__ t, const float* __restrict__ w,
                                                      const int* __restrict__ idx, int64_t n, float inv_batch,
                                                      float* gpart, double* lpart) {
  extern __shared__ float sm[];
  float* sx = sm;                       // [16][LD]
  float* sh1 = sx + MLP_IN * LD;        // [32][LD]
  float* sh2 = sh1 + MLP_H * LD;        // [32][LD]
  float* sa1 = sh2 + MLP_H * LD;        // [32][LD]  dL/d(pre-activation 1)
  float* sa2 = sa1 + MLP_H * LD;        // [32][LD]  dL/d(pre-activation 2)
  float* sdz = sa2 + MLP_H * LD;        // [TB]      dL/dz
  const int r = threadIdx.x;
  const int64_t k = int64_t(blockIdx.x) * TB + r;
  float lossv = 0.0f;
  if (k < n) {
    const int64_t s = idx ? int64_t(idx[k]) : k;
    float x[MLP_IN], h1[MLP_H], h2[MLP_H], z;
#pragma unroll
    for (int q = 0; q < MLP_IN; ++q) { x[q] = X[s * MLP_IN + q]; sx[q * LD + r] = x[q]; }
    mlp_forward_one(W, x, h1, h2, z);
    const float tt = t[s], ww = w ? w[s] : 1.0f;
    const float y = 1.0f / (1.0f + expf(-z));
    lossv = ww * (fmaxf(z, 0.0f) - z * tt + log1pf(expf(-fabsf(z))));
    const float dz = ww * (y - tt) * inv_batch;
    sdz[r] = dz;
    float a2[MLP_H];
#pragma unroll
    for (int o = 0; o < MLP_H; ++o) {
      a2[o] = dz * __ldg(W + MLP_W3 + o) * (1.0f - h2[o] * h2[o]);
      sh2[o * LD + r] = h2[o];
      sa2[o * LD + r] = a2[o];
    }
#pragma unroll 4
    for (int q = 0; q < MLP_H; ++q) {
      float d = 0.0f;
#pragma unroll
      for (int o = 0; o < MLP_H; ++o) d += __ldg(W + MLP_W2 + o * MLP_H + q) * a2[o];
      sa1[q * LD + r] = d * (1.0f - h1[q] * h1[q]);
      sh1[q * LD + r] = h1[q];
    }
  } else {
    for (int q = 0; q < MLP_IN; ++q) sx[q * LD + r] = 0.0f;
    for (int o = 0; o < MLP_H; ++o) { sh1[o * LD + r] = 0.0f; sh2[o * LD + r] = 0.0f; sa1[o * LD + r] = 0.0f; sa2[o * LD + r] = 0.0f; }
    sdz[r] = 0.0f;
  }
  __syncthreads();
  for (int p = r; p < MLP_PARAMS; p += TB) {
    float acc = 0.0f;
    if (p < MLP_B1) {
      const int o = p / MLP_IN, q = p % MLP_IN;
      for (int j = 0; j < TB; ++j) acc += sa1[o * LD + j] * sx[q * LD + j];
    } else if (p < MLP_W2) {
      const int o = p - MLP_B1;
      for (int j = 0; j < TB; ++j) acc += sa1[o * LD + j];
    } else if (p < MLP_B2) {
      const int o = (p - MLP_W2) / MLP_H, q = (p - MLP_W2) % MLP_H;
      for (int j = 0; j < TB; ++j) acc += sa2[o * LD + j] * sh1[q * LD + j];
    } else if (p < MLP_W3) {
      const int o = p - MLP_B2;
      for (int j = 0; j < TB; ++j) acc += sa2[o * LD + j];
    } else if (p < MLP_B3) {
      const int q = p - MLP_W3;
      for (int j = 0; j < TB; ++j) acc += sdz[j] * sh2[q * LD + j];
    } else {
      for (int j = 0; j < TB; ++j) acc += sdz[j];
    }
    gpart[size_t(blockIdx.x) * MLP_PARAMS + p] = acc;
  }
  __shared__ double wl[TB / 32];
  for (int off = 16; off > 0; off >>= 1) lossv += __shfl_xor_sync(0xffffffffu, lossv, off);
  if ((r & 31) == 0) wl[r >> 5] = double(lossv);
  __syncthreads();
  if (r == 0) {
    double l = 0.0;
    for (int k = 0; k < TB / 32; ++k) l += wl[k];
    lpart[blockIdx.x] = l;
  }
}

// The block partials of one gradient evaluation summed in block order: grad[p], and the loss into
// *loss (added to it).
__global__ void mlp_reduce_kernel(const float* gpart, const double* lpart, int nblk, float* grad, double* loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < MLP_PARAMS) {
    float g = 0.0f;
    for (int b = 0; b < nblk; ++b) g += gpart[size_t(b) * MLP_PARAMS + p];
    grad[p] = g;
  }
  if (p == 0) {
    double l = *loss;
    for (int b = 0; b < nblk; ++b) l += lpart[b];
    *loss = l;
  }
}

__global__ void mlp_adam_kernel(float* W, const float* gpart, const double* lpart, int nblk, double* loss, float* m,
                                float* v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) {   // the batch's loss, in block order
    double l = *loss;
    for (int b = 0; b < nblk; ++b) l += lpart[b];
    *loss = l;
  }
  if (p >= n) return;
  float gg = 0.0f;
  for (int b = 0; b < nblk; ++b) gg += gpart[size_t(b) * n + p];
  const float mm = b1 * m[p] + (1.0f - b1) * gg;
  const float vv = b2 * v[p] + (1.0f - b2) * gg * gg;
  m[p] = mm;
  v[p] = vv;
  W[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

#define MLP_CUDA(call)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  explicit DevBuf(size_t bytes) { MLP_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16))); }
  ~DevBuf() { if (p) cudaFree(p); }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

void grad_smem_attr() {
  static bool done = false;
  if (!done) {
    MLP_CUDA(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(GRAD_SMEM)));
    done = true;
  }
}

}  // namespace

extern "C" int hg_mlp_forward(const float* params, const float* X, int64_t n, float* y) {
  try {
    if (!params || !X || !y || n <= 0) return 1;
    DevBuf dW(MLP_PARAMS * sizeof(float)), dX(size_t(n) * MLP_IN * sizeof(float)), dy(size_t(n) * sizeof(float));
    MLP_CUDA(cudaMemcpy(dW.p, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(dX.p, X, size_t(n) * MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    mlp_forward_kernel<<<unsigned((n + 255) / 256), 256>>>(dW.as<float>(), dX.as<float>(), n, dy.as<float>());
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaMemcpy(y, dy.p, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
  } catch (const std::exception&) { return 3; }
}

extern "C" int hg_mlp_grad(const float* params, const float* X, const float* t, const float* w, int64_t n, double* loss,
                           float* grad) {
  try {
    if (!params || !X || !t || !loss || !grad || n <= 0) return 1;
    grad_smem_attr();
    DevBuf dW(MLP_PARAMS * sizeof(float)), dX(size_t(n) * MLP_IN * sizeof(float)), dt(size_t(n) * sizeof(float));
    const int nblk = int((n + TB - 1) / TB);
    DevBuf dw(size_t(w ? n : 1) * sizeof(float)), dg(MLP_PARAMS * sizeof(float)), dl(sizeof(double));
    DevBuf gpart(size_t(nblk) * MLP_PARAMS * sizeof(float)), lpart(size_t(nblk) * sizeof(double));
    MLP_CUDA(cudaMemcpy(dW.p, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(dX.p, X, size_t(n) * MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(dt.p, t, size_t(n) * sizeof(float), cudaMemcpyHostToDevice));
    if (w) MLP_CUDA(cudaMemcpy(dw.p, w, size_t(n) * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemset(dl.p, 0, sizeof(double)));
    mlp_grad_kernel<<<unsigned(nblk), TB, GRAD_SMEM>>>(dW.as<float>(), dX.as<float>(), dt.as<float>(),
                                                       w ? dw.as<float>() : nullptr, nullptr, n, 1.0f / float(n),
                                                       gpart.as<float>(), lpart.as<double>());
    mlp_reduce_kernel<<<(MLP_PARAMS + 255) / 256, 256>>>(gpart.as<float>(), lpart.as<double>(), nblk, dg.as<float>(),
                                                         dl.as<double>());
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaMemcpy(grad, dg.p, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost));
    double l = 0.0;
    MLP_CUDA(cudaMemcpy(&l, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
    *loss = l / double(n);
    return 0;
  } catch (const std::exception&) { return 3; }
}

extern "C" int hg_mlp_train(float* params, const float* X, const float* t, const float* w, int64_t n, int32_t epochs,
                            int32_t batch, double lr, uint64_t seed, double* epoch_loss) {
  try {
    if (!params || !X || !t || n <= 0 || n > INT32_MAX || epochs <= 0 || batch <= 0) return 1;
    grad_smem_attr();
    DevBuf dW(MLP_PARAMS * sizeof(float)), dX(size_t(n) * MLP_IN * sizeof(float)), dt(size_t(n) * sizeof(float));
    const int nblk_max = int((std::min<int64_t>(batch, n) + TB - 1) / TB);
    DevBuf dw(size_t(w ? n : 1) * sizeof(float)), dm(MLP_PARAMS * sizeof(float));
    DevBuf dv(MLP_PARAMS * sizeof(float)), dl(sizeof(double)), didx(size_t(n) * sizeof(int));
    DevBuf gpart(size_t(nblk_max) * MLP_PARAMS * sizeof(float)), lpart(size_t(nblk_max) * sizeof(double));
    MLP_CUDA(cudaMemcpy(dW.p, params, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(dX.p, X, size_t(n) * MLP_IN * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(dt.p, t, size_t(n) * sizeof(float), cudaMemcpyHostToDevice));
    if (w) MLP_CUDA(cudaMemcpy(dw.p, w, size_t(n) * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemset(dm.p, 0, MLP_PARAMS * sizeof(float)));
    MLP_CUDA(cudaMemset(dv.p, 0, MLP_PARAMS * sizeof(float)));
    std::vector<int> perm(static_cast<size_t>(n));
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int64_t step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
      std::shuffle(perm.begin(), perm.end(), rng);
      MLP_CUDA(cudaMemcpy(didx.p, perm.data(), size_t(n) * sizeof(int), cudaMemcpyHostToDevice));
      MLP_CUDA(cudaMemset(dl.p, 0, sizeof(double)));
      for (int64_t b0 = 0; b0 < n; b0 += batch) {
        const int64_t bs = std::min<int64_t>(batch, n - b0);
        const int nblk = int((bs + TB - 1) / TB);
        mlp_grad_kernel<<<unsigned(nblk), TB, GRAD_SMEM>>>(
            dW.as<float>(), dX.as<float>(), dt.as<float>(), w ? dw.as<float>() : nullptr, didx.as<int>() + b0, bs,
            1.0f / float(bs), gpart.as<float>(), lpart.as<double>());
        ++step;
        const float c1 = 1.0f - std::pow(b1, float(step)), c2 = 1.0f - std::pow(b2, float(step));
        mlp_adam_kernel<<<(MLP_PARAMS + 255) / 256, 256>>>(dW.as<float>(), gpart.as<float>(), lpart.as<double>(), nblk,
                                                            dl.as<double>(), dm.as<float>(), dv.as<float>(), MLP_PARAMS,
                                                            float(lr), b1, b2, eps, c1, c2);
      }
      MLP_CUDA(cudaGetLastError());
      double l = 0.0;
      MLP_CUDA(cudaMemcpy(&l, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
      if (epoch_loss) epoch_loss[ep] = l / double(n);
    }
    MLP_CUDA(cudaMemcpy(params, dW.p, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost));
    return 0;
  } catch (const std::exception&) { return 3; }
}
