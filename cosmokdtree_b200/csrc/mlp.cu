// mlp.cu -- the learned k-th-neighbour distance bound.
//
// A 12 -> 64 -> 64 -> 1 ReLU network with BF16 weights and FP32 arithmetic
// predicts, from cheap features of the query's leaf and its ancestors, the
// base-2 logarithm of the distance to the query's k-th neighbour.  Training
// (forward, backward, Adam) and inference are hand-written kernels below; the
// bounded kNN search that consumes the prediction lives in knn.cu.  Nothing here
// affects results: the bounded search reruns every query whose predicted radius
// holds fewer than k points with the plain unbounded search.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ckd_traverse.cuh"
#include "ckd_mlp.cuh"

namespace ckd {
namespace {

// ---------------------------------------------------------------- inference
// Network output z (normalised units) for normalised features xh, with the
// weights as FP32 values in shared memory (W1 row-major [h][f], W2 [i][j]).
__device__ __forceinline__ float mlp_eval(const float* __restrict__ W, const float (&xh)[kMlpF]) {
  float h1[kMlpH];
#pragma unroll
  for (int j = 0; j < kMlpH; ++j) {
    float a = W[kB1 + j];
#pragma unroll
    for (int f = 0; f < kMlpF; ++f) a = fmaf(W[kW1 + j * kMlpF + f], xh[f], a);
    h1[j] = fmaxf(a, 0.0f);
  }
  float z = W[kB3];
#pragma unroll 4
  for (int i = 0; i < kMlpH; ++i) {
    const float4* row = reinterpret_cast<const float4*>(W + kW2 + i * kMlpH);
    float a = W[kB2 + i];
#pragma unroll
    for (int j4 = 0; j4 < kMlpH / 4; ++j4) {
      float4 w = row[j4];
      a = fmaf(w.x, h1[4 * j4], a);
      a = fmaf(w.y, h1[4 * j4 + 1], a);
      a = fmaf(w.z, h1[4 * j4 + 2], a);
      a = fmaf(w.w, h1[4 * j4 + 3], a);
    }
    z = fmaf(W[kW3 + i], fmaxf(a, 0.0f), z);
  }
  return z;
}

// BF16 weights -> FP32 in shared memory (kW2 is a multiple of 4 floats, so the
// W2 rows are 16-byte aligned for the float4 reads in mlp_eval)
__device__ __forceinline__ void load_weights(const __nv_bfloat16* __restrict__ wb, float* W) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) W[i] = __bfloat162float(wb[i]);
  __syncthreads();
}

__device__ __forceinline__ void normalise(const MlpNorm& nm, const float (&f)[kMlpF],
                                          float (&xh)[kMlpF]) {
#pragma unroll
  for (int j = 0; j < kMlpF; ++j) xh[j] = (f[j] - nm.mu[j]) * nm.isg[j];
}

constexpr int kWSmem = (kMlpParams + 3) & ~3;

template <int D>
__global__ void __launch_bounds__(256) k_features(TreeView tv, const double* __restrict__ Q,
                                                  int64_t nq, int k, float* __restrict__ feat) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  double q[D];
#pragma unroll
  for (int j = 0; j < D; ++j) q[j] = Q[i * D + j];
  float f[kMlpF];
  leaf_features<D>(tv, q, locate_leaf<D>(tv.meta, q), k, f);
#pragma unroll
  for (int j = 0; j < kMlpF; ++j) feat[i * kMlpF + j] = f[j];
}

__global__ void __launch_bounds__(128) k_mlp_forward(const __nv_bfloat16* __restrict__ wb,
                                                     MlpNorm nm, const float* __restrict__ feat,
                                                     int64_t n, float* __restrict__ y) {
  __shared__ __align__(16) float W[kWSmem];
  load_weights(wb, W);
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float f[kMlpF], xh[kMlpF];
#pragma unroll
  for (int j = 0; j < kMlpF; ++j) f[j] = feat[i * kMlpF + j];
  normalise(nm, f, xh);
  y[i] = nm.y_mu + nm.y_sigma * mlp_eval(W, xh);
}

// Predicted squared radius r2[q] = 2^(2 (y + margin)) of every query, queries
// visited in leaf order (order[slot] = query, qleaf[query] = its leaf).
template <int D>
__global__ void __launch_bounds__(128) k_mlp_radius(TreeView tv, const __nv_bfloat16* __restrict__ wb,
                                                    MlpNorm nm, const double* __restrict__ Q,
                                                    const int32_t* __restrict__ order,
                                                    const int32_t* __restrict__ qleaf, int64_t nq,
                                                    int k, double* __restrict__ r2) {
  __shared__ __align__(16) float W[kWSmem];
  load_weights(wb, W);
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nq;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t qi = order ? (int64_t)order[s] : s;
    double q[D];
#pragma unroll
    for (int j = 0; j < D; ++j) q[j] = Q[qi * D + j];
    const int32_t leaf = qleaf ? qleaf[qi] : locate_leaf<D>(tv.meta, q);
    float f[kMlpF], xh[kMlpF];
    leaf_features<D>(tv, q, leaf, k, f);
    normalise(nm, f, xh);
    const float y = nm.y_mu + nm.y_sigma * mlp_eval(W, xh) + nm.margin;
    // exp2 of a double keeps the radius meaningful beyond the FP32 range
    double rr = exp2(2.0 * (double)y);
    r2[qi] = isfinite(rr) ? rr : CKD_HUGE;
  }
}

// ----------------------------------------------------------------- training
// Gradient of the mean squared error of the normalised prediction,
//   loss = (1/n) sum_s (z_s - (t_s - y_mu) / y_sigma)^2,
// with respect to the FP32 master weights, evaluated at their BF16 values
// (the forward pass uses the BF16 weights).  One thread per sample in a tile of
// 128; per-sample activations live in shared memory; each thread accumulates a
// fixed set of gradient entries in registers across the tiles it visits and adds
// them to g once.  `scale` = 2 / (number of samples in the step).
constexpr int kTile = 128;
constexpr int kRow = kMlpH + 1;  // padded activation row
constexpr size_t kGradSmem =
    sizeof(float) * ((size_t)kWSmem + (size_t)kTile * (kMlpF + 1) + 2 * (size_t)kTile * kRow + kTile);

__global__ void __launch_bounds__(kTile) k_mlp_grad(const __nv_bfloat16* __restrict__ wb, MlpNorm nm,
                                                    const float* __restrict__ feat,
                                                    const float* __restrict__ target, int64_t n,
                                                    float scale, float* __restrict__ g,
                                                    double* __restrict__ loss) {
  extern __shared__ __align__(16) float sm[];
  float* W = sm;
  float* X = W + kWSmem;                  // [kTile][kMlpF + 1]
  float* H1 = X + kTile * (kMlpF + 1);    // [kTile][kRow]  h1, later dL/da1
  float* H2 = H1 + kTile * kRow;          // [kTile][kRow]  h2, later dL/da2
  float* DZ = H2 + kTile * kRow;          // [kTile]
  load_weights(wb, W);
  const int t = threadIdx.x;
  // gradient entries owned by this thread
  const int i0 = (t >> 3) * 4, j0 = (t & 7) * 8;     // dW2[i0..i0+3][j0..j0+7]
  const int h1r = t >> 1, f0 = (t & 1) * 6;           // dW1[h1r][f0..f0+5]
  float gW2[4][8], gW1[6], gB2 = 0.f, gB1 = 0.f, gW3 = 0.f, gB3 = 0.f;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) gW2[a][b] = 0.f;
#pragma unroll
  for (int a = 0; a < 6; ++a) gW1[a] = 0.f;
  double lsum = 0.0;

  for (int64_t base = (int64_t)blockIdx.x * kTile; base < n; base += (int64_t)gridDim.x * kTile) {
    // ---- forward, one sample per thread
    {
      const int64_t s = base + t;
      const bool ok = s < n;
      float f[kMlpF], xh[kMlpF];
#pragma unroll
      for (int j = 0; j < kMlpF; ++j) f[j] = ok ? feat[s * kMlpF + j] : 0.0f;
      normalise(nm, f, xh);
#pragma unroll
      for (int j = 0; j < kMlpF; ++j) X[t * (kMlpF + 1) + j] = ok ? xh[j] : 0.0f;
      float h1[kMlpH];
#pragma unroll
      for (int j = 0; j < kMlpH; ++j) {
        float a = W[kB1 + j];
#pragma unroll
        for (int ff = 0; ff < kMlpF; ++ff) a = fmaf(W[kW1 + j * kMlpF + ff], xh[ff], a);
        h1[j] = ok ? fmaxf(a, 0.0f) : 0.0f;
        H1[t * kRow + j] = h1[j];
      }
      float z = W[kB3];
      for (int i = 0; i < kMlpH; ++i) {
        const float4* row = reinterpret_cast<const float4*>(W + kW2 + i * kMlpH);
        float a = W[kB2 + i];
#pragma unroll
        for (int j4 = 0; j4 < kMlpH / 4; ++j4) {
          float4 w = row[j4];
          a = fmaf(w.x, h1[4 * j4], a);
          a = fmaf(w.y, h1[4 * j4 + 1], a);
          a = fmaf(w.z, h1[4 * j4 + 2], a);
          a = fmaf(w.w, h1[4 * j4 + 3], a);
        }
        float h2 = ok ? fmaxf(a, 0.0f) : 0.0f;
        H2[t * kRow + i] = h2;
        z = fmaf(W[kW3 + i], h2, z);
      }
      float e = ok ? z - (target[s] - nm.y_mu) / nm.y_sigma : 0.0f;
      lsum += (double)e * e;
      DZ[t] = scale * e;
    }
    __syncthreads();
    // ---- output layer
    if (t < kMlpH) {
      float a = 0.f;
      for (int s = 0; s < kTile; ++s) a = fmaf(DZ[s], H2[s * kRow + t], a);
      gW3 += a;
    } else if (t == kMlpH) {
      float a = 0.f;
      for (int s = 0; s < kTile; ++s) a += DZ[s];
      gB3 += a;
    }
    __syncthreads();
    // ---- dL/da2 = dz * W3 where h2 > 0
    {
      const float dz = DZ[t];
      for (int i = 0; i < kMlpH; ++i) {
        float h = H2[t * kRow + i];
        H2[t * kRow + i] = h > 0.0f ? dz * W[kW3 + i] : 0.0f;
      }
    }
    __syncthreads();
    // ---- dW2 += da2^T h1, db2
    for (int s = 0; s < kTile; ++s) {
      float a[4], b[8];
#pragma unroll
      for (int r = 0; r < 4; ++r) a[r] = H2[s * kRow + i0 + r];
#pragma unroll
      for (int c = 0; c < 8; ++c) b[c] = H1[s * kRow + j0 + c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) gW2[r][c] = fmaf(a[r], b[c], gW2[r][c]);
    }
    if (t < kMlpH) {
      float a = 0.f;
      for (int s = 0; s < kTile; ++s) a += H2[s * kRow + t];
      gB2 += a;
    }
    // ---- dL/da1 = (W2^T da2) where h1 > 0, computed per sample
    float acc[kMlpH];
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) acc[j] = 0.f;
    for (int i = 0; i < kMlpH; ++i) {
      const float d = H2[t * kRow + i];
      const float4* row = reinterpret_cast<const float4*>(W + kW2 + i * kMlpH);
#pragma unroll
      for (int j4 = 0; j4 < kMlpH / 4; ++j4) {
        float4 w = row[j4];
        acc[4 * j4] = fmaf(d, w.x, acc[4 * j4]);
        acc[4 * j4 + 1] = fmaf(d, w.y, acc[4 * j4 + 1]);
        acc[4 * j4 + 2] = fmaf(d, w.z, acc[4 * j4 + 2]);
        acc[4 * j4 + 3] = fmaf(d, w.w, acc[4 * j4 + 3]);
      }
    }
    __syncthreads();  // every thread has read H1 for dW2
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) {
      float h = H1[t * kRow + j];
      H1[t * kRow + j] = h > 0.0f ? acc[j] : 0.0f;
    }
    __syncthreads();
    // ---- dW1 += da1^T x, db1
    for (int s = 0; s < kTile; ++s) {
      const float d = H1[s * kRow + h1r];
#pragma unroll
      for (int c = 0; c < 6; ++c) gW1[c] = fmaf(d, X[s * (kMlpF + 1) + f0 + c], gW1[c]);
    }
    if (t < kMlpH) {
      float a = 0.f;
      for (int s = 0; s < kTile; ++s) a += H1[s * kRow + t];
      gB1 += a;
    }
    __syncthreads();  // the next tile overwrites the activations
  }
  // ---- publish
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) atomicAdd(&g[kW2 + (i0 + r) * kMlpH + j0 + c], gW2[r][c]);
#pragma unroll
  for (int c = 0; c < 6; ++c) atomicAdd(&g[kW1 + h1r * kMlpF + f0 + c], gW1[c]);
  if (t < kMlpH) {
    atomicAdd(&g[kB2 + t], gB2);
    atomicAdd(&g[kB1 + t], gB1);
    atomicAdd(&g[kW3 + t], gW3);
  } else if (t == kMlpH) {
    atomicAdd(&g[kB3], gB3);
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0) atomicAdd(loss, lsum);
}

// Adam (Kingma & Ba 2015) with bias correction folded into the step size;
// refreshes the BF16 copy and clears the gradient.
__global__ void k_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, float lr_t, float b1, float b2,
                       float eps) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.0f - b1) * gi;
  float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] - lr_t * mi / (sqrtf(vi) + eps);
  w[i] = wi;
  wb[i] = __float2bfloat16_rn(wi);
  g[i] = 0.0f;
}

__global__ void k_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kMlpParams) wb[i] = __float2bfloat16_rn(w[i]);
}

// column sums and sums of squares of [feat | target] (13 columns), FP64
__global__ void k_moments(const float* __restrict__ feat, const float* __restrict__ target,
                          int64_t n, double* __restrict__ out) {
  double s[kMlpF + 1], s2[kMlpF + 1];
#pragma unroll
  for (int j = 0; j <= kMlpF; ++j) s[j] = s2[j] = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int j = 0; j <= kMlpF; ++j) {
      double x = j < kMlpF ? feat[i * kMlpF + j] : target[i];
      s[j] += x;
      s2[j] += x * x;
    }
  }
#pragma unroll
  for (int j = 0; j <= kMlpF; ++j) {
    for (int o = 16; o > 0; o >>= 1) {
      s[j] += __shfl_xor_sync(0xffffffffu, s[j], o);
      s2[j] += __shfl_xor_sync(0xffffffffu, s2[j], o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&out[j], s[j]);
      atomicAdd(&out[kMlpF + 1 + j], s2[j]);
    }
  }
}

uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

double uniform01(uint64_t& x) { return ((splitmix64(x) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

// normalisation from the data on first use
ckd_status ensure_norm(ckd_mlp* net, const float* feat, const float* target, int64_t n,
                       cudaStream_t s) {
  if (net->norm_set) return CKD_OK;
  if (n < 2) return fail(CKD_ERR_BAD_ARG, "need at least two samples to set the normalisation");
  double* acc = nullptr;
  CKD_CUDA(dev_alloc((void**)&acc, sizeof(double) * 2 * (kMlpF + 1), s));
  CKD_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 2 * (kMlpF + 1), s));
  k_moments<<<(unsigned)std::min<int64_t>(cdiv(n, 256), 296), 256, 0, s>>>(feat, target, n, acc);
  CKD_LAUNCH_CHECK();
  double h[2 * (kMlpF + 1)];
  CKD_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaStreamSynchronize(s));
  CKD_CUDA(dev_free(acc, s));
  for (int j = 0; j <= kMlpF; ++j) {
    double mu = h[j] / n;
    double var = std::max(0.0, h[kMlpF + 1 + j] / n - mu * mu);
    double sg = std::max(std::sqrt(var), 1e-6);
    if (j < kMlpF) {
      net->norm.mu[j] = (float)mu;
      net->norm.isg[j] = (float)(1.0 / sg);
    } else {
      net->norm.y_mu = (float)mu;
      net->norm.y_sigma = (float)sg;
    }
  }
  net->norm_set = true;
  return CKD_OK;
}

int grad_grid(int64_t n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<int64_t>(1, std::min<int64_t>(cdiv(n, kTile), sms));
}

ckd_status launch_grad(const ckd_mlp* net, const float* feat, const float* target, int64_t n,
                       float scale, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    CKD_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kGradSmem));
    attr = true;
  }
  k_mlp_grad<<<grad_grid(n), kTile, kGradSmem, s>>>(net->wb, net->norm, feat, target, n, scale,
                                                    net->g, net->loss);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

template <int D>
ckd_status features_d(const ckd_tree* t, const double* q, int64_t nq, int k, float* feat,
                      cudaStream_t s) {
  k_features<D><<<(unsigned)cdiv(nq, 256), 256, 0, s>>>(t->view(), q, nq, k, feat);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

template <int D>
ckd_status radius_d(const ckd_tree* t, const ckd_mlp* net, const double* q, const int32_t* order,
                    const int32_t* qleaf, int64_t nq, int k, double* r2, cudaStream_t s) {
  int dev = 0, sms = 148;
  CKD_CUDA(cudaGetDevice(&dev));
  CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int64_t grid = std::min<int64_t>(cdiv(nq, 128), (int64_t)sms * 16);
  k_mlp_radius<D><<<(unsigned)grid, 128, 0, s>>>(t->view(), net->wb, net->norm, q, order, qleaf,
                                                 nq, k, r2);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

}  // namespace

ckd_status mlp_radius(const ckd_tree* t, const ckd_mlp* net, const double* q, const int32_t* order,
                      const int32_t* qleaf, int64_t nq, int k, double* r2, cudaStream_t s) {
  if (mlp_tensor_cores()) return mlp_radius_tc(t, net, q, order, qleaf, nq, k, r2, s);
  switch (t->d) {
    case 1: return radius_d<1>(t, net, q, order, qleaf, nq, k, r2, s);
    case 2: return radius_d<2>(t, net, q, order, qleaf, nq, k, r2, s);
    case 3: return radius_d<3>(t, net, q, order, qleaf, nq, k, r2, s);
    case 4: return radius_d<4>(t, net, q, order, qleaf, nq, k, r2, s);
    case 5: return radius_d<5>(t, net, q, order, qleaf, nq, k, r2, s);
    case 6: return radius_d<6>(t, net, q, order, qleaf, nq, k, r2, s);
    case 7: return radius_d<7>(t, net, q, order, qleaf, nq, k, r2, s);
    case 8: return radius_d<8>(t, net, q, order, qleaf, nq, k, r2, s);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

ckd_status mlp_check(const ckd_mlp* net) {
  if (!net) return fail(CKD_ERR_BAD_ARG, "null network handle");
  int dev = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  if (dev != net->device)
    return fail(CKD_ERR_BAD_ARG, "the current device is not the network's device");
  if (!net->norm_set) return fail(CKD_ERR_BAD_ARG, "the network has not been trained or set");
  return CKD_OK;
}

}  // namespace ckd

using namespace ckd;

extern "C" {

ckd_status ckd_mlp_create(uint64_t seed, ckd_mlp** out) {
  if (!out) return fail(CKD_ERR_BAD_ARG, "null output handle");
  *out = nullptr;
  ckd_mlp* net = new ckd_mlp();
  CKD_CUDA(cudaGetDevice(&net->device));
  // He-normal hidden layers, 1/sqrt(fan_in) output layer, zero biases
  std::vector<float> w(kMlpParams, 0.0f);
  uint64_t st = seed;
  auto normal = [&st]() {
    double u1 = uniform01(st), u2 = uniform01(st);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  };
  for (int i = 0; i < kMlpH * kMlpF; ++i) w[kW1 + i] = (float)(normal() * std::sqrt(2.0 / kMlpF));
  for (int i = 0; i < kMlpH * kMlpH; ++i) w[kW2 + i] = (float)(normal() * std::sqrt(2.0 / kMlpH));
  for (int i = 0; i < kMlpH; ++i) w[kW3 + i] = (float)(normal() * std::sqrt(1.0 / kMlpH));
  float** bufs[4] = {&net->w, &net->g, &net->m, &net->v};
  for (float** b : bufs) {
    cudaError_t e = cudaMalloc((void**)b, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMemset(*b, 0, sizeof(float) * kMlpParams);
    if (e != cudaSuccess) {
      ckd_mlp_free(net);
      return cuda_fail(e, "cudaMalloc(network)");
    }
  }
  cudaError_t e = cudaMalloc((void**)&net->wb, sizeof(__nv_bfloat16) * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc((void**)&net->loss, sizeof(double));
  if (e == cudaSuccess)
    e = cudaMemcpy(net->w, w.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    ckd_mlp_free(net);
    return cuda_fail(e, "network setup");
  }
  k_to_bf16<<<(unsigned)cdiv(kMlpParams, 256), 256>>>(net->w, net->wb);
  note_launch();
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    ckd_mlp_free(net);
    return cuda_fail(e, "network setup");
  }
  *out = net;
  return CKD_OK;
}

ckd_status ckd_mlp_free(ckd_mlp* net) {
  if (!net) return CKD_OK;
  cudaFree(net->w);
  cudaFree(net->wb);
  cudaFree(net->g);
  cudaFree(net->m);
  cudaFree(net->v);
  cudaFree(net->loss);
  delete net;
  return CKD_OK;
}

ckd_status ckd_mlp_get(const ckd_mlp* net, float* params, float* norm, float* margin,
                       int64_t* steps) {
  if (!net) return fail(CKD_ERR_BAD_ARG, "null network handle");
  if (params) CKD_CUDA(cudaMemcpy(params, net->w, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
  if (norm) {
    std::memcpy(norm, net->norm.mu, sizeof(float) * kMlpF);
    std::memcpy(norm + kMlpF, net->norm.isg, sizeof(float) * kMlpF);
    norm[2 * kMlpF] = net->norm.y_mu;
    norm[2 * kMlpF + 1] = net->norm.y_sigma;
  }
  if (margin) *margin = net->norm.margin;
  if (steps) *steps = net->steps;
  return CKD_OK;
}

ckd_status ckd_mlp_set(ckd_mlp* net, const float* params, const float* norm, float margin) {
  if (!net) return fail(CKD_ERR_BAD_ARG, "null network handle");
  if (!std::isfinite(margin)) return fail(CKD_ERR_BAD_ARG, "margin must be finite");
  if (norm) {
    for (int j = 0; j < 2 * kMlpF + 2; ++j)
      if (!std::isfinite(norm[j])) return fail(CKD_ERR_BAD_ARG, "normalisation must be finite");
    if (!(norm[2 * kMlpF + 1] > 0)) return fail(CKD_ERR_BAD_ARG, "target sigma must be positive");
    std::memcpy(net->norm.mu, norm, sizeof(float) * kMlpF);
    std::memcpy(net->norm.isg, norm + kMlpF, sizeof(float) * kMlpF);
    net->norm.y_mu = norm[2 * kMlpF];
    net->norm.y_sigma = norm[2 * kMlpF + 1];
    net->norm_set = true;
  }
  if (params) {
    CKD_CUDA(cudaMemcpy(net->w, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    CKD_CUDA(cudaMemset(net->m, 0, sizeof(float) * kMlpParams));
    CKD_CUDA(cudaMemset(net->v, 0, sizeof(float) * kMlpParams));
    k_to_bf16<<<(unsigned)cdiv(kMlpParams, 256), 256>>>(net->w, net->wb);
    CKD_LAUNCH_CHECK();
    CKD_CUDA(cudaDeviceSynchronize());
    net->steps = 0;
  }
  net->norm.margin = margin;
  return CKD_OK;
}

ckd_status ckd_mlp_features(const ckd_tree* t, const double* q, int64_t nq, int k, float* feat,
                            void* stream) {
  if (!t) return fail(CKD_ERR_BAD_ARG, "null tree handle");
  if (t->n_trees != 1) return fail(CKD_ERR_BAD_ARG, "features are defined for a single tree");
  if (k < 1) return fail(CKD_ERR_BAD_ARG, "k must be a positive integer");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !feat) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  cudaStream_t s = (cudaStream_t)stream;
  switch (t->d) {
    case 1: return features_d<1>(t, q, nq, k, feat, s);
    case 2: return features_d<2>(t, q, nq, k, feat, s);
    case 3: return features_d<3>(t, q, nq, k, feat, s);
    case 4: return features_d<4>(t, q, nq, k, feat, s);
    case 5: return features_d<5>(t, q, nq, k, feat, s);
    case 6: return features_d<6>(t, q, nq, k, feat, s);
    case 7: return features_d<7>(t, q, nq, k, feat, s);
    case 8: return features_d<8>(t, q, nq, k, feat, s);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

ckd_status ckd_mlp_grad(ckd_mlp* net, const float* feat, const float* target, int64_t n,
                        float* grad, float* loss, void* stream) {
  if (!net) return fail(CKD_ERR_BAD_ARG, "null network handle");
  if (n < 1 || !feat || !target || !grad) return fail(CKD_ERR_BAD_ARG, "bad gradient arguments");
  cudaStream_t s = (cudaStream_t)stream;
  CKD_TRY(ensure_norm(net, feat, target, n, s));
  CKD_CUDA(cudaMemsetAsync(net->g, 0, sizeof(float) * kMlpParams, s));
  CKD_CUDA(cudaMemsetAsync(net->loss, 0, sizeof(double), s));
  CKD_TRY(launch_grad(net, feat, target, n, (float)(2.0 / n), s));
  double l = 0;
  CKD_CUDA(cudaMemcpyAsync(grad, net->g, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaMemcpyAsync(&l, net->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaMemsetAsync(net->g, 0, sizeof(float) * kMlpParams, s));
  CKD_CUDA(cudaStreamSynchronize(s));
  if (loss) *loss = (float)(l / n);
  return CKD_OK;
}

ckd_status ckd_mlp_train(ckd_mlp* net, const float* feat, const float* target, int64_t n, int batch,
                         int epochs, float lr, float* loss_hist, void* stream) {
  if (!net) return fail(CKD_ERR_BAD_ARG, "null network handle");
  if (n < 2 || batch < 1 || epochs < 0 || !(lr > 0) || !feat || !target)
    return fail(CKD_ERR_BAD_ARG, "bad training arguments");
  cudaStream_t s = (cudaStream_t)stream;
  CKD_TRY(ensure_norm(net, feat, target, n, s));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int e = 0; e < epochs; ++e) {
    CKD_CUDA(cudaMemsetAsync(net->loss, 0, sizeof(double), s));
    for (int64_t off = 0; off < n; off += batch) {
      const int64_t b = std::min<int64_t>(batch, n - off);
      CKD_TRY(launch_grad(net, feat + off * kMlpF, target + off, b, (float)(2.0 / b), s));
      net->steps += 1;
      const double t = (double)net->steps;
      const float lr_t =
          (float)(lr * std::sqrt(1.0 - std::pow((double)b2, t)) / (1.0 - std::pow((double)b1, t)));
      k_adam<<<(unsigned)cdiv(kMlpParams, 256), 256, 0, s>>>(net->w, net->wb, net->g, net->m,
                                                             net->v, lr_t, b1, b2, eps);
      CKD_LAUNCH_CHECK();
    }
    if (loss_hist) {
      double l = 0;
      CKD_CUDA(cudaMemcpyAsync(&l, net->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
      CKD_CUDA(cudaStreamSynchronize(s));
      loss_hist[e] = (float)(l / n);
    }
  }
  CKD_CUDA(cudaStreamSynchronize(s));
  return CKD_OK;
}

ckd_status ckd_mlp_predict(const ckd_mlp* net, const float* feat, int64_t n, float* y,
                           void* stream) {
  CKD_TRY(mlp_check(net));
  if (n < 0) return fail(CKD_ERR_BAD_ARG, "negative sample count");
  if (n == 0) return CKD_OK;
  if (!feat || !y) return fail(CKD_ERR_BAD_ARG, "null feature or output pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (mlp_tensor_cores()) return mlp_predict_tc(net, feat, n, y, s);
  k_mlp_forward<<<(unsigned)cdiv(n, 128), 128, 0, s>>>(
      net->wb, net->norm, feat, n, y);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

}  // extern "C"
