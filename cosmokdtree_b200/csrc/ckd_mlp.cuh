// ckd_mlp.cuh -- parameter layout and handle of the learned k-th-distance bound.
#pragma once
#include <cuda_bf16.h>

#include "ckd_common.cuh"

namespace ckd {

constexpr int kMlpF = CKD_MLP_FEATURES;  // input features
constexpr int kMlpH = CKD_MLP_HIDDEN;    // width of both hidden layers
// flat FP32 parameter vector: W1 [H][F], b1 [H], W2 [H][H] (row = output unit),
// b2 [H], W3 [H], b3
constexpr int kW1 = 0;
constexpr int kB1 = kW1 + kMlpH * kMlpF;  // 768
constexpr int kW2 = kB1 + kMlpH;          // 832
constexpr int kB2 = kW2 + kMlpH * kMlpH;  // 4928
constexpr int kW3 = kB2 + kMlpH;          // 4992
constexpr int kB3 = kW3 + kMlpH;          // 5056
constexpr int kMlpParams = kB3 + 1;       // 5057
static_assert(kMlpParams == CKD_MLP_PARAMS, "parameter count must match include/ckd.h");
static_assert(kW2 % 4 == 0, "W2 rows are read as float4");

// feature standardisation, target scale and the calibrated margin (log2 units)
struct MlpNorm {
  float mu[kMlpF];
  float isg[kMlpF];  // 1 / sigma
  float y_mu = 0.0f, y_sigma = 1.0f;
  float margin = 0.0f;
};

// leaf of a query and the features of a query in a given leaf
template <int D>
__device__ void leaf_features(const TreeView& tv, const double (&q)[D], int32_t leaf, int k,
                              float (&f)[kMlpF]);

// r2[q] = (predicted k-th distance * 2^margin)^2 for every query (queries visited
// in the given order; qleaf may be null, then each query is located by descent)
ckd_status mlp_radius(const ckd_tree* t, const ckd_mlp* net, const double* q, const int32_t* order,
                      const int32_t* qleaf, int64_t nq, int k, double* r2, cudaStream_t s);
ckd_status mlp_check(const ckd_mlp* net);

}  // namespace ckd

// Host-side network object behind the opaque ckd_mlp* handle.
struct ckd_mlp {
  int device = 0;
  float* w = nullptr;            // FP32 master weights
  __nv_bfloat16* wb = nullptr;   // BF16 copy used by every forward pass
  float* g = nullptr;            // gradient accumulator
  float* m = nullptr;            // Adam first moment
  float* v = nullptr;            // Adam second moment
  double* loss = nullptr;        // summed squared error of the current epoch
  ckd::MlpNorm norm;
  bool norm_set = false;
  int64_t steps = 0;
};
