// ckd_mlp.cuh -- parameter layout and handle of the learned k-th-distance bound.
#pragma once
#include <cuda_bf16.h>

#include "ckd_traverse.cuh"

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

// mean over axes of log2(hi - lo) of a node's [lo0, hi0, lo1, hi1, ...] bounds
template <int D>
__device__ __forceinline__ float mean_log2_side(const double* __restrict__ b, int32_t node) {
  const double* p = b + (int64_t)node * 2 * D;
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    float w = (float)(__ldg(&p[2 * j + 1]) - __ldg(&p[2 * j]));
    s += log2f(fmaxf(w, 1e-30f));
  }
  return s * (1.0f / D);
}

// Features of one query located in `leaf` (order is fixed; the host side and
// the CPU reference of the network only see the resulting vectors):
//  0 log2 count(leaf)           1 mean log2 side of the leaf's cell
//  2 mean log2 side of the leaf's tight box (floored at cell side / 2^20)
//  3 log2 count(sibling)        4 mean log2 side of the sibling's cell
//  5 log2 count(grandparent)    6 mean log2 side of the grandparent's cell
//  7 log2 count(great-grandparent)  8 mean log2 side of its cell
//  9 depth of the leaf          10 log2 k
//  11 0.5 log2 of the query's squared offset from the leaf cell's centre in
//     units of the cell's sides (+ 2^-20)
// Missing ancestors (shallow trees) repeat the nearest existing node.
template <int D>
__device__ __forceinline__ void leaf_features(const TreeView& tv, const double (&q)[D],
                                              int32_t leaf, int k, float (&f)[kMlpF]) {
  NodeMeta ml = load_meta(tv.meta, leaf);
  const int32_t par = ml.parent >= 0 ? ml.parent : leaf;
  NodeMeta mp = load_meta(tv.meta, par);
  const int32_t sib = ml.parent >= 0 ? (mp.left == leaf ? leaf + 1 : mp.left) : leaf;
  const int32_t gp = mp.parent >= 0 ? mp.parent : par;
  NodeMeta mg = load_meta(tv.meta, gp);
  const int32_t ggp = mg.parent >= 0 ? mg.parent : gp;
  NodeMeta mgg = load_meta(tv.meta, ggp);
  NodeMeta ms = load_meta(tv.meta, sib);
  f[0] = log2f((float)max(ml.count, 1));
  f[1] = mean_log2_side<D>(tv.cell, leaf);
  f[2] = fmaxf(mean_log2_side<D>(tv.box, leaf), f[1] - 20.0f);
  f[3] = log2f((float)max(ms.count, 1));
  f[4] = mean_log2_side<D>(tv.cell, sib);
  f[5] = log2f((float)max(mg.count, 1));
  f[6] = mean_log2_side<D>(tv.cell, gp);
  f[7] = log2f((float)max(mgg.count, 1));
  f[8] = mean_log2_side<D>(tv.cell, ggp);
  f[9] = (float)ml.depth;
  f[10] = log2f((float)k);
  const double* c = tv.cell + (int64_t)leaf * 2 * D;
  float off = 0.0f;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double lo = __ldg(&c[2 * j]), hi = __ldg(&c[2 * j + 1]);
    double w = hi - lo;
    if (w > 0) {
      float u = (float)((q[j] - 0.5 * (lo + hi)) / w);
      off = fmaf(u, u, off);
    }
  }
  f[11] = 0.5f * log2f(off + 9.5367431640625e-07f);
}

// leaf of a query by descent (left iff q[axis] < split)
template <int D>
__device__ __forceinline__ int32_t locate_leaf(const NodeMeta* __restrict__ meta,
                                               const double (&q)[D]) {
  int32_t node = 0;
  NodeMeta m = load_meta(meta, 0);
  while (m.left >= 0) {
    double qa = 0.0;
#pragma unroll
    for (int j = 0; j < D; ++j)
      if (j == m.axis) qa = q[j];
    node = qa < m.split ? m.left : m.left + 1;
    m = load_meta(meta, node);
  }
  return node;
}

// r2[q] = (predicted k-th distance * 2^margin)^2 for every query (queries visited
// in the given order; qleaf may be null, then each query is located by descent)
ckd_status mlp_radius(const ckd_tree* t, const ckd_mlp* net, const double* q, const int32_t* order,
                      const int32_t* qleaf, int64_t nq, int k, double* r2, cudaStream_t s);
ckd_status mlp_check(const ckd_mlp* net);
// tensor-core (tcgen05) inference: the same radius / prediction as mlp_radius and
// ckd_mlp_predict with BF16 activations into the MMAs
ckd_status mlp_radius_tc(const ckd_tree* t, const ckd_mlp* net, const double* q,
                         const int32_t* order, const int32_t* qleaf, int64_t nq, int k, double* r2,
                         cudaStream_t s);
ckd_status mlp_predict_tc(const ckd_mlp* net, const float* feat, int64_t n, float* y,
                          cudaStream_t s);

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
