// ckd_traverse.cuh -- per-lane distance helpers and the query ordering pass.
#pragma once
#include <math_constants.h>

#include "ckd_common.cuh"

namespace ckd {

CKD_LD_BEGIN

// Squared distance between the lane's query and leaf-ordered point p
// (cosmokdtree.f90:1441-1465: dx = p - q, minimum image, d2 = sum dx^2 in axis order).
template <int D, bool PER>
__device__ __forceinline__ double point_d2(const TreeView& tv, const double (&q)[D], int32_t p) {
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double dx = dsub(CKD_LDT(&tv.pts[(int64_t)j * tv.n + p]), q[j]);
    if (PER) dx = min_image(dx, tv.L[j]);
    s = (j == 0) ? dmul(dx, dx) : dadd(s, dmul(dx, dx));
  }
  return s;
}

// point_d2 from the packed FP64 records (same operations, same result)
template <int D, bool PER>
__device__ __forceinline__ double point_d2_rec(const TreeView& tv, const double (&q)[D], int32_t p) {
  constexpr int NV = (D + 3) / 4;
  double v[4 * NV];
#pragma unroll
  for (int h = 0; h < NV; ++h) {
    const double2* r = reinterpret_cast<const double2*>(tv.pts64 + (int64_t)p * NV + h);
    const double2 a = CKD_LDT(r), b = CKD_LDT(r + 1);
    v[4 * h] = a.x;
    v[4 * h + 1] = a.y;
    v[4 * h + 2] = b.x;
    v[4 * h + 3] = b.y;
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double dx = dsub(v[j], q[j]);
    if (PER) dx = min_image(dx, tv.L[j]);
    s = (j == 0) ? dmul(dx, dx) : dadd(s, dmul(dx, dx));
  }
  return s;
}

// Conservative lower bound of the squared distance from q to any point of the
// node's tight bounding box.
template <int D, bool PER>
__device__ __forceinline__ double box_mind2(const TreeView& tv, const double (&q)[D], int32_t node) {
  const double* b = tv.box + (int64_t)node * 2 * D;
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double g = axis_gap<PER>(q[j], CKD_LDT(&b[2 * j]), CKD_LDT(&b[2 * j + 1]), tv.L[j]);
    s = (j == 0) ? dmul(g, g) : dadd(s, dmul(g, g));
  }
  return s;
}

// Upper bound of the squared distance from q to any point of the box
// (non-periodic; per axis max(|q-lo|, |q-hi|), cosmokdtree.f90:1509-1510).
template <int D>
__device__ __forceinline__ double box_maxd2(const TreeView& tv, const double (&q)[D], int32_t node) {
  const double* b = tv.box + (int64_t)node * 2 * D;
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double a = fabs(dsub(q[j], CKD_LDT(&b[2 * j])));
    double c = fabs(dsub(q[j], CKD_LDT(&b[2 * j + 1])));
    double g = a > c ? a : c;
    s = (j == 0) ? dmul(g, g) : dadd(s, dmul(g, g));
  }
  return s;
}

// Periodic form of box_maxd2 for the "whole subtree inside the ball" shortcut:
// the direct (unwrapped) upper bound, valid when on every axis both faces lie
// within L/2 of q -- then every point's minimum-image difference is its direct
// difference (min(a, L - a) = a for a <= L/2, also after rounding), so each
// point's computed squared distance is at most this bound.  Returns +inf when
// some axis fails the condition.
template <int D>
__device__ __forceinline__ double box_maxd2_near(const TreeView& tv, const double (&q)[D],
                                                 int32_t node) {
  const double* b = tv.box + (int64_t)node * 2 * D;
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double a = fabs(dsub(q[j], CKD_LDT(&b[2 * j])));
    double c = fabs(dsub(q[j], CKD_LDT(&b[2 * j + 1])));
    double g = a > c ? a : c;
    if (!(g <= 0.5 * tv.L[j])) return CUDART_INF;
    s = (j == 0) ? dmul(g, g) : dadd(s, dmul(g, g));
  }
  return s;
}

__device__ __forceinline__ NodeMeta load_meta(const NodeMeta* m, int32_t node) {
  const int4* p = reinterpret_cast<const int4*>(m + node);
  int4 a = CKD_LDT(p), b = CKD_LDT(p + 1);
  NodeMeta r;
  r.split = __hiloint2double(a.y, a.x);
  r.left = a.z;
  r.axis = a.w;
  r.start = b.x;
  r.count = b.y;
  r.depth = b.z;
  r.parent = b.w;
  return r;
}

CKD_LD_END

// Order queries by the leaf they fall in (a counting sort on the leaf's first
// point), so that the 32 lanes of a warp hold spatially adjacent queries.
ckd_status query_order(const ckd_tree* t, const double* q_dev, int64_t nq, int32_t* order,
                       cudaStream_t s);

}  // namespace ckd
