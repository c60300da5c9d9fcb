// ckd_knn_lane.cuh -- the per-lane kNN traversal with the compact heap, shared by
// the kNN kernels (knn.cu) and the persistent forest kernel (forest_pk.cu).
#pragma once
#include "ckd_common.cuh"
#include "ckd_knn.cuh"
#include "ckd_traverse.cuh"

namespace ckd {
CKD_LD_BEGIN

// ====================================== per-lane traversal, compact heap
// Each lane walks the tree for its own query: both children's FP32 boxes are
// tested when a node is expanded, the nearer child is taken and the other pushed
// with its bound on a per-lane stack, so entries that the shrinking k-th distance
// has pruned are dropped without reloading a node.  Lanes descend until they
// reach a leaf, then scan leaves together (while-while structure): an FP32 screen
// on leaf-relative coordinates, an FP64 recheck and the compact heap.  Used for
// unordered query batches, for the learned path's reruns, by the allocation-free
// entry point and as the learned path's bounded kernel when selected.
//
// BOUNDED: every query starts with its heap full of k sentinels (key r2[q],
// id INT32_MAX) instead of HUGE, so pruning starts at the root.  A point is
// accepted iff (d2, id) < the current worst, so every point with d2 <= r2[q] is
// still seen; when no sentinel is left the heap holds the exact k nearest.  A
// query that ends with a sentinel (fewer than k points within the bound) is
// appended to miss[] for the unbounded rerun and its output row is not written.
//
// The warp's 32 query slots are gw * 32 .. gw * 32 + 31 of the (ordered) batch;
// Hw is the warp's heap base in shared memory ((k + 1) * 32 entries); a query
// without its own root (qroot null) starts at node root0.
template <int D, bool PER, bool BOUNDED, bool PAIR>
__device__ __forceinline__ void knn_lane_run(
    const TreeView& tv, const double* __restrict__ Q, const int32_t* __restrict__ order,
    int64_t nq, int k, int sorted, double* __restrict__ dist, int64_t* __restrict__ idx,
    unsigned long long* __restrict__ stats, const double* __restrict__ r2,
    int32_t* __restrict__ miss, unsigned* __restrict__ nmiss, const int32_t* __restrict__ qleaf,
    const int32_t* __restrict__ qroot, int32_t root0, uint2* Hw, int lane, int64_t gw) {
  constexpr int NV = (D + 3) / 4;
  constexpr unsigned FULL = 0xffffffffu;
  unsigned long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // heap slot s of this lane at H[s * 32 + lane]: (key bits, position); keys are
  // non-negative floats, so their bit patterns order as unsigned integers, and
  // every lane always addresses its own bank pair (no conflicts between lanes
  // at different heap levels)
  uint2* H = Hw + lane;
  const int64_t slot = gw * 32 + lane;
  const bool valid = slot < nq;
  const int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
  QueryScreen<D, PER> qs;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    q[j] = valid ? Q[qi * D + j] : 0.0;
    qs.q32[j] = __double2float_rn(q[j]);
    qs.dlt[j] = kTwoM21 * (fabsf(qs.q32[j]) + tv.slack[j]) * 1.0001f;
  }
  float skey = FLT_MAX;
  int32_t spos = kPosMissing;
  float wd32 = FLT_MAX;
  double rr = CKD_HUGE;
  if (BOUNDED && valid) {
    const double b = r2[qi];
    if (b < CKD_HUGE) {
      rr = b;
      skey = __double2float_rn(b);
      spos = kPosBound;
      wd32 = __double2float_ru(b);
    }
  }
  const CompactCtx<D, PER> cx{tv, rr};
  CompactHeap hp{H, 0u, 0, 0.0f};
  compact_init<D, PER>(hp, k, skey, spos, wd32);
  // Direct box gaps max(lo - xl, xh - hi, 0) while the query's ball cannot reach
  // the periodic box faces (wf: then the closest image of any point that can
  // still enter the heap is the point itself), and point screens on absolute
  // FP32 coordinates with the per-query error bounds Ed (direct) / Ew (minimum
  // image): fl32(fl32(p_j) - fl32(q_j)) is within 2^-23 (B_j + |q_j|) of
  // p_j - q_j, so e_j = 2^-22 (B_j + |q_j|) bounds it with a factor-2 margin and
  // a point whose FP64 squared distance is <= tau has an FP32 sum of squares
  // <= (sqrt(tau) + |e|)^2 / (1 - 2^-20).
  float xl[D], xh[D], Ed = 0.0f, Ew = 0.0f;
  bool wf = !PER;
  {
    float e2 = 0.0f, e2w = 0.0f;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      xl[j] = __fadd_ru(qs.q32[j], qs.dlt[j]);
      xh[j] = __fsub_rd(qs.q32[j], qs.dlt[j]);
      const float ej = __fmaf_ru(kTwoM22, __fadd_ru(tv.slack[j], fabsf(qs.q32[j])), 1e-37f);
      e2 = __fmaf_ru(ej, ej, e2);
      const float ejw = PER ? __fmaf_ru(kTwoM22, (float)tv.L[j], ej) : ej;
      e2w = __fmaf_ru(ejw, ejw, e2w);
    }
    Ed = sqrt_up(e2);
    Ew = sqrt_up(e2w);
  }
  auto box_lb = [&](const float* lo, const float* hi) -> float {
    if (!PER || wf) {
      float s2 = 0.0f;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        const float g = fmaxf(fmaxf(lo[j] - xl[j], xh[j] - hi[j]), 0.0f);
        s2 = fmaf(g, g, s2);
      }
      return s2 * kShrink;
    }
    float lo4[4 * NV], hi4[4 * NV];
#pragma unroll
    for (int j = 0; j < 4 * NV; ++j) {
      lo4[j] = j < D ? lo[j] : 0.0f;
      hi4[j] = j < D ? hi[j] : 0.0f;
    }
    return box_mind_lb<D, PER>(tv, qs, lo4, hi4);
  };
  auto node_lb = [&](int32_t nd) -> float {
    float lo[D], hi[D];
    const float2* b = reinterpret_cast<const float2*>(tv.box32 + (int64_t)nd * 2 * D);
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const float2 lh = CKD_LDT(b + j);
      lo[j] = lh.x;
      hi[j] = lh.y;
    }
    return box_lb(lo, hi);
  };

  uint2 sk[kLaneStack];  // (node, bound bits): one 8-byte entry per pending subtree
  int top = 0;
  int32_t node = valid ? (qroot ? qroot[qi] : root0) : -1;
  if (BOUNDED && valid && qleaf && spos == kPosBound) {
    // start at the lowest ancestor whose cell strictly contains [q - r, q + r]^D
    const float r32 = __fsqrt_ru(hp.wd32);
    int32_t a = qleaf[qi];
    while (a >= 0) {
      const float* c = tv.cell32 + (int64_t)a * 2 * D;
      bool inside = true;
#pragma unroll
      for (int j = 0; j < D; ++j) {
        const float2 lh = CKD_LDT(reinterpret_cast<const float2*>(c) + j);
        inside = inside && __fsub_rd(__fsub_rd(qs.q32[j], r32), qs.dlt[j]) > lh.x &&
                 __fadd_ru(__fadd_ru(qs.q32[j], r32), qs.dlt[j]) < lh.y;
      }
      if (inside) break;
      a = load_meta(tv.meta, a).parent;
    }
    node = a < 0 ? node : a;
  }
  // PAIR: stack entries and `node` carry the leaf flag (a leaf is stored as ~id,
  // < -1 because children ids are >= 1; -1 means "no node") and internal nodes are
  // expanded from their child-pair record alone (both children's FP32 boxes, ids
  // and leaf flags), one dependent load per level.  Otherwise the node's meta is
  // read first, then both children's FP32 boxes.
  constexpr int PF = pair_f4(D);
  bool is_leaf = node >= 0 && PAIR && load_meta(tv.meta, node).left < 0;
  NodeMeta m;
  while (node >= 0) {
    // ---- descend to a leaf, nearer child first
    if (!PAIR) {
      m = load_meta(tv.meta, node);
      while (node >= 0 && m.left >= 0) {
        if (stats) st[0] += 1;
        const float ml = node_lb(m.left);
        const float mr = node_lb(m.left + 1);
        const bool nl = ml <= hp.wd32, nr = mr <= hp.wd32;
        if (nl && nr) {
          const bool lf = ml <= mr;
          sk[top] = make_uint2((unsigned)(lf ? m.left + 1 : m.left), __float_as_uint(lf ? mr : ml));
          ++top;
          node = lf ? m.left : m.left + 1;
        } else if (nl || nr) {
          node = nl ? m.left : m.left + 1;
        } else {
          node = -1;
          while (top > 0) {
            --top;
            const uint2 e = sk[top];
            if (__uint_as_float(e.y) <= hp.wd32) {
              node = (int32_t)e.x;
              break;
            }
          }
        }
        if (node >= 0) m = load_meta(tv.meta, node);
      }
      if (node < 0) break;
    } else {
      while (!is_leaf) {
        if (stats) st[0] += 1;
        const float4* rec = tv.pair + (int64_t)node * PF;
        float lo_l[4 * NV], hi_l[4 * NV], lo_r[4 * NV], hi_r[4 * NV];
#pragma unroll
        for (int h = 0; h < NV; ++h) {
          const float4 a = CKD_LDT(rec + h), b = CKD_LDT(rec + NV + h);
          const float4 c = CKD_LDT(rec + 2 * NV + h), d = CKD_LDT(rec + 3 * NV + h);
          lo_l[4 * h] = a.x; lo_l[4 * h + 1] = a.y; lo_l[4 * h + 2] = a.z; lo_l[4 * h + 3] = a.w;
          hi_l[4 * h] = b.x; hi_l[4 * h + 1] = b.y; hi_l[4 * h + 2] = b.z; hi_l[4 * h + 3] = b.w;
          lo_r[4 * h] = c.x; lo_r[4 * h + 1] = c.y; lo_r[4 * h + 2] = c.z; lo_r[4 * h + 3] = c.w;
          hi_r[4 * h] = d.x; hi_r[4 * h + 1] = d.y; hi_r[4 * h + 2] = d.z; hi_r[4 * h + 3] = d.w;
        }
        const int4 info = CKD_LDT(reinterpret_cast<const int4*>(rec + 4 * NV));
        const float ml = box_lb(lo_l, hi_l);
        const float mr = box_lb(lo_r, hi_r);
        const bool nl = ml <= hp.wd32, nr = mr <= hp.wd32;
        const int32_t el = info.z ? ~info.x : info.x, er = info.w ? ~info.y : info.y;
        int32_t nxt = -1;
        if (nl && nr) {
          const bool lf = ml <= mr;
          sk[top] = make_uint2((unsigned)(lf ? er : el), __float_as_uint(lf ? mr : ml));
          ++top;
          nxt = lf ? el : er;
        } else if (nl || nr) {
          nxt = nl ? el : er;
        } else {
          while (top > 0) {
            --top;
            const uint2 e = sk[top];
            if (__uint_as_float(e.y) <= hp.wd32) {
              nxt = (int32_t)e.x;
              break;
            }
          }
          if (nxt == -1) break;
        }
        is_leaf = nxt < 0;
        node = is_leaf ? ~nxt : nxt;
      }
      if (!is_leaf) break;
      m = load_meta(tv.meta, node);
    }

    // ---- scan the leaf
    if (stats) {
      st[2] += 1;
      st[3] += m.count;
    }
    {
      if (PER && !wf) {
        const float r32 = sqrt_up(hp.wd32);
        bool inside = true;
#pragma unroll
        for (int j = 0; j < D; ++j)
          inside = inside && __fadd_ru(__fadd_ru(fabsf(qs.q32[j]), r32), qs.dlt[j]) <
                                 0.5f * (float)tv.L[j];
        wf = inside;
      }
      for (int base = 0; base < m.count; base += 32) {
        const int cnt = min(32, m.count - base);
        const int32_t p0 = m.start + base;
        const float t = __fadd_ru(sqrt_up(hp.wd32), wf ? Ed : Ew);
        const float thr = __fmul_ru(__fmul_ru(t, t), 1.0000020f);
        unsigned mask = 0;
        for (int i = 0; i < cnt; ++i) {
          float v[4 * NV];
#pragma unroll
          for (int h = 0; h < NV; ++h) {
            const float4 f = CKD_LDT(&tv.pts32[(int64_t)(p0 + i) * NV + h]);
            v[4 * h] = f.x;
            v[4 * h + 1] = f.y;
            v[4 * h + 2] = f.z;
            v[4 * h + 3] = f.w;
          }
          float s2 = 0.0f;
#pragma unroll
          for (int j = 0; j < D; ++j) {
            float a = v[j] - qs.q32[j];
            if (PER && !wf) {
              a = fabsf(a);
              a = fminf(a, (float)tv.L[j] - a);
            }
            s2 = fmaf(a, a, s2);
          }
          if (s2 <= thr) mask |= 1u << i;
        }
        if (stats) st[5] += __popc(mask);
        if (BOUNDED) {
          // two candidates at a time, their FP64 records loaded together (faster
          // for the bounded search, slower for the plain one)
          while (mask) {
            const int i0 = __ffs(mask) - 1;
            mask &= mask - 1;
            const int i1 = mask ? __ffs(mask) - 1 : i0;
            mask &= mask - 1;
            const int32_t pa = p0 + i0, pb = p0 + i1;
            const double da = point_d2_rec<D, PER>(tv, q, pa);
            const double db = point_d2_rec<D, PER>(tv, q, pb);
            if (compact_offer<D, PER, true>(hp, k, cx, q, da, pa) && stats) st[6] += 1;
            if (i1 != i0 && compact_offer<D, PER, true>(hp, k, cx, q, db, pb) && stats) st[6] += 1;
          }
        } else {
          while (mask) {
            const int i = __ffs(mask) - 1;
            mask &= mask - 1;
            const int32_t p = p0 + i;
            const double d2 = point_d2_rec<D, PER>(tv, q, p);
            if (compact_offer<D, PER, false>(hp, k, cx, q, d2, p) && stats) st[6] += 1;
          }
        }
      }
    }
    // ---- next: pop the nearest pending subtree still within reach
    int32_t nxt = -1;
    while (top > 0) {
      --top;
      const uint2 e = sk[top];
      if (__uint_as_float(e.y) <= hp.wd32) {
        nxt = (int32_t)e.x;
        break;
      }
    }
    if (nxt == -1) break;
    if (PAIR) {
      is_leaf = nxt < 0;
      node = is_leaf ? ~nxt : nxt;
    } else {
      node = nxt;
    }
  }
  if (stats) {
    // slots 4 and 7: 32 x the warp's largest leaf-scan and node-test counts, so that
    // against slots 2 and 0 (every lane's) they show how long lanes wait for the
    // slowest query of their warp
    unsigned long long m2 = st[2], m0 = st[0];
    for (int o = 16; o > 0; o >>= 1) {
      m2 = max(m2, __shfl_xor_sync(FULL, m2, o));
      m0 = max(m0, __shfl_xor_sync(FULL, m0, o));
    }
    st[4] = lane == 0 ? 32 * m2 : 0;
    st[7] = lane == 0 ? 32 * m0 : 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      unsigned long long v = st[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
      if (lane == 0) atomicAdd(&stats[c], v);
    }
  }
  const bool missed = BOUNDED && valid && hp.wp == kPosBound;
  unsigned missmask = 0;
  if (BOUNDED) {
    missmask = __ballot_sync(FULL, missed);
    if (missmask) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(nmiss, (unsigned)__popc(missmask));
      base = __shfl_sync(FULL, base, 0);
      if (missed) miss[base + __popc(missmask & ((1u << lane) - 1u))] = (int32_t)qi;
    }
  }
  if (hp.cnt < k) compact_finish<D, PER>(hp, k, cx, q);
  if (sorted && valid && !missed) compact_sort<D, PER>(hp.H, k, cx, q);
  __syncwarp();
  compact_write<D, PER>(tv, hp.H - lane, lane, gw, nq, order, q, k, missmask, dist, idx);
}

CKD_LD_END
}  // namespace ckd
