// ball_box.cu -- ball (radius) and axis-aligned box searches, two-phase CSR.
//
// Ball (cosmokdtree.f90:1015-1212): a point is a result iff its FP64 squared
// distance (reference arithmetic) is <= radius^2 (inclusive, :1126, :1175).  The
// reference's "fully inside" shortcut (:1116-1118, :1332-1366) selects exactly
// the same points, because a node's max-distance bound is never below the
// computed distance of a point inside it; the count pass uses it (with the
// tight box) to skip distance work, on periodic trees too when the box lies
// within half a box side of the query on every axis (box_maxd2_near).  Traversal is left child first, so the
// unsorted order of a row is the reference's non-periodic order (left-first DFS,
// leaf order).  sorted=1 orders each row by (d2, id).
//
// Box (cosmokdtree.f90:1220-1328): descend left iff box_lo[axis] < split, right
// iff box_hi[axis] > split (strict), leaf test lo <= x <= hi on every axis
// (inclusive), no periodic wrap.  Each lane carries one box; the warp walks the
// union of the lanes' paths with a per-entry lane mask, left first, so every
// row comes out in the reference's order.
#include <algorithm>

#include "ckd_common.cuh"
#include "ckd_traverse.cuh"

namespace ckd {

namespace {

constexpr int kStack = 96;

template <int D, bool PER, bool FILL>
__global__ void __launch_bounds__(128) k_ball(TreeView tv, const double* __restrict__ Q,
                                              const int32_t* __restrict__ order, int64_t nq_max,
                                              const unsigned* __restrict__ nq_dev,
                                              double r2, int32_t* __restrict__ gstack,
                                              int stack_len, int64_t* __restrict__ counts,
                                              const int64_t* __restrict__ offsets,
                                              int64_t* __restrict__ oidx,
                                              double* __restrict__ odist, int want_d2) {
  __shared__ int32_t sstk[4][kStack];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  int32_t* stk = gstack ? gstack + gw * stack_len : sstk[w];
  const int64_t nq = nq_dev ? (int64_t)*nq_dev : nq_max;
  if (gw * 32 >= nq) return;  // whole warp past the (device-side) query count
  int64_t slot = gw * 32 + lane;
  bool valid = slot < nq;
  int64_t qi = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  double q[D];
#pragma unroll
  for (int j = 0; j < D; ++j) q[j] = valid ? Q[qi * D + j] : 0.0;
  double rr = valid ? r2 : -1.0;
  int64_t cnt = 0;
  int64_t cur = (FILL && valid) ? offsets[qi] : 0;
  const int64_t cur_end = (FILL && valid) ? offsets[qi + 1] : 0;
  int32_t cov_lo = 0, cov_hi = 0;  // point range already counted whole (count pass)
  int top = 0;
  if (lane == 0) stk[0] = 0;
  __syncwarp();
  while (top >= 0) {
    int32_t node = stk[top];
    --top;
    __syncwarp();
    NodeMeta m = load_meta(tv.meta, node);
    bool need = box_mind2<D, PER>(tv, q, node) <= rr;
    if (!FILL && need && m.start >= cov_lo && m.start < cov_hi) need = false;
    if (!FILL && need && m.left >= 0 &&
        (PER ? box_maxd2_near<D>(tv, q, node) : box_maxd2<D>(tv, q, node)) <= rr) {
      cnt += m.count;  // whole subtree inside the ball
      cov_lo = m.start;
      cov_hi = m.start + m.count;
      need = false;
    }
    unsigned nm = __ballot_sync(0xffffffffu, need);
    if (nm == 0) continue;
    if (m.left < 0) {
      for (int i = 0; i < m.count; ++i) {
        int32_t p = m.start + i;
        double d2 = point_d2<D, PER>(tv, q, p);
        if (need && d2 <= rr) {
          if (FILL) {
            if (cur >= cur_end) continue;  // the row is full (count and fill always agree)
            oidx[cur] = __ldg(&tv.ids[p]);
            odist[cur] = want_d2 ? d2 : sqrt(d2);
            ++cur;
          } else {
            ++cnt;
          }
        }
      }
    } else {
      if (lane == 0) {
        stk[top + 1] = m.left + 1;
        stk[top + 2] = m.left;
      }
      top += 2;
      __syncwarp();
    }
  }
  if (!FILL && valid) counts[qi] = cnt;
}

// Per-row sort by (d2, id) of the fill output (d2 stored in dist), then sqrt.
// Insertion sort for short rows, heap sort otherwise.
__global__ void k_sort_rows(const int64_t* __restrict__ offsets, int64_t nq,
                            int64_t* __restrict__ idx, double* __restrict__ dist) {
  int64_t qi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  int64_t b = offsets[qi], e = offsets[qi + 1], n = e - b;
  double* D2 = dist + b;
  int64_t* I = idx + b;
  auto lt = [](double d1, int64_t i1, double d2, int64_t i2) {
    return d1 < d2 || (d1 == d2 && i1 < i2);
  };
  if (n <= 32) {
    for (int64_t i = 1; i < n; ++i) {
      double d = D2[i];
      int64_t x = I[i];
      int64_t j = i - 1;
      while (j >= 0 && lt(d, x, D2[j], I[j])) {
        D2[j + 1] = D2[j];
        I[j + 1] = I[j];
        --j;
      }
      D2[j + 1] = d;
      I[j + 1] = x;
    }
  } else {
    auto sift = [&](int64_t i, int64_t end, double d, int64_t x) {
      for (;;) {
        int64_t l = 2 * i + 1;
        if (l >= end) break;
        int64_t c = l;
        if (l + 1 < end && lt(D2[l], I[l], D2[l + 1], I[l + 1])) c = l + 1;
        if (!lt(d, x, D2[c], I[c])) break;
        D2[i] = D2[c];
        I[i] = I[c];
        i = c;
      }
      D2[i] = d;
      I[i] = x;
    };
    for (int64_t i = n / 2 - 1; i >= 0; --i) sift(i, n, D2[i], I[i]);
    for (int64_t end = n - 1; end > 0; --end) {
      double d = D2[end];
      int64_t x = I[end];
      D2[end] = D2[0];
      I[end] = I[0];
      sift(0, end, d, x);
    }
  }
  for (int64_t i = 0; i < n; ++i) D2[i] = sqrt(D2[i]);
}

// ---------------------------------------------------------- heavy ball rows
// Rows with at least kHeavyRow results are filled by a whole warp per query:
// one warp-uniform left-first DFS (stack in shared memory), leaves scanned with
// the lanes over the points (FP64 distances, results compacted in point order by
// ballot prefix), and subtrees whose tight box lies entirely inside the ball
// (box_maxd2 / box_maxd2_near <= r^2) emitted in one coalesced pass over their
// contiguous positions.  The order of a row is the per-lane kernel's: left-first
// DFS, leaf order.
constexpr int64_t kHeavyRow = 256;
constexpr int kHeavyStack = 128;

template <int D, bool PER>
__global__ void __launch_bounds__(128) k_ball_fill_warp(TreeView tv, const double* __restrict__ Q,
                                                        const int32_t* __restrict__ rows,
                                                        const unsigned* __restrict__ n_rows,
                                                        double r2, int32_t* __restrict__ gstack,
                                                        int stack_len,
                                                        const int64_t* __restrict__ offsets,
                                                        int64_t* __restrict__ oidx,
                                                        double* __restrict__ odist, int want_d2) {
  __shared__ int32_t sstk[4][kHeavyStack];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int64_t nrows = (int64_t)*n_rows;
  for (int64_t r = (int64_t)blockIdx.x * nw + w; r < nrows; r += (int64_t)gridDim.x * nw) {
    int32_t* stk = gstack ? gstack + ((int64_t)blockIdx.x * nw + w) * stack_len : sstk[w];
    const int64_t qi = rows[r];
    double q[D];
#pragma unroll
    for (int j = 0; j < D; ++j) q[j] = Q[qi * D + j];
    int64_t cur = offsets[qi];
    const int64_t cur_end = offsets[qi + 1];
    int top = 0;
    if (lane == 0) stk[0] = 0;
    __syncwarp();
    while (top >= 0) {
      const int32_t node = stk[top];
      --top;
      __syncwarp();
      const NodeMeta m = load_meta(tv.meta, node);
      if (!(box_mind2<D, PER>(tv, q, node) <= r2)) continue;
      const bool inside =
          m.left >= 0 && (PER ? box_maxd2_near<D>(tv, q, node) : box_maxd2<D>(tv, q, node)) <= r2;
      if (inside) {  // whole subtree: positions m.start .. m.start + count - 1 in order
        for (int32_t i = lane; i < m.count; i += 32) {
          const int32_t p = m.start + i;
          const int64_t o = cur + i;
          if (o < cur_end) {
            const double d2 = point_d2<D, PER>(tv, q, p);
            oidx[o] = __ldg(&tv.ids[p]);
            odist[o] = want_d2 ? d2 : sqrt(d2);
          }
        }
        cur += m.count;
      } else if (m.left < 0) {
        for (int32_t base = 0; base < m.count; base += 32) {
          const int32_t i = base + lane;
          bool hit = false;
          double d2 = 0.0;
          if (i < m.count) {
            d2 = point_d2<D, PER>(tv, q, m.start + i);
            hit = d2 <= r2;
          }
          const unsigned hm = __ballot_sync(0xffffffffu, hit);
          if (hit) {
            const int64_t o = cur + __popc(hm & lt_mask);
            if (o < cur_end) {
              oidx[o] = __ldg(&tv.ids[m.start + i]);
              odist[o] = want_d2 ? d2 : sqrt(d2);
            }
          }
          cur += __popc(hm);
        }
      } else {
        if (lane == 0) {
          stk[top + 1] = m.left + 1;
          stk[top + 2] = m.left;
        }
        top += 2;
        __syncwarp();
      }
    }
    __syncwarp();
  }
}

// rows of the fill split by length: heavy ones (>= kHeavyRow) to `heavy`, the rest
// to `light`, both in the processing order (`order`, the leaf order when given)
__global__ void k_split_rows(const int64_t* __restrict__ offsets, const int32_t* __restrict__ order,
                             int64_t nq, int32_t* __restrict__ heavy,
                             unsigned* __restrict__ n_heavy, int32_t* __restrict__ light,
                             unsigned* __restrict__ n_light) {
  const int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool valid = slot < nq;
  const int64_t i = valid ? (order ? (int64_t)order[slot] : slot) : 0;
  const bool h = valid && offsets[i + 1] - offsets[i] >= kHeavyRow;
  const unsigned hm = __ballot_sync(0xffffffffu, h);
  const unsigned lm = __ballot_sync(0xffffffffu, valid && !h);
  unsigned hb = 0, lb = 0;
  if (lane == 0) {
    if (hm) hb = atomicAdd(n_heavy, (unsigned)__popc(hm));
    if (lm) lb = atomicAdd(n_light, (unsigned)__popc(lm));
  }
  hb = __shfl_sync(0xffffffffu, hb, 0);
  lb = __shfl_sync(0xffffffffu, lb, 0);
  const unsigned below = (1u << lane) - 1u;
  if (h) heavy[hb + __popc(hm & below)] = (int32_t)i;
  if (valid && !h) light[lb + __popc(lm & below)] = (int32_t)i;
}

// Per-lane box search: each lane walks the tree for its own box with a private
// stack, left child first, so a row comes out in the same order as the packet
// kernel below (left-first DFS, leaf order) without the warp serialising the union
// of 32 boxes' paths.  Stack depth <= tree depth + 1 (<= 2 pushes per pop).
constexpr int kBoxLaneStack = 128;

template <int D, bool FILL>
__global__ void __launch_bounds__(128) k_box_lane(TreeView tv, const double* __restrict__ boxes,
                                                  int64_t nb, int64_t* __restrict__ counts,
                                                  const int64_t* __restrict__ offsets,
                                                  int64_t* __restrict__ oidx,
                                                  const int32_t* __restrict__ broot) {
  const int64_t bi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (bi >= nb) return;
  double lo[D], hi[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    lo[j] = boxes[bi * 2 * D + 2 * j];
    hi[j] = boxes[bi * 2 * D + 2 * j + 1];
  }
  int64_t cnt = 0;
  int64_t cur = FILL ? offsets[bi] : 0;
  const int64_t cur_end = FILL ? offsets[bi + 1] : 0;
  int32_t stk[kBoxLaneStack];
  int top = 0;
  stk[0] = broot ? broot[bi] : 0;
  while (top >= 0) {
    const int32_t node = stk[top--];
    const NodeMeta m = load_meta(tv.meta, node);
    if (m.left < 0) {
      for (int i = 0; i < m.count; ++i) {
        const int32_t p = m.start + i;
        bool in = true;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          const double x = __ldg(&tv.pts[(int64_t)j * tv.n + p]);
          in = in && !(x < lo[j] || x > hi[j]);  // :1319
        }
        if (in) {
          if (FILL) {
            if (cur < cur_end) oidx[cur++] = __ldg(&tv.ids[p]);
          } else {
            ++cnt;
          }
        }
      }
    } else {
      double bl = 0.0, bh = 0.0;
#pragma unroll
      for (int j = 0; j < D; ++j)
        if (j == m.axis) {
          bl = lo[j];
          bh = hi[j];
        }
      if (bh > m.split) stk[++top] = m.left + 1;  // :1300 (visited second)
      if (bl < m.split) stk[++top] = m.left;      // :1296 (visited first)
    }
  }
  if (!FILL) counts[bi] = cnt;
}

// Warp-per-box search for small batches, where one lane per box would leave most
// of the GPU idle and each box would pay one dependent load per visited node.
// The warp expands the frontier of visited nodes one level at a time (every lane
// tests one frontier node with the descent rule of :1296-1300, so a level costs
// one dependent load), keeping the frontier in leaf order: children replace
// their parent, left first, and leaves stay in place (stored as ~id).  The final
// frontier lists the visited leaves in the order of the left-first depth-first
// walk, so every row comes out in the reference's order.  A frontier that
// outgrows its buffer falls back to a depth-first walk with a warp stack.
constexpr int kBoxFront = 256;
constexpr int64_t kBoxWarpMax = 32768;  // boxes per call up to which the warp kernel is used

template <int D, bool FILL>
__global__ void __launch_bounds__(128) k_box_warp(TreeView tv, const double* __restrict__ boxes,
                                                  int64_t nb, int64_t* __restrict__ counts,
                                                  const int64_t* __restrict__ offsets,
                                                  int64_t* __restrict__ oidx,
                                                  const int32_t* __restrict__ broot) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ int32_t front[4][2][kBoxFront];
  __shared__ int32_t stk[4][kBoxLaneStack];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t bi = (int64_t)blockIdx.x * (blockDim.x >> 5) + w;
  if (bi >= nb) return;  // the whole warp leaves together
  double lo[D], hi[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    lo[j] = boxes[bi * 2 * D + 2 * j];
    hi[j] = boxes[bi * 2 * D + 2 * j + 1];
  }
  int64_t cnt = 0;
  int64_t cur = FILL ? offsets[bi] : 0;
  const int64_t cur_end = FILL ? offsets[bi + 1] : 0;
  const int32_t root = broot ? broot[bi] : 0;
  // points of one leaf, tested by the lanes and emitted in position order
  auto scan_leaf = [&](int32_t st, int32_t ct) {
    for (int32_t b = 0; b < ct; b += 32) {
      const int32_t p = st + b + lane;
      bool in = b + lane < ct;
      if (in) {
#pragma unroll
        for (int j = 0; j < D; ++j) {
          const double x = __ldg(&tv.pts[(int64_t)j * tv.n + p]);
          in = in && !(x < lo[j] || x > hi[j]);  // :1319
        }
      }
      const unsigned hm = __ballot_sync(FULL, in);
      if (FILL) {
        if (in) {
          const int64_t o = cur + __popc(hm & lt);
          if (o < cur_end) oidx[o] = __ldg(&tv.ids[p]);
        }
        cur += __popc(hm);
      } else {
        cnt += __popc(hm);
      }
    }
  };
  int nf = 1, fb = 0;
  if (lane == 0) front[w][0][0] = root;
  __syncwarp();
  bool overflow = false;
  for (;;) {
    bool any = false;
    for (int c = lane; c < nf; c += 32) any = any || front[w][fb][c] >= 0;
    if (!__any_sync(FULL, any)) break;
    int nn = 0;
    for (int c0 = 0; c0 < nf; c0 += 32) {
      const int c = c0 + lane;
      int32_t o0 = 0, o1 = 0;
      int kout = 0;
      if (c < nf) {
        const int32_t e = front[w][fb][c];
        if (e < 0) {
          o0 = e;
          kout = 1;
        } else {
          const NodeMeta m = load_meta(tv.meta, e);
          if (m.left < 0) {
            o0 = ~e;
            kout = 1;
          } else {
            double bl = 0.0, bh = 0.0;
#pragma unroll
            for (int j = 0; j < D; ++j)
              if (j == m.axis) {
                bl = lo[j];
                bh = hi[j];
              }
            const bool gl = bl < m.split, gr = bh > m.split;  // :1296, :1300
            o0 = gl ? m.left : m.left + 1;
            o1 = m.left + 1;
            kout = (gl ? 1 : 0) + (gr ? 1 : 0);
          }
        }
      }
      const unsigned b1 = __ballot_sync(FULL, kout >= 1), b2 = __ballot_sync(FULL, kout == 2);
      const int pre = __popc(b1 & lt) + __popc(b2 & lt);
      const int tot = __popc(b1) + __popc(b2);
      if (nn + tot <= kBoxFront) {
        if (kout >= 1) front[w][1 - fb][nn + pre] = o0;
        if (kout == 2) front[w][1 - fb][nn + pre + 1] = o1;
      }
      nn += tot;
    }
    __syncwarp();
    if (nn > kBoxFront) {
      overflow = true;
      break;
    }
    nf = nn;
    fb = 1 - fb;
  }
  if (!overflow) {
    for (int c0 = 0; c0 < nf; c0 += 32) {
      int32_t st_l = 0, ct_l = 0;
      if (c0 + lane < nf) {
        const NodeMeta m = load_meta(tv.meta, ~front[w][fb][c0 + lane]);
        st_l = m.start;
        ct_l = m.count;
      }
      const int nl = min(32, nf - c0);
      for (int i = 0; i < nl; ++i)
        scan_leaf(__shfl_sync(FULL, st_l, i), __shfl_sync(FULL, ct_l, i));
    }
  } else {  // depth-first walk, left child first (stack depth <= tree depth + 2)
    int top = 0;
    if (lane == 0) stk[w][0] = root;
    __syncwarp();
    while (top >= 0) {
      const int32_t node = stk[w][top];
      --top;
      __syncwarp();
      const NodeMeta m = load_meta(tv.meta, node);
      if (m.left < 0) {
        scan_leaf(m.start, m.count);
      } else {
        double bl = 0.0, bh = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j)
          if (j == m.axis) {
            bl = lo[j];
            bh = hi[j];
          }
        const bool gr = bh > m.split, gl = bl < m.split;
        if (lane == 0) {
          if (gr) stk[w][top + 1] = m.left + 1;
          if (gl) stk[w][top + 1 + (gr ? 1 : 0)] = m.left;
        }
        top += (gr ? 1 : 0) + (gl ? 1 : 0);
        __syncwarp();
      }
    }
  }
  if (!FILL && lane == 0) counts[bi] = cnt;
}

template <int D, bool FILL>
__global__ void __launch_bounds__(128) k_box(TreeView tv, const double* __restrict__ boxes,
                                             int64_t nb, int32_t* __restrict__ gstack,
                                             int stack_len, int64_t* __restrict__ counts,
                                             const int64_t* __restrict__ offsets,
                                             int64_t* __restrict__ oidx,
                                             const int32_t* __restrict__ broot) {
  __shared__ int32_t snode[4][kStack];
  __shared__ unsigned smask[4][kStack];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  int32_t* stn = gstack ? gstack + gw * 2 * stack_len : snode[w];
  unsigned* stm = gstack ? reinterpret_cast<unsigned*>(gstack + gw * 2 * stack_len + stack_len)
                         : smask[w];
  int64_t bi = gw * 32 + lane;
  bool valid = bi < nb;
  double lo[D], hi[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    lo[j] = valid ? boxes[bi * 2 * D + 2 * j] : 0.0;
    hi[j] = valid ? boxes[bi * 2 * D + 2 * j + 1] : -1.0;
  }
  const unsigned bit = 1u << lane;
  unsigned vm = __ballot_sync(0xffffffffu, valid);
  int64_t cnt = 0;
  int64_t cur = (FILL && valid) ? offsets[bi] : 0;
  const int64_t cur_end = (FILL && valid) ? offsets[bi + 1] : 0;
  int top = 0;
  if (broot) {
    // forest: one start entry per distinct tree among the warp's boxes
    const int32_t r = valid ? broot[bi] : -1;
    const unsigned same = __match_any_sync(0xffffffffu, r);
    const bool leader = valid && (__ffs(same) - 1) == lane;
    const unsigned lead = __ballot_sync(0xffffffffu, leader);
    if (leader) {
      const int slot = __popc(lead & (bit - 1u));
      stn[slot] = r;
      stm[slot] = same;
    }
    top = __popc(lead) - 1;
  } else if (lane == 0) {
    stn[0] = 0;
    stm[0] = vm;
  }
  __syncwarp();
  while (top >= 0) {
    int32_t node = stn[top];
    unsigned mask = stm[top];
    --top;
    __syncwarp();
    bool mine = (mask & bit) != 0;
    NodeMeta m = load_meta(tv.meta, node);
    if (m.left < 0) {
      for (int i = 0; i < m.count; ++i) {
        int32_t p = m.start + i;
        bool in = mine;
#pragma unroll
        for (int j = 0; j < D; ++j) {
          double x = __ldg(&tv.pts[(int64_t)j * tv.n + p]);
          in = in && !(x < lo[j] || x > hi[j]);  // :1319
        }
        if (in) {
          if (FILL) {
            if (cur < cur_end) oidx[cur++] = __ldg(&tv.ids[p]);
          } else {
            ++cnt;
          }
        }
      }
    } else {
      double bl = 0.0, bh = 0.0;
#pragma unroll
      for (int j = 0; j < D; ++j)
        if (j == m.axis) {
          bl = lo[j];
          bh = hi[j];
        }
      unsigned lm = __ballot_sync(0xffffffffu, mine && bl < m.split);  // :1296
      unsigned rm = __ballot_sync(0xffffffffu, mine && bh > m.split);  // :1300
      if (lane == 0) {
        int t2 = top;
        if (rm) {
          ++t2;
          stn[t2] = m.left + 1;
          stm[t2] = rm;
        }
        if (lm) {
          ++t2;
          stn[t2] = m.left;
          stm[t2] = lm;
        }
      }
      top += (rm ? 1 : 0) + (lm ? 1 : 0);
      __syncwarp();
    }
  }
  if (!FILL && valid) counts[bi] = cnt;
}

template <int D, bool PER>
ckd_status ball_launch(const ckd_tree* t, const double* q, const int32_t* order, int64_t nq,
                       double r, bool fill, int sorted, int64_t* counts, const int64_t* offsets,
                       int64_t* idx, double* dist, cudaStream_t s) {
  TreeView tv = t->view();
  const int threads = 128, nw = threads / 32;
  int64_t warps = cdiv(nq, 32);
  unsigned blocks = (unsigned)cdiv(warps, nw);
  int stack_len = std::max(kStack, t->depth + 4);
  int32_t* gstack = nullptr;
  if (stack_len > kStack)
    CKD_CUDA(dev_alloc((void**)&gstack, sizeof(int32_t) * stack_len * (int64_t)blocks * nw, s));
  double r2 = r * r;  // radius**2 (cosmokdtree.f90:1112)
  if (fill) {
    // heavy rows: a warp per query; light rows: the per-lane kernel over a list
    int32_t *heavy = nullptr, *light = nullptr, *hstack = nullptr;
    unsigned* cnt = nullptr;
    CKD_CUDA(dev_alloc((void**)&heavy, sizeof(int32_t) * nq, s));
    CKD_CUDA(dev_alloc((void**)&light, sizeof(int32_t) * nq, s));
    CKD_CUDA(dev_alloc((void**)&cnt, 2 * sizeof(unsigned), s));
    CKD_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), s));
    k_split_rows<<<(unsigned)cdiv(nq, 256), 256, 0, s>>>(offsets, order, nq, heavy, cnt, light,
                                                         cnt + 1);
    CKD_LAUNCH_CHECK();
    k_ball<D, PER, true><<<blocks, threads, 0, s>>>(tv, q, light, nq, cnt + 1, r2, gstack,
                                                     stack_len, nullptr, offsets, idx, dist,
                                                     sorted ? 1 : 0);
    CKD_LAUNCH_CHECK();
    int dev = 0, sms = 148;
    CKD_CUDA(cudaGetDevice(&dev));
    CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t hblocks = std::min<int64_t>(cdiv(nq, 4), (int64_t)sms * 8);
    const int hstack_len = std::max(kHeavyStack, t->depth + 4);
    if (hstack_len > kHeavyStack)
      CKD_CUDA(dev_alloc((void**)&hstack, sizeof(int32_t) * hstack_len * hblocks * 4, s));
    k_ball_fill_warp<D, PER><<<(unsigned)std::max<int64_t>(1, hblocks), 128, 0, s>>>(
        tv, q, heavy, cnt, r2, hstack, hstack_len, offsets, idx, dist, sorted ? 1 : 0);
    CKD_LAUNCH_CHECK();
    for (void* p : {(void*)heavy, (void*)light, (void*)cnt, (void*)hstack}) dev_free(p, s);
  } else {
    k_ball<D, PER, false><<<blocks, threads, 0, s>>>(tv, q, order, nq, nullptr, r2, gstack,
                                                      stack_len, counts, nullptr, nullptr, nullptr,
                                                      0);
    CKD_LAUNCH_CHECK();
  }
  if (fill && sorted) {
    k_sort_rows<<<(unsigned)cdiv(nq, 128), 128, 0, s>>>(offsets, nq, idx, dist);
    CKD_LAUNCH_CHECK();
  }
  if (gstack) CKD_CUDA(dev_free(gstack, s));
  return CKD_OK;
}

template <int D>
ckd_status box_launch(const ckd_tree* t, const double* boxes, int64_t nb, bool fill,
                      int64_t* counts, const int64_t* offsets, int64_t* idx, cudaStream_t s,
                      const int32_t* broot) {
  TreeView tv = t->view();
  const int threads = 128, nw = threads / 32;
  if (t->depth < kBoxLaneStack - 2 && nb <= kBoxWarpMax && box_warp_enabled()) {
    const unsigned wb = (unsigned)cdiv(nb, nw);
    if (fill)
      k_box_warp<D, true><<<wb, threads, 0, s>>>(tv, boxes, nb, nullptr, offsets, idx, broot);
    else
      k_box_warp<D, false><<<wb, threads, 0, s>>>(tv, boxes, nb, counts, nullptr, nullptr, broot);
    CKD_LAUNCH_CHECK();
    return CKD_OK;
  }
  if (t->depth < kBoxLaneStack - 2) {
    const unsigned lb = (unsigned)cdiv(nb, threads);
    if (fill)
      k_box_lane<D, true><<<lb, threads, 0, s>>>(tv, boxes, nb, nullptr, offsets, idx, broot);
    else
      k_box_lane<D, false><<<lb, threads, 0, s>>>(tv, boxes, nb, counts, nullptr, nullptr, broot);
    CKD_LAUNCH_CHECK();
    return CKD_OK;
  }
  int64_t warps = cdiv(nb, 32);
  unsigned blocks = (unsigned)cdiv(warps, nw);
  // a packet stack grows by at most one entry per level past its start entries
  int stack_len = std::max(kStack, t->depth + 4 + (broot ? 32 : 0));
  int32_t* gstack = nullptr;
  if (stack_len > kStack)
    CKD_CUDA(dev_alloc((void**)&gstack, sizeof(int32_t) * 2 * stack_len * (int64_t)blocks * nw, s));
  if (fill)
    k_box<D, true><<<blocks, threads, 0, s>>>(tv, boxes, nb, gstack, stack_len, nullptr, offsets,
                                              idx, broot);
  else
    k_box<D, false><<<blocks, threads, 0, s>>>(tv, boxes, nb, gstack, stack_len, counts, nullptr,
                                               nullptr, broot);
  CKD_LAUNCH_CHECK();
  if (gstack) CKD_CUDA(dev_free(gstack, s));
  return CKD_OK;
}

}  // namespace

bool want_order(const ckd_tree* t, int64_t nq);

ckd_status ball_run(const ckd_tree* t, const double* q, int64_t nq, double r, bool fill, int sorted,
                    int64_t* counts, const int64_t* offsets, int64_t* idx, double* dist,
                    cudaStream_t s) {
  int32_t* order = nullptr;
  if (want_order(t, nq)) {
    CKD_CUDA(dev_alloc((void**)&order, sizeof(int32_t) * nq, s));
    CKD_TRY(query_order(t, q, nq, order, s));
  }
  ckd_status st;
#define CKD_BALL_CASE(DD)                                                                      \
  case DD:                                                                                     \
    st = t->periodic ? ball_launch<DD, true>(t, q, order, nq, r, fill, sorted, counts, offsets, \
                                             idx, dist, s)                                     \
                     : ball_launch<DD, false>(t, q, order, nq, r, fill, sorted, counts,         \
                                              offsets, idx, dist, s);                          \
    break;
  switch (t->d) {
    CKD_BALL_CASE(1)
    CKD_BALL_CASE(2)
    CKD_BALL_CASE(3)
    CKD_BALL_CASE(4)
    CKD_BALL_CASE(5)
    CKD_BALL_CASE(6)
    CKD_BALL_CASE(7)
    CKD_BALL_CASE(8)
    default: st = fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
  }
#undef CKD_BALL_CASE
  if (order) dev_free(order, s);
  return st;
}

ckd_status box_run(const ckd_tree* t, const double* boxes, int64_t nb, bool fill, int64_t* counts,
                   const int64_t* offsets, int64_t* idx, cudaStream_t s, const int32_t* broot) {
  switch (t->d) {
    case 1: return box_launch<1>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
    case 2: return box_launch<2>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
    case 3: return box_launch<3>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
    case 4: return box_launch<4>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
    case 5: return box_launch<5>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
    case 6: return box_launch<6>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
    case 7: return box_launch<7>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
    case 8: return box_launch<8>(t, boxes, nb, fill, counts, offsets, idx, s, broot);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

}  // namespace ckd
