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

template <int D, bool PER, bool FILL, bool ROOTS = false>
__global__ void __launch_bounds__(128) k_ball(TreeView tv, const double* __restrict__ Q,
                                              const int32_t* __restrict__ order, int64_t nq_max,
                                              const unsigned* __restrict__ nq_dev,
                                              double r2, int32_t* __restrict__ gstack,
                                              int stack_len, int64_t* __restrict__ counts,
                                              const int64_t* __restrict__ offsets,
                                              int64_t* __restrict__ oidx,
                                              double* __restrict__ odist, int want_d2,
                                              const int32_t* __restrict__ qroot) {
  // packet stack entries; with ROOTS (forests) each entry also carries the lanes
  // whose balls reached its parent, and the search starts one entry per distinct
  // root among the warp's queries
  __shared__ int32_t sstk[4][kStack];
  __shared__ unsigned smsk[4][ROOTS ? kStack : 1];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t gw = (int64_t)blockIdx.x * nw + w;
  int32_t* stk = gstack ? gstack + gw * 2 * stack_len : sstk[w];
  unsigned* msk = gstack && ROOTS
                      ? reinterpret_cast<unsigned*>(gstack + gw * 2 * stack_len + stack_len)
                      : smsk[w];
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
  if (ROOTS) {
    const int32_t root = valid ? qroot[qi] : -1;
    const unsigned grp = __match_any_sync(0xffffffffu, root);
    const bool leader = valid && lane == __ffs(grp) - 1;
    const unsigned leaders = __ballot_sync(0xffffffffu, leader);
    if (leader) {
      const int e = __popc(leaders & ((1u << lane) - 1u));
      stk[e] = root;
      msk[e] = grp;
    }
    top = __popc(leaders) - 1;
  } else if (lane == 0) {
    stk[0] = 0;
  }
  __syncwarp();
  while (top >= 0) {
    int32_t node = stk[top];
    const unsigned em = ROOTS ? msk[top] : 0xffffffffu;
    --top;
    __syncwarp();
    NodeMeta m = load_meta(tv.meta, node);
    bool need = ((em >> lane) & 1u) && box_mind2<D, PER>(tv, q, node) <= rr;
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
        if (ROOTS) {
          msk[top + 1] = nm;
          msk[top + 2] = nm;
        }
      }
      top += 2;
      __syncwarp();
    }
  }
  if (!FILL && valid) counts[qi] = cnt;
}

__device__ __forceinline__ bool key_lt(double d1, int64_t i1, double d2, int64_t i2) {
  return d1 < d2 || (d1 == d2 && i1 < i2);
}

// Per-row sort by (d2, id) of the fill output (d2 stored in dist), then sqrt.
// Rows of at most 32 results: insertion sort by their own thread.  Longer rows
// are listed for k_sort_big (a block per row), with a scratch range for the
// rows longer than one shared-memory tile.
constexpr int kSortTile = 2048;
__global__ void k_sort_rows(const int64_t* __restrict__ offsets, int64_t nq,
                            int64_t* __restrict__ idx, double* __restrict__ dist,
                            int32_t* __restrict__ big, unsigned long long* __restrict__ sel,
                            int64_t* __restrict__ tmp_off) {
  int64_t qi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nq) return;
  int64_t b = offsets[qi], e = offsets[qi + 1], n = e - b;
  if (n > 32) {
    const unsigned long long slot = atomicAdd(&sel[0], 1ull);
    big[slot] = (int32_t)qi;
    tmp_off[slot] = n > kSortTile ? (int64_t)atomicAdd(&sel[1], (unsigned long long)n) : 0;
    return;
  }
  double* D2 = dist + b;
  int64_t* I = idx + b;
  for (int64_t i = 1; i < n; ++i) {
    double d = D2[i];
    int64_t x = I[i];
    int64_t j = i - 1;
    while (j >= 0 && key_lt(d, x, D2[j], I[j])) {
      D2[j + 1] = D2[j];
      I[j + 1] = I[j];
      --j;
    }
    D2[j + 1] = d;
    I[j + 1] = x;
  }
  for (int64_t i = 0; i < n; ++i) D2[i] = sqrt(D2[i]);
}

// A block per listed row: tiles of kSortTile sorted in shared memory (bitonic),
// then merge passes of doubling width between the row and its scratch range
// (merge path: each thread finds where its 8 outputs start by binary search).
// Keys (d2, id) are distinct within a row, so the order is total.
__global__ void __launch_bounds__(256) k_sort_big(const int64_t* __restrict__ offsets,
                                                  const int32_t* __restrict__ big,
                                                  const unsigned long long* __restrict__ sel,
                                                  const int64_t* __restrict__ tmp_off,
                                                  int64_t* __restrict__ idx,
                                                  double* __restrict__ dist,
                                                  int64_t* __restrict__ tidx,
                                                  double* __restrict__ tdist) {
  __shared__ double sk[kSortTile];
  __shared__ int64_t si[kSortTile];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int64_t nbig = (int64_t)sel[0];
  for (int64_t r = blockIdx.x; r < nbig; r += gridDim.x) {
    const int32_t qi = big[r];
    const int64_t b = offsets[qi], n = offsets[qi + 1] - b;
    double* D2 = dist + b;
    int64_t* I = idx + b;
    for (int64_t t0 = 0; t0 < n; t0 += kSortTile) {
      const int m = (int)min((int64_t)kSortTile, n - t0);
      int P = 1;
      while (P < m) P <<= 1;
      for (int i = tid; i < P; i += nt) {
        sk[i] = i < m ? D2[t0 + i] : INFINITY;
        si[i] = i < m ? I[t0 + i] : INT64_MAX;
      }
      __syncthreads();
      for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int i = tid; i < P; i += nt) {
            const int ixj = i ^ j;
            if (ixj > i) {
              const bool up = (i & k) == 0;
              if (key_lt(sk[ixj], si[ixj], sk[i], si[i]) == up) {
                const double td = sk[i];
                const int64_t ti = si[i];
                sk[i] = sk[ixj];
                si[i] = si[ixj];
                sk[ixj] = td;
                si[ixj] = ti;
              }
            }
          }
          __syncthreads();
        }
      for (int i = tid; i < m; i += nt) {
        D2[t0 + i] = sk[i];
        I[t0 + i] = si[i];
      }
      __syncthreads();
    }
    if (n > kSortTile) {
      double* sD = D2;
      int64_t* sI = I;
      double* dD = tdist + tmp_off[r];
      int64_t* dI = tidx + tmp_off[r];
      for (int64_t w = kSortTile; w < n; w <<= 1) {
        for (int64_t s0 = 0; s0 < n; s0 += 2 * w) {
          const int64_t na = min(w, n - s0);
          const int64_t nb = max((int64_t)0, min(w, n - s0 - w));
          const double* AD = sD + s0;
          const int64_t* AI = sI + s0;
          const double* BD = AD + na;
          const int64_t* BI = AI + na;
          const int64_t mt = na + nb;
          for (int64_t k0 = (int64_t)tid * 8; k0 < mt; k0 += (int64_t)nt * 8) {
            int64_t lo = max((int64_t)0, k0 - nb), hi = min(k0, na);
            while (lo < hi) {
              const int64_t mid = (lo + hi) >> 1;
              if (key_lt(AD[mid], AI[mid], BD[k0 - 1 - mid], BI[k0 - 1 - mid])) lo = mid + 1;
              else hi = mid;
            }
            int64_t i = lo, j = k0 - lo;
            const int64_t kend = min(k0 + 8, mt);
            for (int64_t k = k0; k < kend; ++k) {
              const bool ta = j >= nb || (i < na && key_lt(AD[i], AI[i], BD[j], BI[j]));
              if (ta) {
                dD[s0 + k] = AD[i];
                dI[s0 + k] = AI[i];
                ++i;
              } else {
                dD[s0 + k] = BD[j];
                dI[s0 + k] = BI[j];
                ++j;
              }
            }
          }
        }
        __syncthreads();
        double* tD = sD;
        sD = dD;
        dD = tD;
        int64_t* tI = sI;
        sI = dI;
        dI = tI;
      }
      if (sD != D2)
        for (int64_t i = tid; i < n; i += nt) {
          D2[i] = sD[i];
          I[i] = sI[i];
        }
      __syncthreads();
    }
    for (int64_t i = tid; i < n; i += nt) D2[i] = sqrt(D2[i]);
    __syncthreads();
  }
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

// A whole subtree of at least kTaskMin points inside a heavy row's ball is not
// copied by the warp that found it but recorded as emission tasks of at most
// kTaskChunk points, which k_ball_emit spreads over the whole GPU: a row of
// millions of points no longer serialises on one warp.  When the task buffer is
// full the warp copies the subtree itself (same output).
constexpr int32_t kTaskMin = 1024;
constexpr int32_t kTaskChunk = 4096;
constexpr unsigned kTaskCap = 1u << 20;
struct EmitTask {
  int64_t out;  // first output slot
  int32_t start, count, qi, pad;
};

template <int D, bool PER>
__global__ void __launch_bounds__(128) k_ball_fill_warp(TreeView tv, const double* __restrict__ Q,
                                                        const int32_t* __restrict__ rows,
                                                        const unsigned* __restrict__ n_rows,
                                                        double r2, int32_t* __restrict__ gstack,
                                                        int stack_len,
                                                        const int64_t* __restrict__ offsets,
                                                        int64_t* __restrict__ oidx,
                                                        double* __restrict__ odist, int want_d2,
                                                        EmitTask* __restrict__ tasks,
                                                        unsigned* __restrict__ n_tasks,
                                                        const int32_t* __restrict__ qroot) {
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
    if (lane == 0) stk[0] = qroot ? qroot[qi] : 0;
    __syncwarp();
    while (top >= 0) {
      const int32_t node = stk[top];
      --top;
      __syncwarp();
      const NodeMeta m = load_meta(tv.meta, node);
      if (!(box_mind2<D, PER>(tv, q, node) <= r2)) continue;
      const bool inside =
          m.left >= 0 && (PER ? box_maxd2_near<D>(tv, q, node) : box_maxd2<D>(tv, q, node)) <= r2;
      if (inside && tasks && m.count >= kTaskMin && cur < cur_end) {
        const int64_t len = min((int64_t)m.count, cur_end - cur);
        const unsigned nt = (unsigned)((len + kTaskChunk - 1) / kTaskChunk);
        unsigned tb = 0;
        if (lane == 0) tb = atomicAdd(n_tasks, nt);
        tb = __shfl_sync(0xffffffffu, tb, 0);
        if (tb + nt <= kTaskCap) {
          for (unsigned c = lane; c < nt; c += 32) {
            EmitTask e;
            e.out = cur + (int64_t)c * kTaskChunk;
            e.start = m.start + (int32_t)c * kTaskChunk;
            e.count = (int32_t)min((int64_t)kTaskChunk, len - (int64_t)c * kTaskChunk);
            e.qi = (int32_t)qi;
            e.pad = 0;
            tasks[tb + c] = e;
          }
          cur += m.count;
          continue;
        }
      }
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

// Copies of the recorded whole-subtree chunks, a warp per chunk.
template <int D, bool PER>
__global__ void __launch_bounds__(128) k_ball_emit(TreeView tv, const double* __restrict__ Q,
                                                   const EmitTask* __restrict__ tasks,
                                                   const unsigned* __restrict__ n_tasks,
                                                   int64_t* __restrict__ oidx,
                                                   double* __restrict__ odist, int want_d2) {
  const int lane = threadIdx.x & 31;
  const int64_t nt = min((int64_t)*n_tasks, (int64_t)kTaskCap);
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < nt;
       t += nwarps) {
    const EmitTask e = tasks[t];
    double q[D];
#pragma unroll
    for (int j = 0; j < D; ++j) q[j] = Q[(int64_t)e.qi * D + j];
#pragma unroll 4
    for (int32_t i = lane; i < e.count; i += 32) {
      const int32_t p = e.start + i;
      const double d2 = point_d2<D, PER>(tv, q, p);
      oidx[e.out + i] = __ldg(&tv.ids[p]);
      odist[e.out + i] = want_d2 ? d2 : sqrt(d2);
    }
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
// A subtree of at least this many points whose split the box straddles (both
// children would be visited) is tested against the box as a whole: when
// its tight bounding box lies strictly inside the query box, every split below it
// lies strictly inside too (a sliding-midpoint split lies between, or on, its node's
// points), so the strict descent (:1296-1300) reaches every leaf and the inclusive
// test (:1319) accepts every point: the subtree's whole leaf-ordered range is the
// answer, in the depth-first order of its leaves.
constexpr int32_t kBoxWholeMin = 64;
template <int D>
__device__ __forceinline__ bool box_holds_node(const TreeView& tv, int32_t node,
                                               const double (&lo)[D], const double (&hi)[D]) {
  const double* b = tv.box + (int64_t)node * 2 * D;
  bool in = true;
#pragma unroll
  for (int j = 0; j < D; ++j) in = in && lo[j] < __ldg(b + 2 * j) && __ldg(b + 2 * j + 1) < hi[j];
  return in;
}

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
      const bool gl = bl < m.split, gr = bh > m.split;
      if (gl && gr && m.count >= kBoxWholeMin && box_holds_node<D>(tv, node, lo, hi)) {
        if (FILL) {
          for (int i = 0; i < m.count && cur < cur_end; ++i)
            oidx[cur++] = __ldg(&tv.ids[m.start + i]);
        } else {
          cnt += m.count;
        }
        continue;
      }
      if (gr) stk[++top] = m.left + 1;  // :1300 (visited second)
      if (gl) stk[++top] = m.left;      // :1296 (visited first)
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
// Boxes per call up to which the warp kernel is used on a single tree; beyond, a lane
// per box is faster for evenly filled boxes (2^20 boxes of side 0.005 on 2^20 uniform
// points: 0.80 vs 4.8 ms).  Forest boxes always take the warp kernel: their trees are
// clusters whose central boxes hold most of the points, and a lane per box leaves the
// whole search waiting on the heaviest lanes (128k boxes on 2000 NFW trees: 25.4 vs
// 40.8 ms, and 11.8 ms with the whole-subtree ranges above).
constexpr int64_t kBoxWarpMax = 32768;

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
  // points of one leaf, tested by the lanes and emitted in position order; a
  // subtree inside the box (whole) is counted or emitted without the tests
  auto scan_leaf = [&](int32_t st, int32_t ct, bool whole) {
    if (!FILL && whole) {
      cnt += ct;
      return;
    }
    for (int32_t b = 0; b < ct; b += 32) {
      const int32_t p = st + b + lane;
      bool in = b + lane < ct;
      if (in && !whole) {
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
            if (gl && gr && m.count >= kBoxWholeMin && box_holds_node<D>(tv, e, lo, hi)) {
              o0 = ~e;  // a subtree inside the box: scanned as one range, like a leaf
              kout = 1;
            } else {
              o0 = gl ? m.left : m.left + 1;
              o1 = m.left + 1;
              kout = (gl ? 1 : 0) + (gr ? 1 : 0);
            }
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
      int32_t st_l = 0, ct_l = 0, wh_l = 0;
      if (c0 + lane < nf) {
        const NodeMeta m = load_meta(tv.meta, ~front[w][fb][c0 + lane]);
        st_l = m.start;
        ct_l = m.count;
        wh_l = m.left >= 0;  // an internal node in the frontier lies inside the box
      }
      const int nl = min(32, nf - c0);
      for (int i = 0; i < nl; ++i)
        scan_leaf(__shfl_sync(FULL, st_l, i), __shfl_sync(FULL, ct_l, i),
                  __shfl_sync(FULL, wh_l, i) != 0);
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
        scan_leaf(m.start, m.count, false);
      } else {
        double bl = 0.0, bh = 0.0;
#pragma unroll
        for (int j = 0; j < D; ++j)
          if (j == m.axis) {
            bl = lo[j];
            bh = hi[j];
          }
        const bool gr = bh > m.split, gl = bl < m.split;
        if (gl && gr && m.count >= kBoxWholeMin && box_holds_node<D>(tv, node, lo, hi)) {
          scan_leaf(m.start, m.count, true);
          continue;
        }
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
                       int64_t* idx, double* dist, cudaStream_t s, const int32_t* qroot) {
  TreeView tv = t->view();
  const int threads = 128, nw = threads / 32;
  int64_t warps = cdiv(nq, 32);
  unsigned blocks = (unsigned)cdiv(warps, nw);
  // a packet stack holds at most one pending sibling per level, plus the roots
  int stack_len = std::max(kStack, t->depth + 4 + (qroot ? 32 : 0));
  Scratch sc(s);
  int32_t* gstack = nullptr;
  if (stack_len > kStack)
    CKD_CUDA(sc.alloc(&gstack, sizeof(int32_t) * 2 * stack_len * (int64_t)blocks * nw));
  double r2 = r * r;  // radius**2 (cosmokdtree.f90:1112)
  if (fill) {
    // heavy rows: a warp per query; light rows: the per-lane kernel over a list
    int32_t *heavy = nullptr, *light = nullptr, *hstack = nullptr;
    unsigned* cnt = nullptr;
    CKD_CUDA(sc.alloc(&heavy, sizeof(int32_t) * nq));
    CKD_CUDA(sc.alloc(&light, sizeof(int32_t) * nq));
    CKD_CUDA(sc.alloc(&cnt, 2 * sizeof(unsigned)));
    CKD_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), s));
    k_split_rows<<<(unsigned)cdiv(nq, 256), 256, 0, s>>>(offsets, order, nq, heavy, cnt, light,
                                                         cnt + 1);
    CKD_LAUNCH_CHECK();
    if (qroot)
      k_ball<D, PER, true, true><<<blocks, threads, 0, s>>>(tv, q, light, nq, cnt + 1, r2, gstack,
                                                            stack_len, nullptr, offsets, idx,
                                                            dist, sorted ? 1 : 0, qroot);
    else
      k_ball<D, PER, true><<<blocks, threads, 0, s>>>(tv, q, light, nq, cnt + 1, r2, gstack,
                                                       stack_len, nullptr, offsets, idx, dist,
                                                       sorted ? 1 : 0, nullptr);
    CKD_LAUNCH_CHECK();
    int dev = 0, sms = 148;
    CKD_CUDA(cudaGetDevice(&dev));
    CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t hblocks = std::min<int64_t>(cdiv(nq, 4), (int64_t)sms * 8);
    const int hstack_len = std::max(kHeavyStack, t->depth + 4);
    if (hstack_len > kHeavyStack)
      CKD_CUDA(sc.alloc(&hstack, sizeof(int32_t) * hstack_len * hblocks * 4));
    EmitTask* tasks = nullptr;
    unsigned* ntask = nullptr;
    CKD_CUDA(sc.alloc(&tasks, sizeof(EmitTask) * kTaskCap));
    CKD_CUDA(sc.alloc(&ntask, sizeof(unsigned)));
    CKD_CUDA(cudaMemsetAsync(ntask, 0, sizeof(unsigned), s));
    k_ball_fill_warp<D, PER><<<(unsigned)std::max<int64_t>(1, hblocks), 128, 0, s>>>(
        tv, q, heavy, cnt, r2, hstack, hstack_len, offsets, idx, dist, sorted ? 1 : 0, tasks,
        ntask, qroot);
    CKD_LAUNCH_CHECK();
    k_ball_emit<D, PER><<<(unsigned)sms * 8, 128, 0, s>>>(tv, q, tasks, ntask, idx, dist,
                                                          sorted ? 1 : 0);
    CKD_LAUNCH_CHECK();
  } else {
    if (qroot)
      k_ball<D, PER, false, true><<<blocks, threads, 0, s>>>(tv, q, order, nq, nullptr, r2,
                                                             gstack, stack_len, counts, nullptr,
                                                             nullptr, nullptr, 0, qroot);
    else
      k_ball<D, PER, false><<<blocks, threads, 0, s>>>(tv, q, order, nq, nullptr, r2, gstack,
                                                        stack_len, counts, nullptr, nullptr,
                                                        nullptr, 0, nullptr);
    CKD_LAUNCH_CHECK();
  }
  if (fill && sorted) {
    int32_t* big = nullptr;
    int64_t* toff = nullptr;
    unsigned long long* sel = nullptr;
    CKD_CUDA(sc.alloc(&big, sizeof(int32_t) * nq));
    CKD_CUDA(sc.alloc(&toff, sizeof(int64_t) * nq));
    CKD_CUDA(sc.alloc(&sel, 2 * sizeof(unsigned long long)));
    CKD_CUDA(cudaMemsetAsync(sel, 0, 2 * sizeof(unsigned long long), s));
    k_sort_rows<<<(unsigned)cdiv(nq, 128), 128, 0, s>>>(offsets, nq, idx, dist, big, sel, toff);
    CKD_LAUNCH_CHECK();
    unsigned long long hs[2] = {0, 0};
    CKD_CUDA(cudaMemcpyAsync(hs, sel, sizeof(hs), cudaMemcpyDeviceToHost, s));
    CKD_CUDA(cudaStreamSynchronize(s));
    if (hs[0] > 0) {
      int64_t* tidx = nullptr;
      double* tdist = nullptr;
      if (hs[1] > 0) {
        CKD_CUDA(sc.alloc(&tidx, sizeof(int64_t) * hs[1]));
        CKD_CUDA(sc.alloc(&tdist, sizeof(double) * hs[1]));
      }
      int dev = 0, sms = 148;
      CKD_CUDA(cudaGetDevice(&dev));
      CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      const unsigned g = (unsigned)std::min<unsigned long long>(hs[0], (unsigned long long)sms * 8);
      k_sort_big<<<g, 256, 0, s>>>(offsets, big, sel, toff, idx, dist, tidx, tdist);
      CKD_LAUNCH_CHECK();
    }
  }
  return CKD_OK;
}

template <int D>
ckd_status box_launch(const ckd_tree* t, const double* boxes, int64_t nb, bool fill,
                      int64_t* counts, const int64_t* offsets, int64_t* idx, cudaStream_t s,
                      const int32_t* broot) {
  TreeView tv = t->view();
  const int threads = 128, nw = threads / 32;
  if (t->depth < kBoxLaneStack - 2 && (nb <= kBoxWarpMax || broot) && box_warp_enabled()) {
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
  Scratch sc(s);
  int32_t* gstack = nullptr;
  if (stack_len > kStack)
    CKD_CUDA(sc.alloc(&gstack, sizeof(int32_t) * 2 * stack_len * (int64_t)blocks * nw));
  if (fill)
    k_box<D, true><<<blocks, threads, 0, s>>>(tv, boxes, nb, gstack, stack_len, nullptr, offsets,
                                              idx, broot);
  else
    k_box<D, false><<<blocks, threads, 0, s>>>(tv, boxes, nb, gstack, stack_len, counts, nullptr,
                                               nullptr, broot);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

}  // namespace

bool want_order(const ckd_tree* t, int64_t nq);
ckd_status query_order_roots(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                             const int32_t* qroot, cudaStream_t s);

ckd_status ball_run(const ckd_tree* t, const double* q, int64_t nq, double r, bool fill, int sorted,
                    int64_t* counts, const int64_t* offsets, int64_t* idx, double* dist,
                    cudaStream_t s, const int32_t* qroot) {
  int32_t* order = nullptr;
  Scratch sc(s);
  if (want_order(t, nq)) {
    CKD_CUDA(sc.alloc(&order, sizeof(int32_t) * nq));
    CKD_TRY(query_order_roots(t, q, nq, order, qroot, s));
  }
  ckd_status st;
#define CKD_BALL_CASE(DD)                                                                      \
  case DD:                                                                                     \
    st = t->periodic ? ball_launch<DD, true>(t, q, order, nq, r, fill, sorted, counts, offsets, \
                                             idx, dist, s, qroot)                              \
                     : ball_launch<DD, false>(t, q, order, nq, r, fill, sorted, counts,         \
                                              offsets, idx, dist, s, qroot);                   \
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
