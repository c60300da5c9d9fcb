// forest_pk.cu -- a forest of independent trees built and queried by ONE persistent
// launch that pulls its work from a device queue.
//
// The reference builds one tree per call (src/cosmokdtree.f90:124-238; the box side
// is a module global, :87) and answers every query with its own traversal
// (:504-540).  Catalogues of thousands of small, uneven trees (haloes,
// subvolumes) would leave the GPU idle between per-tree launches, so here every
// CTA of one resident grid takes items from a queue in global memory:
//
//   (tree t, level l, group g)  split open nodes of tree t at depth l: the
//       sliding-midpoint rule of cosmokdtree.f90:347-410 (longest cell side,
//       ties to the larger spread, midpoint, slide to the extreme point when a
//       side would be empty) and a stable partition (:455-497 up to the order of
//       equal keys, which is canonical here: the lowest original index first).
//       A level is cut into groups (one open node of 2048+ points, split by the
//       whole CTA, or up to 128 smaller nodes, a warp each) so that the levels
//       of large trees spread over many CTAs.  The last group of a level to
//       finish pushes the next level's groups, or, when no node is left open,
//       tree t's query blocks.
//   (tree t, query block b)  the exact kNN of up to `qblock` of t's queries:
//       one query per lane, the per-lane traversal with the compact heap
//       (ckd_knn_lane.cuh) started at t's root.
//
// An item is pushed only after everything it reads has been written (fenced), so
// no item ever waits for another.  CTAs that find the queue empty poll it until
// every pushed item has finished; each poll sleeps and the polling is bounded:
// past the limit the CTA records CKD_ERR_TIMEOUT and returns, and the others stop
// at their next poll.  Trees come out exactly as ckd_forest_build makes them
// (same splits, same leaf sets, same leaf order), so every search gives the same
// results; node ids differ (children pairs are handed out as levels finish).
//
// Tree records written in this launch are read back in it through L2 (__ldcg,
// and CKD_TREE_LOADS_L2 for the shared search helpers): an SM's L1 is not
// coherent with other SMs' stores.
#define CKD_TREE_LOADS_L2
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ckd_common.cuh"
#include "ckd_knn.cuh"
#include "ckd_knn_lane.cuh"

namespace ckd {

ckd_status forest_pk_limits(int k, int d);

namespace {

constexpr int kPkThreads = 128;
constexpr int kPkWarps = kPkThreads / 32;
constexpr int kPkItems = 4;          // positions per thread per pass of a CTA-wide split
constexpr int kBigNode = 2048;       // nodes this large are split by the whole CTA
constexpr int kPkMaxDepth = kLaneStack - 2;  // deepest node the per-lane search can hold
constexpr int kPkMaxLevels = 256;    // deepest level a tree may reach
constexpr int kPkGroupNodes = 128;   // small open nodes per group item of a level
constexpr int kPkMaxGroups = 512;    // group items per level of one tree
constexpr unsigned long long kItemBuild = 1ull, kItemQuery = 2ull;

struct PkState {
  unsigned long long head;  // next queue slot to claim
  unsigned long long tail;  // next queue slot to fill
  long long outstanding;    // items pushed (or withheld) and not finished
  int error;                // first failure (ckd_status), 0 = none
  int nodes;                // node ids handed out (roots 0..T-1 first)
  int max_depth;
  int n_leaves;
  int pad[2];
};

struct PkArgs {
  TreeView tv;          // read side of the forest (records read through L2)
  NodeMeta* meta;
  double* box;
  double* cell;
  float* box32;
  float* cell32;
  double* centre;
  float4* pair;
  double* pts;
  int32_t* ids;
  float4* pts32;
  double4* pts64;
  int32_t* ext;         // [node][2d]: first position of the minimum / maximum per axis
  double* X[2];         // working copies of the points being split (SoA, stride n)
  int32_t* I[2];
  int32_t* lists;       // per tree: two halves of open-node ids (big from the front)
  const int64_t* lbase; // per tree: offset of its halves in `lists`
  int2* tcnt;           // per tree, per level parity: (big, small) open nodes listed
  int32_t* tdone;       // per tree: group items of its current level that finished
  float* tslack;        // [tree][d]: screen slack of the tree (max |coordinate| + L)
  const int64_t* off;   // point offsets (T + 1)
  const int64_t* qoff;  // query offsets (T + 1)
  const double* Q;      // queries, row-major (nq, d), grouped by tree
  double* dist;
  int64_t* idx;
  unsigned long long* queue;
  PkState* st;
  int64_t queue_cap;
  long long spin_limit;  // polls (each ~256 ns asleep) before giving up
  int T;
  int leaf;
  int k;
  int sorted;
  int qblock;
  int node_cap;
};

__device__ __forceinline__ int pk_error(const PkArgs& a) {
  return *reinterpret_cast<volatile int*>(&a.st->error);
}
__device__ __forceinline__ void pk_fail(const PkArgs& a, int code) {
  atomicCAS(&a.st->error, 0, code);
}

__device__ __forceinline__ unsigned long long pk_item(unsigned long long type, int t, uint32_t pl) {
  return (type << 62) | ((unsigned long long)(uint32_t)t << 32) | pl;
}

// Push `m` items (called by one thread; `outstanding` was raised beforehand).
__device__ void pk_push(const PkArgs& a, unsigned long long type, int t, uint32_t first, uint32_t m) {
  const unsigned long long pos = atomicAdd(&a.st->tail, (unsigned long long)m);
  if (pos + m > (unsigned long long)a.queue_cap) {
    pk_fail(a, CKD_ERR_OOM);
    return;
  }
  for (uint32_t i = 0; i < m; ++i) {
    __threadfence();
    atomicExch(&a.queue[pos + i], pk_item(type, t, first + i));
  }
}

// Claim the next item (thread 0).  0: stop (all done, an error, or timeout).
__device__ unsigned long long pk_claim(const PkArgs& a) {
  volatile unsigned long long* vq = a.queue;
  for (long long it = 0; it < a.spin_limit; ++it) {
    if (pk_error(a)) return 0;
    const unsigned long long h = atomicAdd(&a.st->head, 0ull);
    const unsigned long long tl = atomicAdd(&a.st->tail, 0ull);
    if (h < tl) {
      if (h >= (unsigned long long)a.queue_cap) {  // only after a failed push
        pk_fail(a, CKD_ERR_OOM);
        return 0;
      }
      if (atomicCAS(&a.st->head, h, h + 1) != h) continue;
      for (long long w = 0; w < a.spin_limit; ++w) {  // the pusher may not have written it yet
        const unsigned long long v = vq[h];
        if (v) {
          __threadfence();
          return v;
        }
        __nanosleep(64);
      }
      pk_fail(a, CKD_ERR_TIMEOUT);
      return 0;
    }
    if (atomicAdd(reinterpret_cast<unsigned long long*>(&a.st->outstanding), 0ull) == 0ull)
      return 0;
    __nanosleep(256);
  }
  pk_fail(a, CKD_ERR_TIMEOUT);
  return 0;
}

// ------------------------------------------------------------ node records
template <int D>
struct SideStats {  // per child: tight box and first positions of its extremes
  double mn[D], mx[D];
  int32_t mnp[D], mxp[D];
};

template <int D>
__device__ __forceinline__ void stats_init(SideStats<D>& s) {
#pragma unroll
  for (int j = 0; j < D; ++j) {
    s.mn[j] = CUDART_INF;
    s.mx[j] = -CUDART_INF;
    s.mnp[j] = 0x7fffffff;
    s.mxp[j] = 0x7fffffff;
  }
}

template <int D>
__device__ __forceinline__ void stats_add(SideStats<D>& s, const double (&x)[D], int32_t p) {
#pragma unroll
  for (int j = 0; j < D; ++j) {
    if (x[j] < s.mn[j] || (x[j] == s.mn[j] && p < s.mnp[j])) {
      s.mn[j] = x[j];
      s.mnp[j] = p;
    }
    if (x[j] > s.mx[j] || (x[j] == s.mx[j] && p < s.mxp[j])) {
      s.mx[j] = x[j];
      s.mxp[j] = p;
    }
  }
}

template <int D>
__device__ __forceinline__ void stats_merge(SideStats<D>& s, const SideStats<D>& o) {
#pragma unroll
  for (int j = 0; j < D; ++j) {
    if (o.mn[j] < s.mn[j] || (o.mn[j] == s.mn[j] && o.mnp[j] < s.mnp[j])) {
      s.mn[j] = o.mn[j];
      s.mnp[j] = o.mnp[j];
    }
    if (o.mx[j] > s.mx[j] || (o.mx[j] == s.mx[j] && o.mxp[j] < s.mxp[j])) {
      s.mx[j] = o.mx[j];
      s.mxp[j] = o.mxp[j];
    }
  }
}

template <int D>
__device__ __forceinline__ void stats_warp_reduce(SideStats<D>& s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    SideStats<D> x;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      x.mn[j] = __shfl_xor_sync(0xffffffffu, s.mn[j], o);
      x.mx[j] = __shfl_xor_sync(0xffffffffu, s.mx[j], o);
      x.mnp[j] = __shfl_xor_sync(0xffffffffu, s.mnp[j], o);
      x.mxp[j] = __shfl_xor_sync(0xffffffffu, s.mxp[j], o);
    }
    stats_merge(s, x);
  }
}

// Block-wide merge of every thread's stats (all threads get the result).
template <int D>
__device__ void stats_block_reduce(SideStats<D>& s, SideStats<D>* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  stats_warp_reduce(s);
  __syncthreads();
  if (lane == 0) sh[w] = s;
  __syncthreads();
  s = sh[0];
  for (int i = 1; i < kPkWarps; ++i) stats_merge(s, sh[i]);
  __syncthreads();
}

// The records of a new node (or a root): meta, tight box, extremes, cell and the
// FP32 copies; a leaf also gets its centre.
template <int D>
__device__ void write_node(const PkArgs& a, int32_t c, int32_t start, int32_t count, int32_t depth,
                           int32_t parent, const SideStats<D>& s, const double* cel, bool leaf) {
  NodeMeta m;
  m.split = 0.0;
  m.left = -1;
  m.axis = -1;
  m.start = start;
  m.count = count;
  m.depth = depth;
  m.parent = parent;
  a.meta[c] = m;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const int64_t b = (int64_t)c * 2 * D + 2 * j;
    a.box[b] = s.mn[j];
    a.box[b + 1] = s.mx[j];
    a.cell[b] = cel[2 * j];
    a.cell[b + 1] = cel[2 * j + 1];
    a.box32[b] = __double2float_rd(s.mn[j]);
    a.box32[b + 1] = __double2float_ru(s.mx[j]);
    a.cell32[b] = __double2float_ru(cel[2 * j]);
    a.cell32[b + 1] = __double2float_rd(cel[2 * j + 1]);
    a.ext[b] = s.mnp[j];
    a.ext[b + 1] = s.mxp[j];
    if (leaf) a.centre[(int64_t)c * D + j] = leaf_centre(s.mn[j], s.mx[j]);
  }
}

// A point's final copies: SoA FP64, id, FP32 record, FP64 record.
template <int D>
__device__ __forceinline__ void write_final_point(const PkArgs& a, int64_t p, const double (&x)[D],
                                                  int32_t id) {
  constexpr int NV = (D + 3) / 4;
  const int64_t n = a.tv.n;
  float v[4 * NV];
  double w[4 * NV];
#pragma unroll
  for (int j = 0; j < 4 * NV; ++j) {
    w[j] = j < D ? x[j < D ? j : 0] : 0.0;
    v[j] = j < D ? __double2float_rn(w[j]) : 0.0f;
  }
#pragma unroll
  for (int j = 0; j < D; ++j) a.pts[(int64_t)j * n + p] = x[j];
  a.ids[p] = id;
#pragma unroll
  for (int h = 0; h < NV; ++h) {
    a.pts32[p * NV + h] = make_float4(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
    a.pts64[p * NV + h] = make_double4(w[4 * h], w[4 * h + 1], w[4 * h + 2], w[4 * h + 3]);
  }
}

template <int D>
__device__ __forceinline__ void load_point(const double* X, int64_t n, int64_t p, double (&x)[D]) {
#pragma unroll
  for (int j = 0; j < D; ++j) x[j] = __ldcg(X + (int64_t)j * n + p);
}

// The split rule of cosmokdtree.f90:347-410 for node `nd` (its tight box and
// cell in registers): axis, split value, mode (0 midpoint, 1 slide to the
// minimum -- the first point holding it goes left alone, 2 slide to the maximum
// -- it goes right alone) and the slide point's position.
template <int D>
__device__ __forceinline__ void decide(const double* bx, const double* cl, const int32_t* ex,
                                       int& axis, double& mid, int& mode, int32_t& slide) {
  double maxside = dsub(cl[1], cl[0]);
  axis = 0;
#pragma unroll
  for (int j = 1; j < D; ++j) {
    const double side = dsub(cl[2 * j + 1], cl[2 * j]);
    if (side > maxside) {
      maxside = side;
      axis = j;
    }
    if (side == maxside && dsub(bx[2 * j + 1], bx[2 * j]) > dsub(bx[2 * axis + 1], bx[2 * axis]))
      axis = j;
  }
  mid = dmul(0.5, dadd(cl[2 * axis], cl[2 * axis + 1]));
  const double minx = bx[2 * axis], maxx = bx[2 * axis + 1];
  mode = 0;
  slide = -1;
  if (minx >= mid) {
    mid = minx;
    mode = 1;
    slide = ex[2 * axis];
  } else if (maxx < mid) {
    mid = maxx;
    mode = 2;
    slide = ex[2 * axis + 1];
  }
}

// What one group item gathers in shared memory and publishes once at its end: the
// leaves it made and its open children for the next level's list (the hot global
// counters are touched once per item, not once per split; entries past the
// buffers go straight to the global list).
constexpr int kAccBig = 64;
constexpr int kAccSmall = 2 * kPkGroupNodes + 16;
struct ItemAcc {
  int nleaves;
  int nbig;
  int nsmall;
  int32_t big[kAccBig];
  int32_t small[kAccSmall];
};

// Records of a split node and its two children, then the children's place in
// the next level (called by one thread).
template <int D>
__device__ void finish_split(const PkArgs& a, int t, int32_t nd, const NodeMeta& m,
                             const double* cl, int axis, double mid, int32_t cid, int32_t nl,
                             const SideStats<D>& sl, const SideStats<D>& sr, int32_t* list_nxt,
                             int64_t lcap, int* s_nb, int* s_ns, ItemAcc& acc) {
  constexpr int NV = (D + 3) / 4;
  constexpr int PF = pair_f4(D);
  const int32_t cnt[2] = {nl, m.count - nl};
  const int32_t st0[2] = {m.start, m.start + nl};
  for (int side = 0; side < 2; ++side) {
    double cc[2 * D];
#pragma unroll
    for (int j = 0; j < 2 * D; ++j) cc[j] = cl[j];
    if (side == 0)
      cc[2 * axis + 1] = mid;
    else
      cc[2 * axis] = mid;
    const bool lf = cnt[side] <= a.leaf;
    write_node<D>(a, cid + side, st0[side], cnt[side], m.depth + 1, nd, side ? sr : sl, cc, lf);
    if (lf) {
      atomicAdd(&acc.nleaves, 1);
    } else if (cnt[side] >= kBigNode) {
      const int i = atomicAdd(&acc.nbig, 1);
      if (i < kAccBig)
        acc.big[i] = cid + side;
      else
        list_nxt[atomicAdd(s_nb, 1)] = cid + side;
    } else {
      const int i = atomicAdd(&acc.nsmall, 1);
      if (i < kAccSmall)
        acc.small[i] = cid + side;
      else
        list_nxt[lcap - 1 - atomicAdd(s_ns, 1)] = cid + side;
    }
  }
  NodeMeta mm = m;
  mm.split = mid;
  mm.left = cid;
  mm.axis = axis;
  a.meta[nd] = mm;
  float4* rec = a.pair + (int64_t)nd * PF;
  for (int side = 0; side < 2; ++side) {
    const SideStats<D>& s = side ? sr : sl;
    float lo[4 * NV], hi[4 * NV];
#pragma unroll
    for (int j = 0; j < 4 * NV; ++j) {
      lo[j] = j < D ? __double2float_rd(s.mn[j < D ? j : 0]) : 0.0f;
      hi[j] = j < D ? __double2float_ru(s.mx[j < D ? j : 0]) : 0.0f;
    }
#pragma unroll
    for (int h = 0; h < NV; ++h) {
      rec[side * 2 * NV + h] = make_float4(lo[4 * h], lo[4 * h + 1], lo[4 * h + 2], lo[4 * h + 3]);
      rec[side * 2 * NV + NV + h] = make_float4(hi[4 * h], hi[4 * h + 1], hi[4 * h + 2], hi[4 * h + 3]);
    }
  }
  const int4 info = make_int4(cid, cid + 1, cnt[0] <= a.leaf ? 1 : 0, cnt[1] <= a.leaf ? 1 : 0);
  rec[4 * NV] = *reinterpret_cast<const float4*>(&info);
  const int4 range = make_int4(st0[0], cnt[0], st0[1], cnt[1]);
  rec[4 * NV + 1] = *reinterpret_cast<const float4*>(&range);
  (void)t;
}

__device__ __forceinline__ void load_node(const PkArgs& a, int32_t nd, int d2, NodeMeta& m,
                                          double* bx, double* cl, int32_t* ex) {
  const int4* p = reinterpret_cast<const int4*>(a.meta + nd);
  const int4 u = __ldcg(p), v = __ldcg(p + 1);
  m.split = __hiloint2double(u.y, u.x);
  m.left = u.z;
  m.axis = u.w;
  m.start = v.x;
  m.count = v.y;
  m.depth = v.z;
  m.parent = v.w;
  for (int j = 0; j < d2; ++j) {
    bx[j] = __ldcg(a.box + (int64_t)nd * d2 + j);
    cl[j] = __ldcg(a.cell + (int64_t)nd * d2 + j);
    ex[j] = __ldcg(a.ext + (int64_t)nd * d2 + j);
  }
}

// ---------------------------------------------------------------- splits
// One node split by one warp.
template <int D>
__device__ void split_warp(const PkArgs& a, int t, int32_t nd, int32_t cid, const double* Xc,
                           const int32_t* Ic, double* Xn, int32_t* In, int32_t* list_nxt,
                           int64_t lcap, int* s_nb, int* s_ns, ItemAcc& acc) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t n = a.tv.n;
  NodeMeta m;
  double bx[2 * D], cl[2 * D];
  int32_t ex[2 * D];
  load_node(a, nd, 2 * D, m, bx, cl, ex);
  int axis, mode;
  double mid;
  int32_t slide;
  decide<D>(bx, cl, ex, axis, mid, mode, slide);
  const int64_t s0 = m.start, s1 = (int64_t)m.start + m.count;
  int32_t nl;
  if (mode == 1) {
    nl = 1;
  } else if (mode == 2) {
    nl = m.count - 1;
  } else {
    int c = 0;
    for (int64_t p = s0 + lane; p < s1; p += 32) c += __ldcg(Xc + (int64_t)axis * n + p) < mid;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    nl = c;
  }
  const bool leafL = nl <= a.leaf, leafR = m.count - nl <= a.leaf;
  SideStats<D> sl, sr;
  stats_init(sl);
  stats_init(sr);
  int32_t lb = 0, rb = 0;
  for (int64_t base = s0; base < s1; base += 32) {
    const int64_t p = base + lane;
    const bool v = p < s1;
    double x[D];
    int32_t id = 0;
    bool left = false;
    if (v) {
      load_point<D>(Xc, n, p, x);
      id = __ldcg(Ic + p);
      double xa = x[0];
#pragma unroll
      for (int j = 1; j < D; ++j)
        if (j == axis) xa = x[j];
      left = mode == 0 ? xa < mid : (mode == 1 ? p == slide : p != slide);
    }
    const unsigned bl = __ballot_sync(0xffffffffu, v && left);
    const unsigned br = __ballot_sync(0xffffffffu, v && !left);
    if (v) {
      const int64_t dst = left ? s0 + lb + __popc(bl & lt) : s0 + nl + rb + __popc(br & lt);
      if (left ? leafL : leafR) {
        write_final_point<D>(a, dst, x, id);
      } else {
#pragma unroll
        for (int j = 0; j < D; ++j) Xn[(int64_t)j * n + dst] = x[j];
        In[dst] = id;
      }
      stats_add(left ? sl : sr, x, (int32_t)dst);
    }
    lb += __popc(bl);
    rb += __popc(br);
  }
  stats_warp_reduce(sl);
  stats_warp_reduce(sr);
  if (lane == 0)
    finish_split<D>(a, t, nd, m, cl, axis, mid, cid, nl, sl, sr, list_nxt, lcap, s_nb, s_ns, acc);
}

// Exclusive prefix over the CTA of per-(pass, warp) counts, in position order
// (position base + it * kPkThreads + threadIdx.x).  cw[it * W + w] holds the
// warp's count; on return it holds its offset and *tot the total.
__device__ __forceinline__ void block_prefix(int32_t* cw, int32_t* tot) {
  constexpr int N = kPkItems * kPkWarps;
  static_assert(N <= 32, "one warp scans the pass counts");
  __syncthreads();
  if (threadIdx.x < 32) {
    const int v = threadIdx.x < N ? cw[threadIdx.x] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if ((int)threadIdx.x >= o) x += y;
    }
    if (threadIdx.x < N) cw[threadIdx.x] = x - v;
    if (threadIdx.x == 31) *tot = x;
  }
  __syncthreads();
}

struct BlockShared {
  int32_t cl[kPkItems * kPkWarps];
  int32_t cr[kPkItems * kPkWarps];
  int32_t tl, tr;
  int32_t cnt;
  int32_t cid;
};

// One node split by the whole CTA.
template <int D>
__device__ void split_block(const PkArgs& a, int t, int32_t nd, int32_t cid, const double* Xc,
                            const int32_t* Ic, double* Xn, int32_t* In, int32_t* list_nxt,
                            int64_t lcap, int* s_nb, int* s_ns, BlockShared& sh,
                            SideStats<D>* shs, ItemAcc& acc) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t n = a.tv.n;
  NodeMeta m;
  double bx[2 * D], cl[2 * D];
  int32_t ex[2 * D];
  load_node(a, nd, 2 * D, m, bx, cl, ex);
  int axis, mode;
  double mid;
  int32_t slide;
  decide<D>(bx, cl, ex, axis, mid, mode, slide);
  const int64_t s0 = m.start, s1 = (int64_t)m.start + m.count;
  if (threadIdx.x == 0) sh.cnt = 0;
  __syncthreads();
  int32_t nl;
  if (mode == 1) {
    nl = 1;
  } else if (mode == 2) {
    nl = m.count - 1;
  } else {
    int c = 0;
    for (int64_t p = s0 + threadIdx.x; p < s1; p += kPkThreads)
      c += __ldcg(Xc + (int64_t)axis * n + p) < mid;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) atomicAdd(&sh.cnt, c);
    __syncthreads();
    nl = sh.cnt;
  }
  const bool leafL = nl <= a.leaf, leafR = m.count - nl <= a.leaf;
  SideStats<D> sl, sr;
  stats_init(sl);
  stats_init(sr);
  int32_t lb = 0, rb = 0;
  for (int64_t base = s0; base < s1; base += (int64_t)kPkItems * kPkThreads) {
    double x[kPkItems][D];
    int32_t id[kPkItems];
    bool left[kPkItems], v[kPkItems];
    unsigned bl[kPkItems], br[kPkItems];
#pragma unroll
    for (int it = 0; it < kPkItems; ++it) {
      const int64_t p = base + (int64_t)it * kPkThreads + threadIdx.x;
      v[it] = p < s1;
      left[it] = false;
      id[it] = 0;
      if (v[it]) {
        load_point<D>(Xc, n, p, x[it]);
        id[it] = __ldcg(Ic + p);
        double xa = x[it][0];
#pragma unroll
        for (int j = 1; j < D; ++j)
          if (j == axis) xa = x[it][j];
        left[it] = mode == 0 ? xa < mid : (mode == 1 ? p == slide : p != slide);
      }
      bl[it] = __ballot_sync(0xffffffffu, v[it] && left[it]);
      br[it] = __ballot_sync(0xffffffffu, v[it] && !left[it]);
      if (lane == 0) {
        sh.cl[it * kPkWarps + w] = __popc(bl[it]);
        sh.cr[it * kPkWarps + w] = __popc(br[it]);
      }
    }
    block_prefix(sh.cl, &sh.tl);
    block_prefix(sh.cr, &sh.tr);
#pragma unroll
    for (int it = 0; it < kPkItems; ++it) {
      if (!v[it]) continue;
      const int64_t p = base + (int64_t)it * kPkThreads + threadIdx.x;
      const int64_t dst = left[it]
                              ? s0 + lb + sh.cl[it * kPkWarps + w] + __popc(bl[it] & lt)
                              : s0 + nl + rb + sh.cr[it * kPkWarps + w] + __popc(br[it] & lt);
      if (left[it] ? leafL : leafR) {
        write_final_point<D>(a, dst, x[it], id[it]);
      } else {
#pragma unroll
        for (int j = 0; j < D; ++j) Xn[(int64_t)j * n + dst] = x[it][j];
        In[dst] = id[it];
      }
      stats_add(left[it] ? sl : sr, x[it], (int32_t)dst);
      (void)p;
    }
    lb += sh.tl;
    rb += sh.tr;
    __syncthreads();  // the pass counts are rewritten by the next pass
  }
  stats_block_reduce(sl, shs);
  stats_block_reduce(sr, shs);
  if (threadIdx.x == 0)
    finish_split<D>(a, t, nd, m, cl, axis, mid, cid, nl, sl, sr, list_nxt, lcap, s_nb, s_ns, acc);
  __syncthreads();
}

// Root of tree t: bounding box (with the first positions of the extremes),
// validation, cell, FP32 screen slack; a root of at most `leaf` points becomes a
// leaf at once.  Returns false when the tree needs no split.
template <int D, bool PER>
__device__ bool root_init(const PkArgs& a, int t, SideStats<D>* shs, int* s_bad) {
  const int64_t n = a.tv.n;
  const int64_t s0 = __ldcg(a.off + t), s1 = __ldcg(a.off + t + 1);
  const double* X0 = a.X[0];
  if (threadIdx.x == 0) *s_bad = 0;
  __syncthreads();
  SideStats<D> s;
  stats_init(s);
  bool bad = false;
  for (int64_t p = s0 + threadIdx.x; p < s1; p += kPkThreads) {
    double x[D];
    load_point<D>(X0, n, p, x);
#pragma unroll
    for (int j = 0; j < D; ++j) bad = bad || !isfinite(x[j]);
    stats_add(s, x, (int32_t)p);
  }
  if (bad) atomicExch(s_bad, 1);
  stats_block_reduce(s, shs);  // contains barriers: s_bad is settled after it
  if (*s_bad) {
    if (threadIdx.x == 0) pk_fail(a, CKD_ERR_BAD_ARG);
    return false;
  }
  double cl[2 * D];
  bool outside = false, far = false;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    const double L = a.tv.L[j];
    if (PER) {
      cl[2 * j] = -0.5 * L;
      cl[2 * j + 1] = 0.5 * L;
      outside = outside || s.mn[j] < -L / 2 || s.mx[j] > L / 2;
    } else {
      cl[2 * j] = s.mn[j];
      cl[2 * j + 1] = s.mx[j];
    }
    const double b = fmax(fabs(s.mn[j]), fabs(s.mx[j])) + (PER ? L : 0.0);
    far = far || !(b < 1e18);
    if (threadIdx.x == 0) a.tslack[(int64_t)t * D + j] = (float)(b * (1.0 + 1e-6));
  }
  if (outside || far) {
    if (threadIdx.x == 0) pk_fail(a, outside ? CKD_ERR_OUT_OF_BOX : CKD_ERR_BAD_ARG);
    return false;
  }
  const int32_t cnt = (int32_t)(s1 - s0);
  const bool lf = cnt <= a.leaf;
  if (threadIdx.x == 0) {
    write_node<D>(a, t, (int32_t)s0, cnt, 0, -1, s, cl, lf);
    if (lf) atomicAdd(&a.st->n_leaves, 1);
    __threadfence();
  }
  __syncthreads();  // the root's records are read by every warp that splits it
  if (lf) {  // the points are final as they are
    for (int64_t p = s0 + threadIdx.x; p < s1; p += kPkThreads) {
      double x[D];
      load_point<D>(X0, n, p, x);
      write_final_point<D>(a, p, x, __ldcg(a.I[0] + p));
    }
    __threadfence();
  }
  return !lf;
}

// Group items of a level with nb big and ns small open nodes: a big node each,
// or kPkGroupNodes small nodes each, at most kPkMaxGroups.
__device__ __forceinline__ int level_groups(int nb, int ns) {
  const int g = max(nb, (ns + kPkGroupNodes - 1) / kPkGroupNodes);
  return max(1, min(g, kPkMaxGroups));
}

// Called by thread 0 of each group item of tree t's level l once its work is
// written and fenced.  The last group to finish pushes what follows: the next
// level's group items, or, when no node is left open, t's query blocks.
__device__ void level_done(const PkArgs& a, int t, int l, int groups) {
  if (atomicAdd(&a.tdone[t], 1) != groups - 1) return;
  __threadfence();  // the other groups' list entries and counts are visible now
  a.tdone[t] = 0;
  int* nx = reinterpret_cast<int*>(a.tcnt + 2 * t + ((l + 1) & 1));
  const int nb = atomicAdd(nx, 0), ns = atomicAdd(nx + 1, 0);
  a.tcnt[2 * t + (l & 1)] = make_int2(0, 0);  // free for level l + 2's list
  __threadfence();
  if (nb + ns > 0) {
    if (l + 1 >= kPkMaxLevels) {
      pk_fail(a, CKD_ERR_DEPTH);
      return;
    }
    const int g = level_groups(nb, ns);
    atomicAdd(reinterpret_cast<unsigned long long*>(&a.st->outstanding), (unsigned long long)g);
    pk_push(a, kItemBuild, t, (uint32_t)(l + 1) << 16, (uint32_t)g);
    return;
  }
  const int64_t nq = __ldcg(a.qoff + t + 1) - __ldcg(a.qoff + t);
  const uint32_t nblk = (uint32_t)((nq + a.qblock - 1) / a.qblock);
  if (nblk == 0) return;
  __threadfence();
  atomicAdd(reinterpret_cast<unsigned long long*>(&a.st->outstanding), (unsigned long long)nblk);
  pk_push(a, kItemQuery, t, 0, nblk);
}

// Group g of tree t's level l; returns the level's number of groups.  Every open
// node is split exactly once, so the group takes the child ids of all its nodes
// with one atomic; leaves, depth and the open children are published once at the
// end.
template <int D, bool PER>
__device__ int pk_level(const PkArgs& a, int t, int l, int g, BlockShared& bsh,
                        SideStats<D>* shs, int* s_bad, ItemAcc& acc, int* s_base) {
  const int cur = l & 1;
  const double* Xc = a.X[cur];
  const int32_t* Ic = a.I[cur];
  double* Xn = a.X[cur ^ 1];
  int32_t* In = a.I[cur ^ 1];
  const int64_t s0 = __ldcg(a.off + t), s1 = __ldcg(a.off + t + 1);
  const int64_t lcap = (s1 - s0) / (a.leaf + 1) + 2;
  const int64_t lb = __ldcg(a.lbase + t);
  const int32_t* list_cur = a.lists + lb + cur * lcap;
  int32_t* list_nxt = a.lists + lb + (cur ^ 1) * lcap;
  // the next level's list counts, shared by every group of this level
  int* nxt = reinterpret_cast<int*>(a.tcnt + 2 * t + (cur ^ 1));
  int nb, ns, groups;
  if (l == 0) {
    if (!root_init<D, PER>(a, t, shs, s_bad)) {
      __syncthreads();
      return 1;
    }
    nb = (s1 - s0) >= kBigNode ? 1 : 0;
    ns = 1 - nb;
    groups = 1;
  } else {
    const int2 c = __ldcg(a.tcnt + 2 * t + cur);
    nb = c.x;
    ns = c.y;
    groups = level_groups(nb, ns);
  }
  const int mybig = nb > g ? (nb - g + groups - 1) / groups : 0;  // i = g, g + groups, ...
  const int i0 = (int)((int64_t)g * ns / groups), i1 = (int)((int64_t)(g + 1) * ns / groups);
  const int mine = mybig + (i1 - i0);
  if (threadIdx.x == 0) {
    acc.nleaves = acc.nbig = acc.nsmall = 0;
    const int base = mine > 0 ? atomicAdd(&a.st->nodes, 2 * mine) : 0;
    if (mine > 0 && (int64_t)base + 2 * mine > a.node_cap) pk_fail(a, CKD_ERR_OOM);
    if (mine > 0 && l + 1 > kPkMaxDepth) pk_fail(a, CKD_ERR_DEPTH);
    *s_base = base;
    *s_bad = pk_error(a);
  }
  __syncthreads();
  if (*s_bad) return groups;  // the whole CTA leaves together
  const int32_t base = *s_base;
  for (int i = g, j = 0; i < nb; i += groups, ++j) {
    const int32_t nd = l == 0 ? t : __ldcg(list_cur + i);
    split_block<D>(a, t, nd, base + 2 * j, Xc, Ic, Xn, In, list_nxt, lcap, nxt, nxt + 1, bsh,
                   shs, acc);
  }
  const int w = threadIdx.x >> 5;
  for (int i = i0 + w; i < i1; i += kPkWarps) {
    const int32_t nd = l == 0 ? t : __ldcg(list_cur + lcap - 1 - i);
    split_warp<D>(a, t, nd, base + 2 * (mybig + i - i0), Xc, Ic, Xn, In, list_nxt, lcap, nxt,
                  nxt + 1, acc);
  }
  __syncthreads();
  // publish: the group's open children into the next level's list, its leaves
  // and depth into the launch's counts
  if (threadIdx.x == 0) {
    const int kb = min(acc.nbig, kAccBig), ks = min(acc.nsmall, kAccSmall);
    acc.nbig = kb ? atomicAdd(nxt, kb) : 0;         // now: first list slot of each kind
    acc.nsmall = ks ? atomicAdd(nxt + 1, ks) : 0;
    bsh.tl = kb;
    bsh.tr = ks;
    if (acc.nleaves) atomicAdd(&a.st->n_leaves, acc.nleaves);
    if (mine > 0) atomicMax(&a.st->max_depth, l + 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < bsh.tl; i += kPkThreads) list_nxt[acc.nbig + i] = acc.big[i];
  for (int i = threadIdx.x; i < bsh.tr; i += kPkThreads)
    list_nxt[lcap - 1 - (acc.nsmall + i)] = acc.small[i];
  __threadfence();
  __syncthreads();
  return groups;
}

template <int D, bool PER>
__device__ void pk_queries(const PkArgs& a, TreeView& tv, int t, uint32_t b, uint2* heaps) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t q0 = __ldcg(a.qoff + t) + (int64_t)b * a.qblock;
  const int64_t q1 = min(q0 + a.qblock, __ldcg(a.qoff + t + 1));
  if (q0 >= q1) return;
  // the screen's slack of this tree (its coordinates bound every point and box
  // a query of this tree can meet)
#pragma unroll
  for (int j = 0; j < D; ++j) tv.slack[j] = __ldcg(a.tslack + (int64_t)t * D + j);
  uint2* Hw = heaps + (size_t)w * 32 * (a.k + 1);
  const int64_t nq = q1 - q0;
  for (int64_t g = w; g * 32 < nq; g += kPkWarps)
    knn_lane_run<D, PER, false, true>(tv, a.Q + q0 * D, nullptr, nq, a.k, a.sorted,
                                      a.dist + q0 * a.k, a.idx + q0 * a.k, nullptr, nullptr,
                                      nullptr, nullptr, nullptr, nullptr, t, Hw, lane, g);
}

template <int D, bool PER>
__global__ void __launch_bounds__(kPkThreads, 4) k_forest_pk(PkArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned long long s_item;
  __shared__ int s_bad, s_base;
  __shared__ ItemAcc acc;
  __shared__ BlockShared bsh;
  __shared__ SideStats<D> shs[kPkWarps];
  TreeView tv = a.tv;
  uint2* heaps = reinterpret_cast<uint2*>(smem);
  for (;;) {
    if (threadIdx.x == 0) s_item = pk_claim(a);
    __syncthreads();
    const unsigned long long item = s_item;
    __syncthreads();
    if (item == 0) break;
    const unsigned long long type = item >> 62;
    const int t = (int)((item >> 32) & 0x3fffffffull);
    const uint32_t pl = (uint32_t)(item & 0xffffffffull);
    if (type == kItemBuild) {
      const int l = (int)(pl >> 16), g = (int)(pl & 0xffffu);
      const int groups = pk_level<D, PER>(a, t, l, g, bsh, shs, &s_bad, acc, &s_base);
      if (threadIdx.x == 0 && !pk_error(a)) level_done(a, t, l, groups);
    } else {
      pk_queries<D, PER>(a, tv, t, pl, heaps);
      __threadfence();
      __syncthreads();
    }
    if (threadIdx.x == 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(&a.st->outstanding), ~0ull);  // - 1
    __syncthreads();
  }
}

// Queue reset and the first items: the roots in decreasing size (the largest
// trees start first), with `withhold` of them counted but never pushed (a test of
// the bounded polling: the launch then ends with CKD_ERR_TIMEOUT).
__global__ void k_pk_reset(PkState* st, unsigned long long* queue, int64_t queue_cap,
                           const int32_t* roots, int T, int withhold) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int pushed = T - withhold;
  if (i < queue_cap) queue[i] = i < pushed ? pk_item(kItemBuild, roots[i + withhold], 0) : 0ull;
  if (i == 0) {
    st->head = 0;
    st->tail = (unsigned long long)pushed;
    st->outstanding = T;
    st->error = 0;
    st->nodes = T;
    st->max_depth = 0;
    st->n_leaves = 0;
  }
}

// Input rows (n, d) -> SoA working copy; ids local to their tree.
__global__ void k_pk_points(const double* __restrict__ in, int64_t n, int d,
                            const int64_t* __restrict__ off, int32_t T, double* __restrict__ X,
                            int32_t* __restrict__ I) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  for (int j = 0; j < d; ++j) X[(int64_t)j * n + p] = in[p * d + j];
  int32_t lo = 0, hi = T - 1;
  while (lo < hi) {
    const int32_t mid = (lo + hi + 1) >> 1;
    if (off[mid] <= p)
      lo = mid;
    else
      hi = mid - 1;
  }
  I[p] = (int32_t)(p - off[lo]);
}

}  // namespace

// ------------------------------------------------------------------ host
struct ForestPlan {
  int device = 0;
  ckd_tree* tree = nullptr;  // arrays owned by the plan
  int64_t T = 0, n = 0, nq = 0;
  int d = 3, k = 8, leaf = 16, sorted = 1, qblock = 128, periodic = 0;
  double L[CKD_MAX_D] = {0};
  int32_t node_cap = 0;
  int64_t queue_cap = 0;
  const double* pts_in = nullptr;  // caller's device points (n, d)
  const double* Q = nullptr;       // caller's device queries (nq, d)
  double* dist = nullptr;
  int64_t* idx = nullptr;
  std::vector<void*> bufs;
  int64_t* off = nullptr;
  int64_t* qoff = nullptr;
  int64_t* lbase = nullptr;
  int32_t* lists = nullptr;
  int2* tcnt = nullptr;
  int32_t* tdone = nullptr;
  float* tslack = nullptr;
  int32_t* roots = nullptr;
  int32_t* ext = nullptr;
  double* X[2] = {nullptr, nullptr};
  int32_t* I[2] = {nullptr, nullptr};
  unsigned long long* queue = nullptr;
  PkState* st = nullptr;
  std::vector<int64_t> off_h;
  int grid = 0;
  size_t smem = 0;
};

namespace {

template <typename T>
cudaError_t plan_alloc(ForestPlan* p, T** out, size_t bytes) {
  void* q = nullptr;
  const cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
  if (e == cudaSuccess) {
    p->bufs.push_back(q);
    *out = reinterpret_cast<T*>(q);
  }
  return e;
}

template <int D, bool PER>
ckd_status pk_launch(ForestPlan* p, cudaStream_t s, int withhold, long long spin_limit) {
  const int T = (int)p->T;
  ckd_tree* t = p->tree;
  const unsigned rb = (unsigned)cdiv(std::max<int64_t>(p->queue_cap, 1), 256);
  CKD_CUDA(cudaMemsetAsync(p->tcnt, 0, sizeof(int2) * 2 * T, s));
  CKD_CUDA(cudaMemsetAsync(p->tdone, 0, sizeof(int32_t) * T, s));
  k_pk_reset<<<rb, 256, 0, s>>>(p->st, p->queue, p->queue_cap, p->roots, T, withhold);
  CKD_LAUNCH_CHECK();
  k_pk_points<<<(unsigned)cdiv(p->n, 256), 256, 0, s>>>(p->pts_in, p->n, D, p->off, T, p->X[0],
                                                       p->I[0]);
  CKD_LAUNCH_CHECK();
  PkArgs a;
  std::memset(&a, 0, sizeof(a));
  a.tv = t->view();
  a.meta = t->meta;
  a.box = t->box;
  a.cell = t->cell;
  a.box32 = t->box32;
  a.cell32 = t->cell32;
  a.centre = t->centre;
  a.pair = t->pair;
  a.pts = t->pts;
  a.ids = t->ids;
  a.pts32 = t->pts32;
  a.pts64 = t->pts64;
  a.ext = p->ext;
  a.X[0] = p->X[0];
  a.X[1] = p->X[1];
  a.I[0] = p->I[0];
  a.I[1] = p->I[1];
  a.lists = p->lists;
  a.lbase = p->lbase;
  a.tcnt = p->tcnt;
  a.tdone = p->tdone;
  a.tslack = p->tslack;
  a.off = p->off;
  a.qoff = p->qoff;
  a.Q = p->Q;
  a.dist = p->dist;
  a.idx = p->idx;
  a.queue = p->queue;
  a.st = p->st;
  a.queue_cap = p->queue_cap;
  a.spin_limit = spin_limit;
  a.T = T;
  a.leaf = p->leaf;
  a.k = p->k;
  a.sorted = p->sorted;
  a.qblock = p->qblock;
  a.node_cap = p->node_cap;
  k_forest_pk<D, PER><<<(unsigned)p->grid, kPkThreads, p->smem, s>>>(a);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

template <int D, bool PER>
ckd_status pk_prepare(ForestPlan* p) {
  p->smem = (size_t)kPkWarps * compact_heap_bytes(p->k);
  CKD_CUDA(cudaFuncSetAttribute(k_forest_pk<D, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)p->smem));
  int per_sm = 0, sms = 148;
  CKD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_forest_pk<D, PER>, kPkThreads,
                                                         p->smem));
  CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device));
  if (per_sm < 1) return fail(CKD_ERR_CUDA, "persistent forest kernel does not fit on an SM");
  p->grid = per_sm * sms;
  return CKD_OK;
}

}  // namespace

ckd_status forest_pk_limits(int k, int d) {
  if (k < 1 || k > kSmemK) return fail(CKD_ERR_BAD_ARG, "persistent forest kNN needs 1 <= k <= 64");
  if (d < 1 || d > CKD_MAX_D) return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
  return CKD_OK;
}

void forest_plan_release(ForestPlan* p) {
  if (!p) return;
  cudaDeviceSynchronize();
  for (void* b : p->bufs) cudaFree(b);
  if (p->tree) {
    // the arrays belonged to the plan (freed above)
    delete p->tree;
  }
  delete p;
}

ckd_status forest_plan_create(const double* pts_dev, const int64_t* offsets, int64_t T, int d,
                              int leaf, const double* boxsize, const double* q_dev,
                              const int64_t* q_offsets, int64_t nq, int k, int sorted,
                              double* dist_dev, int64_t* idx_dev, double node_factor,
                              int qblock, ForestPlan** out) {
  *out = nullptr;
  CKD_TRY(forest_pk_limits(k, d));
  if (T < 1 || T >= (1 << 30)) return fail(CKD_ERR_BAD_ARG, "a forest plan needs 1 .. 2^30-1 trees");
  if (leaf < 1) return fail(CKD_ERR_BAD_ARG, "Leaf size must be a positive integer");
  if (qblock < 32 || qblock > (1 << 20)) return fail(CKD_ERR_BAD_ARG, "query block must be 32..2^20");
  if (!pts_dev || !offsets || !q_offsets || (nq > 0 && (!q_dev || !dist_dev || !idx_dev)))
    return fail(CKD_ERR_BAD_ARG, "null pointer");
  std::vector<int64_t> off(offsets, offsets + T + 1), qo(q_offsets, q_offsets + T + 1);
  if (off[0] != 0 || qo[0] != 0) return fail(CKD_ERR_BAD_ARG, "offsets must start at 0");
  for (int64_t i = 0; i < T; ++i) {
    if (off[i + 1] <= off[i]) return fail(CKD_ERR_BAD_ARG, "every tree needs at least one point");
    if (qo[i + 1] < qo[i]) return fail(CKD_ERR_BAD_ARG, "query offsets must not decrease");
  }
  if (qo[T] != nq) return fail(CKD_ERR_BAD_ARG, "query offsets must end at nq");
  const int64_t n = off[T];
  if (n >= 0x7fffffffll) return fail(CKD_ERR_BAD_ARG, "more than 2^31-2 points are not supported");
  if (!(node_factor > 0)) node_factor = 0.45;
  const double cap = (double)T + node_factor * (double)n + 1024.0;
  if (cap >= 2.0e9) return fail(CKD_ERR_BAD_ARG, "node capacity beyond 2^31");
  int dev = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  ForestPlan* p = new ForestPlan();
  struct Guard {
    ForestPlan** p;
    ~Guard() {
      if (*p) forest_plan_release(*p);
    }
  } guard{&p};
  p->device = dev;
  p->T = T;
  p->n = n;
  p->nq = nq;
  p->d = d;
  p->k = k;
  p->leaf = leaf;
  p->sorted = sorted ? 1 : 0;
  p->qblock = qblock;
  p->pts_in = pts_dev;
  p->Q = q_dev;
  p->dist = dist_dev;
  p->idx = idx_dev;
  p->periodic = boxsize ? 1 : 0;
  for (int j = 0; j < d; ++j) {
    if (boxsize && !(boxsize[j] > 0 && std::isfinite(boxsize[j])))
      return fail(CKD_ERR_BAD_ARG, "boxsize entries must be positive and finite");
    p->L[j] = boxsize ? boxsize[j] : 0.0;
  }
  p->node_cap = (int32_t)cap;
  // level items: every tree's levels, a group per kPkGroupNodes small open nodes
  // (open nodes over all levels are internal nodes, at most half the node
  // capacity), a group per big open node (at most n / kBigNode per level)
  p->queue_cap = T * (int64_t)kPkMaxLevels + (int64_t)(cap / 2) / kPkGroupNodes +
                 32 * (n / kBigNode) + 64;
  for (int64_t i = 0; i < T; ++i) p->queue_cap += (qo[i + 1] - qo[i] + qblock - 1) / qblock;
  p->off_h = off;
  // list halves per tree: at most (points / (leaf + 1) + 2) open nodes per level
  std::vector<int64_t> lb(T);
  int64_t ltot = 0;
  for (int64_t i = 0; i < T; ++i) {
    lb[i] = ltot;
    ltot += 2 * ((off[i + 1] - off[i]) / (leaf + 1) + 2);
  }
  std::vector<int32_t> order(T);
  for (int64_t i = 0; i < T; ++i) order[i] = (int32_t)i;
  std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
    return off[x + 1] - off[x] > off[y + 1] - off[y];
  });
  ckd_tree* t = new ckd_tree();
  p->tree = t;
  t->device = dev;
  t->n = n;
  t->d = d;
  t->leaf = leaf;
  t->periodic = p->periodic;
  t->input_dtype = CKD_F64;
  for (int j = 0; j < d; ++j) t->L[j] = p->L[j];
  t->n_trees = T;
  t->tree_off = off;
  const int NV = (d + 3) / 4;
  const int64_t C = p->node_cap;
  CKD_CUDA(plan_alloc(p, &t->meta, sizeof(NodeMeta) * C));
  CKD_CUDA(plan_alloc(p, &t->box, sizeof(double) * 2 * d * C));
  CKD_CUDA(plan_alloc(p, &t->cell, sizeof(double) * 2 * d * C));
  CKD_CUDA(plan_alloc(p, &t->box32, sizeof(float) * 2 * d * C));
  CKD_CUDA(plan_alloc(p, &t->cell32, sizeof(float) * 2 * d * C));
  CKD_CUDA(plan_alloc(p, &t->centre, sizeof(double) * d * C));
  CKD_CUDA(plan_alloc(p, &t->pair, sizeof(float4) * pair_f4(d) * C));
  CKD_CUDA(plan_alloc(p, &p->ext, sizeof(int32_t) * 2 * d * C));
  CKD_CUDA(plan_alloc(p, &t->pts, sizeof(double) * d * n));
  CKD_CUDA(plan_alloc(p, &t->ids, sizeof(int32_t) * n));
  CKD_CUDA(plan_alloc(p, &t->pts32, sizeof(float4) * NV * n));
  CKD_CUDA(plan_alloc(p, &t->pts64, sizeof(double4) * NV * n));
  for (int b = 0; b < 2; ++b) {
    CKD_CUDA(plan_alloc(p, &p->X[b], sizeof(double) * d * n));
    CKD_CUDA(plan_alloc(p, &p->I[b], sizeof(int32_t) * n));
  }
  CKD_CUDA(plan_alloc(p, &p->off, sizeof(int64_t) * (T + 1)));
  CKD_CUDA(plan_alloc(p, &p->qoff, sizeof(int64_t) * (T + 1)));
  CKD_CUDA(plan_alloc(p, &p->lbase, sizeof(int64_t) * T));
  CKD_CUDA(plan_alloc(p, &p->lists, sizeof(int32_t) * ltot));
  CKD_CUDA(plan_alloc(p, &p->tcnt, sizeof(int2) * 2 * T));
  CKD_CUDA(plan_alloc(p, &p->tdone, sizeof(int32_t) * T));
  CKD_CUDA(plan_alloc(p, &p->tslack, sizeof(float) * d * T));
  CKD_CUDA(plan_alloc(p, &p->roots, sizeof(int32_t) * T));
  CKD_CUDA(plan_alloc(p, &p->queue, sizeof(unsigned long long) * p->queue_cap));
  CKD_CUDA(plan_alloc(p, &p->st, sizeof(PkState)));
  CKD_CUDA(cudaMemcpy(p->off, off.data(), sizeof(int64_t) * (T + 1), cudaMemcpyHostToDevice));
  CKD_CUDA(cudaMemcpy(p->qoff, qo.data(), sizeof(int64_t) * (T + 1), cudaMemcpyHostToDevice));
  CKD_CUDA(cudaMemcpy(p->lbase, lb.data(), sizeof(int64_t) * T, cudaMemcpyHostToDevice));
  CKD_CUDA(cudaMemcpy(p->roots, order.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice));
  switch (d * 2 + p->periodic) {
#define CKD_PKP(DD)                                            \
  case 2 * DD: CKD_TRY((pk_prepare<DD, false>(p))); break;     \
  case 2 * DD + 1: CKD_TRY((pk_prepare<DD, true>(p))); break;
    CKD_PKP(1) CKD_PKP(2) CKD_PKP(3) CKD_PKP(4) CKD_PKP(5) CKD_PKP(6) CKD_PKP(7) CKD_PKP(8)
#undef CKD_PKP
  }
  *out = p;
  p = nullptr;  // the guard keeps it
  return CKD_OK;
}

ckd_status forest_plan_run(ForestPlan* p, cudaStream_t s, int withhold, long long spin_limit) {
  if (withhold < 0 || withhold > p->T) return fail(CKD_ERR_BAD_ARG, "withheld items out of range");
  switch (p->d * 2 + p->periodic) {
#define CKD_PKL(DD)                                                             \
  case 2 * DD: return pk_launch<DD, false>(p, s, withhold, spin_limit);         \
  case 2 * DD + 1: return pk_launch<DD, true>(p, s, withhold, spin_limit);
    CKD_PKL(1) CKD_PKL(2) CKD_PKL(3) CKD_PKL(4) CKD_PKL(5) CKD_PKL(6) CKD_PKL(7) CKD_PKL(8)
#undef CKD_PKL
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

// Status of the last run (synchronises the stream): the first failure recorded
// on the device, and the forest's counts and screen slack for later searches.
ckd_status forest_plan_status(ForestPlan* p, cudaStream_t s) {
  CKD_CUDA(cudaStreamSynchronize(s));
  PkState h;
  CKD_CUDA(cudaMemcpy(&h, p->st, sizeof(PkState), cudaMemcpyDeviceToHost));
  if (h.error == CKD_ERR_TIMEOUT)
    return fail(CKD_ERR_TIMEOUT, "persistent forest launch: the work queue's wait ran out");
  if (h.error == CKD_ERR_OOM)
    return fail(CKD_ERR_OOM, "persistent forest launch: node capacity or queue exceeded (raise "
                             "the node factor)");
  if (h.error == CKD_ERR_DEPTH)
    return fail(CKD_ERR_DEPTH, "persistent forest launch: a tree is deeper than the per-lane "
                               "search supports (125 levels)");
  if (h.error == CKD_ERR_OUT_OF_BOX) return fail(CKD_ERR_OUT_OF_BOX, "Points outside (-L/2, L/2) range");
  if (h.error == CKD_ERR_BAD_ARG)
    return fail(CKD_ERR_BAD_ARG, "points contain NaN or infinite coordinates, or coordinates "
                                 "beyond 1e18");
  if (h.error != 0) return fail(CKD_ERR_CUDA, "persistent forest launch failed");
  if (h.outstanding != 0 || h.head != h.tail)
    return fail(CKD_ERR_CUDA, "persistent forest launch ended with work left");
  ckd_tree* t = p->tree;
  t->n_nodes = h.nodes;
  t->n_leaves = h.n_leaves;
  t->depth = h.max_depth;
  std::vector<float> sl((size_t)p->T * p->d);
  CKD_CUDA(cudaMemcpy(sl.data(), p->tslack, sizeof(float) * sl.size(), cudaMemcpyDeviceToHost));
  t->screen_ok = true;
  for (int j = 0; j < p->d; ++j) {
    float m = 0.0f;
    for (int64_t i = 0; i < p->T; ++i) m = std::max(m, sl[(size_t)i * p->d + j]);
    t->slack[j] = m;
  }
  return CKD_OK;
}

const ckd_tree* forest_plan_tree(const ForestPlan* p) { return p->tree; }

}  // namespace ckd
