// ckd_common.cuh -- shared types and device helpers of libckd (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <cfloat>
#include <string>
#include <vector>

#include "../../include/ckd.h"

#define CKD_MAX_D 8

// Loads of tree records in the search helpers (ckd_traverse.cuh, ckd_knn.cuh,
// ckd_knn_lane.cuh).  By default they take the read-only path (__ldg): the tree
// does not change during a launch.  A translation unit whose kernel reads tree
// records written earlier in the same launch (the persistent forest kernel)
// defines CKD_TREE_LOADS_L2 before including these headers: its loads then go
// to L2 (__ldcg), because an SM's L1 is not coherent with other SMs' stores.
// The helpers live in an inline namespace named after the policy, so the two
// compiled forms never share a symbol.
#ifdef CKD_TREE_LOADS_L2
#define CKD_LDT(p) __ldcg(p)
#define CKD_LD_BEGIN inline namespace loads_l2 {
#else
#define CKD_LDT(p) __ldg(p)
#define CKD_LD_BEGIN inline namespace loads_nc {
#endif
#define CKD_LD_END }

namespace ckd {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
ckd_status fail(ckd_status st, const std::string& msg);
ckd_status cuda_fail(cudaError_t e, const char* what);

#define CKD_CUDA(call)                                       \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return ::ckd::cuda_fail(_e, #call); \
  } while (0)

// every kernel launch is followed by this: counts the launch, reports launch errors
void note_launch();
#define CKD_LAUNCH_CHECK()                 \
  do {                                     \
    ::ckd::note_launch();                  \
    CKD_CUDA(cudaGetLastError());          \
  } while (0)

#define CKD_TRY(call)                    \
  do {                                   \
    ckd_status _s = (call);              \
    if (_s != CKD_OK) return _s;         \
  } while (0)

// kNN kernel choice (ckd_set_knn_variant): 0 automatic, 1 FP64 packet traversal,
// 7/8 per-lane compact heap, 9 warp-converged
int knn_variant();
// tuning knobs (see ckd_set_tuning): blocks-per-SM cap (0 = none), warps per block
int knn_blocks_per_sm();
int knn_warps_per_block();
// learned-bound search kernel: 0 bounded per-lane with compact heap (k_knn_lane2),
// 3 as 0 with child-pair-record descent (default), 4 bounded warp-converged
int learned_kernel();
// query leaf ordering before a search: 0 automatic, 1 always, 2 never
int query_order_mode();
// learned-bound network inference on the tensor cores (tcgen05) instead of FP32 FMAs
bool mlp_tensor_cores();
bool box_warp_enabled();

// events bracketing the main search kernel when kernel timing is on
void timing_begin(cudaStream_t s);
void timing_end(cudaStream_t s);

// stream-ordered scratch allocation from a per-device pool
cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t s);
cudaError_t dev_free(void* p, cudaStream_t s);

// The pool buffers of one call: each joins the guard when it is allocated and
// returns to the pool (in stream order) when the guard goes out of scope, on the
// error paths too.
struct Scratch {
  cudaStream_t s;
  std::vector<void*> ps;
  explicit Scratch(cudaStream_t st) : s(st) {}
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
  ~Scratch() {
    for (void* p : ps) dev_free(p, s);
  }
  template <typename T>
  cudaError_t alloc(T** p, size_t bytes) {
    const cudaError_t e = dev_alloc(reinterpret_cast<void**>(p), bytes, s);
    if (e == cudaSuccess)
      ps.push_back(*p);
    else
      *p = nullptr;
    return e;
  }
  // hand a buffer to the caller instead of freeing it
  void release(const void* p) {
    for (auto& x : ps)
      if (x == p) x = nullptr;
  }
};

// ------------------------------------------------------------- node layout
// One 32-byte record per node.  Children of an internal node are allocated as a
// pair: right = left + 1.  start/count give the node's range in the leaf-ordered
// point arrays (every subtree is contiguous there).
struct __align__(16) NodeMeta {
  double split;   // splitting value (cosmokdtree.f90:412 node%point)
  int32_t left;   // left child, -1 for a leaf
  int32_t axis;   // splitting axis, -1 for a leaf
  int32_t start;  // first leaf-ordered point of the subtree
  int32_t count;  // number of points in the subtree
  int32_t depth;  // root = 0
  int32_t parent; // -1 for the root
};
static_assert(sizeof(NodeMeta) == 32, "NodeMeta must be 32 bytes");

// Read-only view of a built tree handed to kernels.
struct TreeView {
  int32_t n;
  int32_t n_nodes;
  int32_t d;
  int32_t periodic;
  double L[CKD_MAX_D];       // box side (periodic)
  const NodeMeta* meta;      // [n_nodes]
  const double* box;         // [n_nodes][2d] tight bounding box lo0,hi0,lo1,hi1,...
  const double* cell;        // [n_nodes][2d] sliding-midpoint cell (reference node bounds)
  const double* pts;         // SoA [d][n], leaf order
  const int32_t* ids;        // [n] original index per leaf-ordered point
  // FP32 screening copies: node boxes rounded outwards, and each point's
  // absolute coordinates rounded to FP32 (zero padded), 1 (d <= 4) or 2 float4
  // per point, for screens whose error bound depends only on the query and the
  // coordinate range
  const float* box32;        // [n_nodes][2d]
  const float4* pts32;       // [n][(d + 3) / 4]
  // the FP64 points again, one 32-byte (d <= 4) or 64-byte record per point, so an
  // exact distance evaluation touches one or two sectors instead of d
  const double4* pts64;      // [n][(d + 3) / 4]
  float slack[CKD_MAX_D];    // per-axis absolute slack of FP32 node-box gaps
  // bottom-up search records
  const float4* pair;        // per internal node: both children's FP32 boxes + ids/flags
  const float* cell32;       // [n_nodes][2d] cells rounded inwards (lo up, hi down)
  const double* centre;      // [n_nodes][d] leaf centres (leaf_centre of the FP64 box)
};

// Child-pair record of an internal node, (4 * NV + 2) float4s with NV = (d+3)/4:
// left lo[NV], left hi[NV], right lo[NV], right hi[NV], then int4 {left node,
// right node, left is-leaf, right is-leaf}, then int4 {left start, left count,
// right start, right count} (the children's ranges of leaf-ordered positions).
__host__ __device__ constexpr int pair_f4(int d) { return 4 * ((d + 3) / 4) + 2; }

// Leaf frame used by the FP32 screen: centre c = 0.5 * (lo + hi) of the leaf's
// FP64 box (the same separately rounded operations when the FP32 copy is made
// and when a query is screened), and the half-extent R >= |p - c| of its points.
__device__ __forceinline__ double leaf_centre(double lo, double hi) {
  return __dmul_rn(0.5, __dadd_rn(lo, hi));
}

// --------------------------------------------------------- exact FP64 math
// Every FP64 product and sum below is separately rounded (explicit _rn
// intrinsics block FMA contraction), the evaluation order of
// cosmokdtree.f90:1441-1465 (axis order, d2 = 0 + dx0^2 + dx1^2 + ...).
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }

// minimum image of a coordinate difference: min(|dx|, L - |dx|)  (cosmokdtree.f90:1455)
__device__ __forceinline__ double min_image(double dx, double L) {
  double a = fabs(dx);
  double b = dsub(L, a);
  return a < b ? a : b;
}

// Lower bound of the squared distance from q to any point of [lo, hi] on one
// axis.  Non-periodic: distance to the nearer face (cosmokdtree.f90:1536-1542).
// Periodic: the nearer of the two faces under the minimum image, which bounds
// every point of the interval from below (also after rounding, because each
// rounded operation is monotone in its inputs).
template <bool PER>
__device__ __forceinline__ double axis_gap(double x, double lo, double hi, double L) {
  if (x >= lo && x <= hi) return 0.0;
  if (!PER) return x < lo ? dsub(lo, x) : dsub(x, hi);
  double a = min_image(dsub(x, lo), L);
  double b = min_image(dsub(x, hi), L);
  return a < b ? a : b;
}

// ------------------------------------------------------ ordered double keys
// Monotone map double -> uint64 so that atomicMin/atomicMax on the key order
// doubles (NaNs sort beyond the infinities).
__device__ __forceinline__ unsigned long long dkey_bits(unsigned long long b) {
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ unsigned long long dkey(double x) {
  return dkey_bits((unsigned long long)__double_as_longlong(x));
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}
__host__ __device__ inline unsigned long long dkey_host_pos_inf_min() { return ~0ull; }  // key above any double

// HUGE(0.0) of the reference promoted to FP64 (cosmokdtree.f90:517)
#define CKD_HUGE ((double)FLT_MAX)

// ------------------------------------------------------------------ misc
__host__ __device__ inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Launch helpers implemented in scan.cu
// exclusive scan of n int32 values into int64 (out has n+1 entries, out[n] = total)
ckd_status scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, cudaStream_t s);
// exclusive scan of n int64 values (out has n+1 entries)
ckd_status scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);
// exclusive scan of n int32 values into int32 (out has n+1 entries)
ckd_status scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s);
// owner[i] = row t of CSR offsets off (n_rows + 1 entries) holding item i
ckd_status csr_owner(const int64_t* off_dev, int32_t n_rows, int64_t n_items, int32_t* owner,
                     cudaStream_t s);

}  // namespace ckd

// Host-side tree object behind the opaque ckd_tree* handle.
struct ckd_tree {
  int device = 0;
  int64_t n = 0;
  int d = 0;
  int leaf = 16;
  int periodic = 0;
  int input_dtype = CKD_F64;
  double L[CKD_MAX_D] = {0};
  int32_t n_nodes = 0;
  int32_t n_leaves = 0;
  int32_t depth = 0;
  // a forest holds n_trees independent trees: tree t owns points
  // tree_off[t] .. tree_off[t+1]-1 (ids local to the tree) and is rooted at node t
  int64_t n_trees = 1;
  std::vector<int64_t> tree_off;
  ckd::NodeMeta* meta = nullptr;
  double* box = nullptr;
  double* cell = nullptr;
  double* pts = nullptr;
  int32_t* ids = nullptr;
  float* box32 = nullptr;
  float4* pts32 = nullptr;
  double4* pts64 = nullptr;
  float slack[CKD_MAX_D] = {0};
  bool screen_ok = false;  // FP32 screen usable (coordinates well inside FP32 range)
  float4* pair = nullptr;
  float* cell32 = nullptr;
  double* centre = nullptr;
  ckd::TreeView view() const {
    ckd::TreeView v;
    v.n = (int32_t)n;
    v.n_nodes = n_nodes;
    v.d = d;
    v.periodic = periodic;
    for (int j = 0; j < CKD_MAX_D; ++j) v.L[j] = L[j];
    v.meta = meta;
    v.box = box;
    v.cell = cell;
    v.pts = pts;
    v.ids = ids;
    v.box32 = box32;
    v.pts32 = pts32;
    v.pts64 = pts64;
    for (int j = 0; j < CKD_MAX_D; ++j) v.slack[j] = slack[j];
    v.pair = pair;
    v.cell32 = cell32;
    v.centre = centre;
    return v;
  }
};
