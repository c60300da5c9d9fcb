// api.cu -- the extern "C" boundary of libckd (declared in include/ckd.h).
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ckd_common.cuh"
#include "ckd_mlp.cuh"

namespace ckd {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }
ckd_status fail(ckd_status st, const std::string& msg) {
  g_err = msg;
  return st;
}
ckd_status cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky-free error so later calls can proceed
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return CKD_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ||
      e == cudaErrorNoKernelImageForDevice)
    return CKD_ERR_NO_DEVICE;
  return CKD_ERR_CUDA;
}

static std::atomic<int64_t> g_launches{0};
static std::atomic<int> g_knn_variant{0};
int knn_variant() { return g_knn_variant.load(std::memory_order_relaxed); }
static std::atomic<int> g_knn_bps{0}, g_knn_wpb{2};
int knn_blocks_per_sm() { return g_knn_bps.load(std::memory_order_relaxed); }
int knn_warps_per_block() { return g_knn_wpb.load(std::memory_order_relaxed); }
static std::atomic<int> g_learned_kernel{3};
int learned_kernel() { return g_learned_kernel.load(std::memory_order_relaxed); }
static std::atomic<int> g_order_mode{0};
int query_order_mode() { return g_order_mode.load(std::memory_order_relaxed); }
static std::atomic<int> g_mlp_tc{1};
bool mlp_tensor_cores() { return g_mlp_tc.load(std::memory_order_relaxed) != 0; }
static std::atomic<int> g_box_warp{1};
bool box_warp_enabled() { return g_box_warp.load(std::memory_order_relaxed) != 0; }
// persistent forest launch: how long an idle CTA polls the work queue (ms), and
// how many first items the host withholds (0 outside tests)
static std::atomic<int> g_pk_wait_ms{20000}, g_pk_withhold{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ------------------------------------------------------------ kernel timing
static std::atomic<int> g_timing{0};
static cudaEvent_t g_ev[2];
static bool g_ev_ok = false, g_ev_recorded = false;
void timing_begin(cudaStream_t s) {
  if (!g_timing.load()) return;
  if (!g_ev_ok) {
    cudaEventCreate(&g_ev[0]);
    cudaEventCreate(&g_ev[1]);
    g_ev_ok = true;
  }
  cudaEventRecord(g_ev[0], s);
}
void timing_end(cudaStream_t s) {
  if (!g_timing.load() || !g_ev_ok) return;
  cudaEventRecord(g_ev[1], s);
  g_ev_recorded = true;
}

// ---------------------------------------------------------- scratch memory
// One stream-ordered pool per device, keeping freed blocks cached.
static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64];
static bool g_pool_ok[64];

static cudaError_t pool_for_current(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool_ok[dev]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    e = cudaMemPoolCreate(&g_pool[dev], &props);
    if (e != cudaSuccess) return e;
    uint64_t thr = ~0ull;
    cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &thr);
    g_pool_ok[dev] = true;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

// Optional cap on the bytes the pool holds for callers at any time (tuning key 9,
// MiB, 0 = none): an allocation that would take the pool's in-use bytes past it
// fails as out of memory, so callers can bound the library's footprint (and the
// allocation-failure paths can be exercised from the host).
static std::atomic<int64_t> g_pool_cap{0};

cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool;
  cudaError_t e = pool_for_current(&pool);
  if (e != cudaSuccess) return e;
  if (bytes == 0) bytes = 16;
  const int64_t cap = g_pool_cap.load(std::memory_order_relaxed);
  if (cap > 0) {
    uint64_t used = 0;
    e = cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    if (e != cudaSuccess) return e;
    if ((int64_t)(used + bytes) > cap) {
      *p = nullptr;
      return cudaErrorMemoryAllocation;
    }
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}
cudaError_t dev_free(void* p, cudaStream_t s) { return p ? cudaFreeAsync(p, s) : cudaSuccess; }

ckd_status build_dispatch(ckd_tree* t, const void* pts_dev, int dtype, cudaStream_t s);
ckd_status knn_run(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted, double* dist,
                   int64_t* idx, cudaStream_t s);
ckd_status knn_multi_k(const ckd_tree* t, const double* q, int64_t nq, const int32_t* kq,
                       int kmax, int sorted, double* dist, int64_t* idx, cudaStream_t s,
                       const ckd_mlp* net = nullptr, int64_t* nfb_out = nullptr);
ckd_status knn_host_pipelined(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted,
                              double* dist, int64_t* idx, cudaStream_t s);
void release_host_staging();
ckd_status knn_ordered(const ckd_tree* t, const double* q, const int32_t* order, int64_t nq, int k,
                       int sorted, double* dist, int64_t* idx, cudaStream_t s);
ckd_status query_order(const ckd_tree* t, const double* q_dev, int64_t nq, int32_t* order,
                       cudaStream_t s);
ckd_status knn_stats(int enable, int64_t* out);
ckd_status knn_noalloc(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted,
                       double* dist, int64_t* idx, cudaStream_t s);
ckd_status knn_learned(const ckd_tree* t, const ckd_mlp* net, const double* q, int64_t nq, int k,
                       int sorted, double* dist, int64_t* idx, int64_t* nfb, cudaStream_t s);
ckd_status ball_run(const ckd_tree* t, const double* q, int64_t nq, double r, bool fill, int sorted,
                    int64_t* counts, const int64_t* offsets, int64_t* idx, double* dist,
                    cudaStream_t s,
                    const int32_t* qroot = nullptr);
ckd_status box_run(const ckd_tree* t, const double* boxes, int64_t nb, bool fill, int64_t* counts,
                   const int64_t* offsets, int64_t* idx, cudaStream_t s,
                   const int32_t* broot = nullptr);
ckd_status forest_knn(const ckd_tree* t, const double* q, const int32_t* qroot, int64_t nq, int k,
                      int sorted, double* dist, int64_t* idx, cudaStream_t s);

static ckd_status check_device(int* dev_out) {
  int dev = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  int major = 0;
  CKD_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) return fail(CKD_ERR_NO_DEVICE, "libckd is built for sm_100a (B200) devices only");
  if (dev_out) *dev_out = dev;
  return CKD_OK;
}

static ckd_status check_tree(const ckd_tree* t) {
  if (!t) return fail(CKD_ERR_BAD_ARG, "null tree handle");
  int dev = 0;
  CKD_CUDA(cudaGetDevice(&dev));
  if (dev != t->device) return fail(CKD_ERR_BAD_ARG, "the current device is not the tree's device");
  return CKD_OK;
}

// Tree arrays come from the library's stream-ordered pool (a freed tree's memory
// is reused by the next build without new device mappings).  Work that may still
// read the tree ends first, as with cudaFree.
static void release_tree(ckd_tree* t) {
  if (!t) return;
  cudaDeviceSynchronize();
  void* ps[] = {t->meta, t->box,   t->cell, t->pts,    t->ids,   t->box32,
                t->pts32, t->pts64, t->pair, t->cell32, t->centre};
  for (void* p : ps)
    if (p) cudaFreeAsync(p, 0);
  delete t;
}

void release_tree_handle(ckd_tree* t) { release_tree(t); }

}  // namespace ckd

using namespace ckd;

extern "C" {

int ckd_version(void) { return 100; }

const char* ckd_last_error(void) { return g_err.c_str(); }

}  // extern "C"

namespace ckd {
// Shared by ckd_build and ckd_forest_build: off = tree offsets (n_trees + 1).
static ckd_status build_common(const void* pts, int64_t n, int d, int dtype, int leaf,
                               const double* boxsize, int pts_on_device, void* stream,
                               std::vector<int64_t> off, ckd_tree** out) {
  if (!out) return fail(CKD_ERR_BAD_ARG, "null output handle pointer");
  *out = nullptr;
  if (!pts) return fail(CKD_ERR_BAD_ARG, "null points pointer");
  if (n < 1) return fail(CKD_ERR_BAD_ARG, "at least one point is required");
  if (n >= 0x7fffffffll) return fail(CKD_ERR_BAD_ARG, "more than 2^31-2 points are not supported");
  if (d < 1 || d > CKD_MAX_D) return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
  if (leaf < 1) return fail(CKD_ERR_BAD_ARG, "Leaf size must be a positive integer");
  if (dtype != CKD_F64 && dtype != CKD_F32) return fail(CKD_ERR_BAD_ARG, "dtype must be F64 or F32");
  int dev = 0;
  CKD_TRY(check_device(&dev));
  cudaStream_t s = (cudaStream_t)stream;
  ckd_tree* t = new ckd_tree();
  t->device = dev;
  t->n = n;
  t->n_trees = (int64_t)off.size() - 1;
  t->tree_off = std::move(off);
  t->d = d;
  t->leaf = leaf;
  t->input_dtype = dtype;
  if (boxsize) {
    t->periodic = 1;
    for (int j = 0; j < d; ++j) {
      if (!(boxsize[j] > 0) || !std::isfinite(boxsize[j])) {
        delete t;
        return fail(CKD_ERR_BAD_ARG, "boxsize entries must be positive and finite");
      }
      t->L[j] = boxsize[j];
    }
  }
  const void* src = pts;
  void* staging = nullptr;
  size_t esz = dtype == CKD_F32 ? 4 : 8;
  ckd_status st = CKD_OK;
  if (!pts_on_device) {
    cudaError_t e = dev_alloc(&staging, esz * n * d, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(staging, pts, esz * n * d, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) st = cuda_fail(e, "copying points to the device");
    src = staging;
  }
  if (st == CKD_OK) st = build_dispatch(t, src, dtype, s);
  if (staging) dev_free(staging, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (st == CKD_OK && e != cudaSuccess) st = cuda_fail(e, "build");
  if (st != CKD_OK) {
    release_tree(t);
    return st;
  }
  *out = t;
  return CKD_OK;
}

static ckd_status check_single(const ckd_tree* t) {
  CKD_TRY(check_tree(t));
  if (t->n_trees != 1)
    return fail(CKD_ERR_BAD_ARG, "the handle is a forest; use the ckd_forest_* entry points");
  return CKD_OK;
}

static ckd_status check_forest(const ckd_tree* t) {
  CKD_TRY(check_tree(t));
  return CKD_OK;
}
}  // namespace ckd

extern "C" {

ckd_status ckd_build(const void* pts, int64_t n, int d, int dtype, int leaf, const double* boxsize,
                     int pts_on_device, void* stream, ckd_tree** out) {
  return build_common(pts, n, d, dtype, leaf, boxsize, pts_on_device, stream, {0, n}, out);
}

ckd_status ckd_forest_build(const void* pts, const int64_t* offsets, int64_t n_trees, int d,
                            int dtype, int leaf, const double* boxsize, int pts_on_device,
                            void* stream, ckd_tree** out) {
  if (out) *out = nullptr;
  if (!offsets || n_trees < 1) return fail(CKD_ERR_BAD_ARG, "a forest needs offsets of >= 1 trees");
  if (n_trees >= 0x7fffffffll) return fail(CKD_ERR_BAD_ARG, "too many trees");
  std::vector<int64_t> off(offsets, offsets + n_trees + 1);
  if (off[0] != 0) return fail(CKD_ERR_BAD_ARG, "forest offsets must start at 0");
  for (int64_t i = 0; i < n_trees; ++i)
    if (off[i + 1] <= off[i]) return fail(CKD_ERR_BAD_ARG, "every tree needs at least one point");
  const int64_t total = off[n_trees];  // before `off` is moved into the call
  return build_common(pts, total, d, dtype, leaf, boxsize, pts_on_device, stream, std::move(off),
                      out);
}

ckd_status ckd_forest_info(const ckd_tree* t, int64_t* n_trees, int64_t* offsets) {
  if (!t) return fail(CKD_ERR_BAD_ARG, "null tree handle");
  if (n_trees) *n_trees = t->n_trees;
  if (offsets) std::memcpy(offsets, t->tree_off.data(), sizeof(int64_t) * t->tree_off.size());
  return CKD_OK;
}

ckd_status ckd_forest_knn(const ckd_tree* t, const double* q, const int64_t* q_offsets, int64_t nq,
                          int k, int sorted, double* dist, int64_t* idx, void* stream) {
  CKD_TRY(check_forest(t));
  if (k < 1) return fail(CKD_ERR_BAD_ARG, "k must be a positive integer");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !q_offsets || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query, offset or output pointer");
  if (nq > INT32_MAX) return fail(CKD_ERR_BAD_ARG, "at most 2^31 - 1 queries per call");
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* qroot = nullptr;
  CKD_CUDA(dev_alloc((void**)&qroot, sizeof(int32_t) * nq, s));
  ckd_status st = csr_owner(q_offsets, (int32_t)t->n_trees, nq, qroot, s);
  if (st == CKD_OK) st = forest_knn(t, q, qroot, nq, k, sorted, dist, idx, s);
  dev_free(qroot, s);
  return st;
}

static ckd_status forest_box(const ckd_tree* t, const double* boxes, const int64_t* b_offsets,
                             int64_t nb, bool fill, int64_t* counts, const int64_t* offsets,
                             int64_t* idx, void* stream) {
  CKD_TRY(check_forest(t));
  if (nb < 0) return fail(CKD_ERR_BAD_ARG, "negative box count");
  if (nb == 0) return CKD_OK;
  if (!boxes || !b_offsets || (fill ? (!offsets || !idx) : !counts))
    return fail(CKD_ERR_BAD_ARG, "null box, offset or output pointer");
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* broot = nullptr;
  CKD_CUDA(dev_alloc((void**)&broot, sizeof(int32_t) * nb, s));
  ckd_status st = csr_owner(b_offsets, (int32_t)t->n_trees, nb, broot, s);
  if (st == CKD_OK) st = box_run(t, boxes, nb, fill, counts, offsets, idx, s, broot);
  dev_free(broot, s);
  return st;
}

ckd_status ckd_forest_box_count(const ckd_tree* t, const double* boxes, const int64_t* b_offsets,
                                int64_t nb, int64_t* counts, void* stream) {
  return forest_box(t, boxes, b_offsets, nb, false, counts, nullptr, nullptr, stream);
}

ckd_status ckd_forest_box_fill(const ckd_tree* t, const double* boxes, const int64_t* b_offsets,
                               int64_t nb, const int64_t* offsets, int64_t* idx, void* stream) {
  return forest_box(t, boxes, b_offsets, nb, true, nullptr, offsets, idx, stream);
}

static ckd_status forest_ball(const ckd_tree* t, const double* q, const int64_t* q_offsets,
                              int64_t nq, double radius, bool fill, int sorted, int64_t* counts,
                              const int64_t* offsets, int64_t* idx, double* dist, void* stream) {
  CKD_TRY(check_forest(t));
  if (!(radius > 0) || !std::isfinite(radius))
    return fail(CKD_ERR_BAD_ARG, "Radius must be a positive number");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !q_offsets || (fill ? (!offsets || !idx || !dist) : !counts))
    return fail(CKD_ERR_BAD_ARG, "null query, offset or output pointer");
  if (nq > INT32_MAX) return fail(CKD_ERR_BAD_ARG, "at most 2^31 - 1 queries per call");
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* qroot = nullptr;
  CKD_CUDA(dev_alloc((void**)&qroot, sizeof(int32_t) * nq, s));
  ckd_status st = csr_owner(q_offsets, (int32_t)t->n_trees, nq, qroot, s);
  if (st == CKD_OK)
    st = ball_run(t, q, nq, radius, fill, sorted, counts, offsets, idx, dist, s, qroot);
  dev_free(qroot, s);
  return st;
}

ckd_status ckd_forest_ball_count(const ckd_tree* t, const double* q, const int64_t* q_offsets,
                                 int64_t nq, double radius, int64_t* counts, void* stream) {
  return forest_ball(t, q, q_offsets, nq, radius, false, 0, counts, nullptr, nullptr, nullptr,
                     stream);
}

ckd_status ckd_forest_ball_fill(const ckd_tree* t, const double* q, const int64_t* q_offsets,
                                int64_t nq, double radius, int sorted, const int64_t* offsets,
                                int64_t* idx, double* dist, void* stream) {
  return forest_ball(t, q, q_offsets, nq, radius, true, sorted, nullptr, offsets, idx, dist,
                     stream);
}

ckd_status ckd_pool_usage(int64_t* used, int64_t* reserved) {
  cudaMemPool_t pool;
  CKD_CUDA(pool_for_current(&pool));
  uint64_t u = 0, r = 0;
  CKD_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
  CKD_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
  if (used) *used = (int64_t)u;
  if (reserved) *reserved = (int64_t)r;
  return CKD_OK;
}

ckd_status ckd_release_cached_memory(void) {
  cudaMemPool_t pool;
  CKD_CUDA(pool_for_current(&pool));
  CKD_CUDA(cudaDeviceSynchronize());
  CKD_CUDA(cudaMemPoolTrimTo(pool, 0));
  release_host_staging();
  return CKD_OK;
}

ckd_status ckd_free(ckd_tree* tree) {
  if (!tree) return CKD_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(tree->device);
  release_tree(tree);
  cudaSetDevice(cur);
  return CKD_OK;
}

ckd_status ckd_tree_info(const ckd_tree* t, int64_t* n, int* d, int* leaf, int* periodic,
                         int32_t* n_nodes, int32_t* n_leaves, int32_t* depth, int* device) {
  if (!t) return fail(CKD_ERR_BAD_ARG, "null tree handle");
  if (n) *n = t->n;
  if (d) *d = t->d;
  if (leaf) *leaf = t->leaf;
  if (periodic) *periodic = t->periodic;
  if (n_nodes) *n_nodes = t->n_nodes;
  if (n_leaves) *n_leaves = t->n_leaves;
  if (depth) *depth = t->depth;
  if (device) *device = t->device;
  return CKD_OK;
}

ckd_status ckd_tree_export(const ckd_tree* t, int32_t* axis, double* split, int64_t* start,
                           int64_t* count, int64_t* left, int64_t* right, double* cell, double* box,
                           int64_t* ids) {
  CKD_TRY(check_single(t));
  const int m = t->n_nodes, d2 = 2 * t->d;
  std::vector<NodeMeta> meta(m);
  std::vector<double> hc((size_t)m * d2), hb((size_t)m * d2);
  CKD_CUDA(cudaMemcpy(meta.data(), t->meta, sizeof(NodeMeta) * m, cudaMemcpyDeviceToHost));
  if (cell) CKD_CUDA(cudaMemcpy(hc.data(), t->cell, sizeof(double) * m * d2, cudaMemcpyDeviceToHost));
  if (box) CKD_CUDA(cudaMemcpy(hb.data(), t->box, sizeof(double) * m * d2, cudaMemcpyDeviceToHost));
  if (ids) {
    std::vector<int32_t> hi(t->n);
    CKD_CUDA(cudaMemcpy(hi.data(), t->ids, sizeof(int32_t) * t->n, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < t->n; ++i) ids[i] = hi[i];
  }
  // preorder, left subtree first
  std::vector<int32_t> pre(m, -1);
  std::vector<int32_t> order;
  order.reserve(m);
  std::vector<int32_t> st{0};
  while (!st.empty()) {
    int32_t a = st.back();
    st.pop_back();
    pre[a] = (int32_t)order.size();
    order.push_back(a);
    if (meta[a].left >= 0) {
      st.push_back(meta[a].left + 1);
      st.push_back(meta[a].left);
    }
  }
  if ((int)order.size() != m) return fail(CKD_ERR_CUDA, "internal error: tree is not connected");
  for (int i = 0; i < m; ++i) {
    const NodeMeta& x = meta[order[i]];
    bool lf = x.left < 0;
    if (axis) axis[i] = lf ? -1 : x.axis;
    if (split) split[i] = lf ? 0.0 : x.split;
    if (start) start[i] = x.start;
    if (count) count[i] = x.count;
    if (left) left[i] = lf ? -1 : pre[x.left];
    if (right) right[i] = lf ? -1 : pre[x.left + 1];
    if (cell) std::memcpy(cell + (size_t)i * d2, &hc[(size_t)order[i] * d2], sizeof(double) * d2);
    if (box) std::memcpy(box + (size_t)i * d2, &hb[(size_t)order[i] * d2], sizeof(double) * d2);
  }
  return CKD_OK;
}

ckd_status ckd_knn(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted, double* dist,
                   int64_t* idx, void* stream) {
  CKD_TRY(check_single(t));
  if (k < 1) return fail(CKD_ERR_BAD_ARG, "k must be a positive integer");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  return knn_run(t, q, nq, k, sorted, dist, idx, (cudaStream_t)stream);
}

ckd_status ckd_knn_multi_k(const ckd_tree* t, const double* q, int64_t nq, const int32_t* k_dev,
                           int kmax, int sorted, double* dist, int64_t* idx, void* stream) {
  CKD_TRY(check_single(t));
  if (kmax < 1 || kmax > 65536) return fail(CKD_ERR_BAD_ARG, "kmax must be 1..65536");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !k_dev || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query, k or output pointer");
  if (nq > INT32_MAX) return fail(CKD_ERR_BAD_ARG, "at most 2^31 - 1 queries per call");
  return knn_multi_k(t, q, nq, k_dev, kmax, sorted, dist, idx, (cudaStream_t)stream);
}

ckd_status ckd_knn_learned_multi_k(const ckd_tree* t, const ckd_mlp* net, const double* q,
                                   int64_t nq, const int32_t* k_dev, int kmax, int sorted,
                                   double* dist, int64_t* idx, int64_t* n_fallback,
                                   void* stream) {
  CKD_TRY(check_single(t));
  CKD_TRY(mlp_check(net));
  if (kmax < 1 || kmax > 65536) return fail(CKD_ERR_BAD_ARG, "kmax must be 1..65536");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (n_fallback) *n_fallback = 0;
  if (nq == 0) return CKD_OK;
  if (!q || !k_dev || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query, k or output pointer");
  if (nq > INT32_MAX) return fail(CKD_ERR_BAD_ARG, "at most 2^31 - 1 queries per call");
  return knn_multi_k(t, q, nq, k_dev, kmax, sorted, dist, idx, (cudaStream_t)stream, net,
                     n_fallback);
}

ckd_status ckd_query_order(const ckd_tree* t, const double* q, int64_t nq, int32_t* order,
                           void* stream) {
  CKD_TRY(check_single(t));
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !order) return fail(CKD_ERR_BAD_ARG, "null query or order pointer");
  return query_order(t, q, nq, order, (cudaStream_t)stream);
}

ckd_status ckd_knn_ordered(const ckd_tree* t, const double* q, int64_t nq, const int32_t* order,
                           int k, int sorted, double* dist, int64_t* idx, void* stream) {
  CKD_TRY(check_single(t));
  if (k < 1) return fail(CKD_ERR_BAD_ARG, "k must be a positive integer");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  return knn_ordered(t, q, order, nq, k, sorted, dist, idx, (cudaStream_t)stream);
}

int64_t ckd_launch_count(void) { return g_launches.load(); }

ckd_status ckd_knn_stats(int enable, int64_t* out8) { return knn_stats(enable, out8); }

ckd_status ckd_set_knn_variant(int variant) {
  if (!(variant == 0 || variant == 1 || variant == 7 || variant == 8))
    return fail(CKD_ERR_BAD_ARG, "kNN variant must be 0, 1, 7 or 8");
  g_knn_variant.store(variant);
  return CKD_OK;
}

ckd_status ckd_set_kernel_timing(int enable) {
  g_timing.store(enable ? 1 : 0);
  return CKD_OK;
}

ckd_status ckd_kernel_ms(float* ms) {
  if (!ms) return fail(CKD_ERR_BAD_ARG, "null output");
  *ms = -1.0f;
  if (!g_ev_recorded) return CKD_OK;
  CKD_CUDA(cudaEventSynchronize(g_ev[1]));
  CKD_CUDA(cudaEventElapsedTime(ms, g_ev[0], g_ev[1]));
  return CKD_OK;
}

ckd_status ckd_set_tuning(int key, int value) {
  switch (key) {
    case 0: return ckd_set_knn_variant(value);
    case 1:
      if (value < 0 || value > 64) return fail(CKD_ERR_BAD_ARG, "blocks per SM must be 0..64");
      g_knn_bps.store(value);
      return CKD_OK;
    case 2:
      if (value < 1 || value > 8) return fail(CKD_ERR_BAD_ARG, "warps per block must be 1..8");
      g_knn_wpb.store(value);
      return CKD_OK;
    case 4:
      if (!(value == 0 || value == 3))
        return fail(CKD_ERR_BAD_ARG, "learned kernel must be 0 or 3");
      g_learned_kernel.store(value);
      return CKD_OK;
    case 6:
      if (value < 0 || value > 2) return fail(CKD_ERR_BAD_ARG, "query ordering must be 0, 1 or 2");
      g_order_mode.store(value);
      return CKD_OK;
    case 7:
      if (value < 0 || value > 1) return fail(CKD_ERR_BAD_ARG, "MLP inference path must be 0 or 1");
      g_mlp_tc.store(value);
      return CKD_OK;
    case 8:
      if (value < 0 || value > 1) return fail(CKD_ERR_BAD_ARG, "box kernel choice must be 0 or 1");
      g_box_warp.store(value);
      return CKD_OK;
    case 9:
      if (value < 0) return fail(CKD_ERR_BAD_ARG, "pool cap must be >= 0 MiB");
      g_pool_cap.store((int64_t)value << 20);
      return CKD_OK;
    case 10:
      if (value < 1 || value > 600000) return fail(CKD_ERR_BAD_ARG, "queue wait must be 1..600000 ms");
      g_pk_wait_ms.store(value);
      return CKD_OK;
    case 11:
      if (value < 0) return fail(CKD_ERR_BAD_ARG, "withheld items must be >= 0");
      g_pk_withhold.store(value);
      return CKD_OK;

  }
  return fail(CKD_ERR_BAD_ARG, "unknown tuning key");
}

ckd_status ckd_knn_noalloc(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted,
                           double* dist, int64_t* idx, void* stream) {
  CKD_TRY(check_single(t));
  if (k < 1) return fail(CKD_ERR_BAD_ARG, "k must be a positive integer");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  return knn_noalloc(t, q, nq, k, sorted, dist, idx, (cudaStream_t)stream);
}

ckd_status ckd_knn_learned(const ckd_tree* t, const ckd_mlp* net, const double* q, int64_t nq,
                           int k, int sorted, double* dist, int64_t* idx, int64_t* n_fallback,
                           void* stream) {
  CKD_TRY(check_single(t));
  CKD_TRY(mlp_check(net));
  if (k < 1) return fail(CKD_ERR_BAD_ARG, "k must be a positive integer");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (n_fallback) *n_fallback = 0;
  if (nq == 0) return CKD_OK;
  if (!q || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  if (nq > INT32_MAX) return fail(CKD_ERR_BAD_ARG, "at most 2^31 - 1 queries per call");
  return knn_learned(t, net, q, nq, k, sorted, dist, idx, n_fallback, (cudaStream_t)stream);
}

// Host buffers from this many queries on take the chunked pipeline (host_pipe.cu).
constexpr int64_t kHostPipeRows = int64_t(1) << 20;

ckd_status ckd_knn_host(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted,
                        double* dist, int64_t* idx, void* stream) {
  CKD_TRY(check_single(t));
  if (k < 1) return fail(CKD_ERR_BAD_ARG, "k must be a positive integer");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !dist || !idx) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (nq >= kHostPipeRows && k <= (1 << 20))
    return knn_host_pipelined(t, q, nq, k, sorted, dist, idx, s);
  double *dq = nullptr, *dd = nullptr;
  int64_t* di = nullptr;
  ckd_status st = CKD_OK;
  cudaError_t e = dev_alloc((void**)&dq, sizeof(double) * nq * t->d, s);
  if (e == cudaSuccess) e = dev_alloc((void**)&dd, sizeof(double) * nq * k, s);
  if (e == cudaSuccess) e = dev_alloc((void**)&di, sizeof(int64_t) * nq * k, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dq, q, sizeof(double) * nq * t->d, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) st = cuda_fail(e, "ckd_knn_host: device buffers");
  if (st == CKD_OK) st = knn_run(t, dq, nq, k, sorted, dd, di, s);
  if (st == CKD_OK) {
    e = cudaMemcpyAsync(dist, dd, sizeof(double) * nq * k, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(idx, di, sizeof(int64_t) * nq * k, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) st = cuda_fail(e, "ckd_knn_host: result copy");
  }
  dev_free(dq, s);
  dev_free(dd, s);
  dev_free(di, s);
  e = cudaStreamSynchronize(s);
  if (st == CKD_OK && e != cudaSuccess) st = cuda_fail(e, "ckd_knn_host");
  return st;
}

ckd_status ckd_ball_count(const ckd_tree* t, const double* q, int64_t nq, double radius,
                          int64_t* counts, void* stream) {
  CKD_TRY(check_single(t));
  if (!(radius > 0) || !std::isfinite(radius))
    return fail(CKD_ERR_BAD_ARG, "Radius must be a positive number");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !counts) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  return ball_run(t, q, nq, radius, false, 0, counts, nullptr, nullptr, nullptr,
                  (cudaStream_t)stream);
}

ckd_status ckd_ball_fill(const ckd_tree* t, const double* q, int64_t nq, double radius, int sorted,
                         const int64_t* offsets, int64_t* idx, double* dist, void* stream) {
  CKD_TRY(check_single(t));
  if (!(radius > 0) || !std::isfinite(radius))
    return fail(CKD_ERR_BAD_ARG, "Radius must be a positive number");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !offsets || !idx || !dist) return fail(CKD_ERR_BAD_ARG, "null query or output pointer");
  return ball_run(t, q, nq, radius, true, sorted, nullptr, offsets, idx, dist,
                  (cudaStream_t)stream);
}

ckd_status ckd_box_count(const ckd_tree* t, const double* boxes, int64_t nb, int64_t* counts,
                         void* stream) {
  CKD_TRY(check_single(t));
  if (nb < 0) return fail(CKD_ERR_BAD_ARG, "negative box count");
  if (nb == 0) return CKD_OK;
  if (!boxes || !counts) return fail(CKD_ERR_BAD_ARG, "null box or output pointer");
  return box_run(t, boxes, nb, false, counts, nullptr, nullptr, (cudaStream_t)stream);
}

ckd_status ckd_box_fill(const ckd_tree* t, const double* boxes, int64_t nb, const int64_t* offsets,
                        int64_t* idx, void* stream) {
  CKD_TRY(check_single(t));
  if (nb < 0) return fail(CKD_ERR_BAD_ARG, "negative box count");
  if (nb == 0) return CKD_OK;
  if (!boxes || !offsets || !idx) return fail(CKD_ERR_BAD_ARG, "null box or output pointer");
  return box_run(t, boxes, nb, true, nullptr, offsets, idx, (cudaStream_t)stream);
}

// ---------------------------------------------- two-phase CSR on host buffers
// For callers without device memory of their own (Fortran, C, other FFIs): the
// count phase returns the CSR offsets in host memory, the caller allocates the
// rows and the fill phase writes them.  Both phases are synchronous.
namespace {
struct DevScratch {
  cudaStream_t s;
  std::vector<void*> ps;
  void* get(size_t bytes, cudaError_t& e) {
    void* p = nullptr;
    e = dev_alloc(&p, bytes, s);
    if (e == cudaSuccess) ps.push_back(p);
    return p;
  }
  ~DevScratch() {
    for (void* p : ps) dev_free(p, s);
    cudaStreamSynchronize(s);
  }
};

ckd_status offsets_to_host(const int64_t* counts, int64_t n, int64_t* offsets_host,
                           DevScratch& sc) {
  cudaError_t e;
  int64_t* off = (int64_t*)sc.get(sizeof(int64_t) * (n + 1), e);
  CKD_CUDA(e);
  CKD_TRY(scan_i64(counts, off, n, sc.s));
  CKD_CUDA(cudaMemcpyAsync(offsets_host, off, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost,
                           sc.s));
  CKD_CUDA(cudaStreamSynchronize(sc.s));
  return CKD_OK;
}
}  // namespace

ckd_status ckd_ball_count_host(const ckd_tree* t, const double* q, int64_t nq, double radius,
                               int64_t* offsets_host, void* stream) {
  CKD_TRY(check_single(t));
  if (!(radius > 0) || !std::isfinite(radius))
    return fail(CKD_ERR_BAD_ARG, "Radius must be a positive number");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (!offsets_host) return fail(CKD_ERR_BAD_ARG, "null offsets pointer");
  offsets_host[0] = 0;
  if (nq == 0) return CKD_OK;
  if (!q) return fail(CKD_ERR_BAD_ARG, "null query pointer");
  DevScratch sc{(cudaStream_t)stream, {}};
  cudaError_t e;
  double* dq = (double*)sc.get(sizeof(double) * nq * t->d, e);
  CKD_CUDA(e);
  int64_t* cnt = (int64_t*)sc.get(sizeof(int64_t) * nq, e);
  CKD_CUDA(e);
  CKD_CUDA(cudaMemcpyAsync(dq, q, sizeof(double) * nq * t->d, cudaMemcpyHostToDevice, sc.s));
  CKD_TRY(ball_run(t, dq, nq, radius, false, 0, cnt, nullptr, nullptr, nullptr, sc.s));
  return offsets_to_host(cnt, nq, offsets_host, sc);
}

ckd_status ckd_ball_fill_host(const ckd_tree* t, const double* q, int64_t nq, double radius,
                              int sorted, const int64_t* offsets_host, int64_t* idx_host,
                              double* dist_host, void* stream) {
  CKD_TRY(check_single(t));
  if (!(radius > 0) || !std::isfinite(radius))
    return fail(CKD_ERR_BAD_ARG, "Radius must be a positive number");
  if (nq < 0) return fail(CKD_ERR_BAD_ARG, "negative query count");
  if (nq == 0) return CKD_OK;
  if (!q || !offsets_host) return fail(CKD_ERR_BAD_ARG, "null query or offsets pointer");
  const int64_t total = offsets_host[nq];
  if (total < 0) return fail(CKD_ERR_BAD_ARG, "negative result count");
  if (total > 0 && (!idx_host || !dist_host)) return fail(CKD_ERR_BAD_ARG, "null output pointer");
  DevScratch sc{(cudaStream_t)stream, {}};
  cudaError_t e;
  double* dq = (double*)sc.get(sizeof(double) * nq * t->d, e);
  CKD_CUDA(e);
  int64_t* off = (int64_t*)sc.get(sizeof(int64_t) * (nq + 1), e);
  CKD_CUDA(e);
  int64_t* di = (int64_t*)sc.get(sizeof(int64_t) * std::max<int64_t>(total, 1), e);
  CKD_CUDA(e);
  double* dd = (double*)sc.get(sizeof(double) * std::max<int64_t>(total, 1), e);
  CKD_CUDA(e);
  CKD_CUDA(cudaMemcpyAsync(dq, q, sizeof(double) * nq * t->d, cudaMemcpyHostToDevice, sc.s));
  CKD_CUDA(cudaMemcpyAsync(off, offsets_host, sizeof(int64_t) * (nq + 1), cudaMemcpyHostToDevice,
                           sc.s));
  if (total > 0) {
    CKD_TRY(ball_run(t, dq, nq, radius, true, sorted, nullptr, off, di, dd, sc.s));
    CKD_CUDA(cudaMemcpyAsync(idx_host, di, sizeof(int64_t) * total, cudaMemcpyDeviceToHost, sc.s));
    CKD_CUDA(cudaMemcpyAsync(dist_host, dd, sizeof(double) * total, cudaMemcpyDeviceToHost, sc.s));
  }
  CKD_CUDA(cudaStreamSynchronize(sc.s));
  return CKD_OK;
}

ckd_status ckd_box_count_host(const ckd_tree* t, const double* boxes, int64_t nb,
                              int64_t* offsets_host, void* stream) {
  CKD_TRY(check_single(t));
  if (nb < 0) return fail(CKD_ERR_BAD_ARG, "negative box count");
  if (!offsets_host) return fail(CKD_ERR_BAD_ARG, "null offsets pointer");
  offsets_host[0] = 0;
  if (nb == 0) return CKD_OK;
  if (!boxes) return fail(CKD_ERR_BAD_ARG, "null box pointer");
  DevScratch sc{(cudaStream_t)stream, {}};
  cudaError_t e;
  double* db = (double*)sc.get(sizeof(double) * nb * 2 * t->d, e);
  CKD_CUDA(e);
  int64_t* cnt = (int64_t*)sc.get(sizeof(int64_t) * nb, e);
  CKD_CUDA(e);
  CKD_CUDA(cudaMemcpyAsync(db, boxes, sizeof(double) * nb * 2 * t->d, cudaMemcpyHostToDevice, sc.s));
  CKD_TRY(box_run(t, db, nb, false, cnt, nullptr, nullptr, sc.s));
  return offsets_to_host(cnt, nb, offsets_host, sc);
}

ckd_status ckd_box_fill_host(const ckd_tree* t, const double* boxes, int64_t nb,
                             const int64_t* offsets_host, int64_t* idx_host, void* stream) {
  CKD_TRY(check_single(t));
  if (nb < 0) return fail(CKD_ERR_BAD_ARG, "negative box count");
  if (nb == 0) return CKD_OK;
  if (!boxes || !offsets_host) return fail(CKD_ERR_BAD_ARG, "null box or offsets pointer");
  const int64_t total = offsets_host[nb];
  if (total < 0) return fail(CKD_ERR_BAD_ARG, "negative result count");
  if (total > 0 && !idx_host) return fail(CKD_ERR_BAD_ARG, "null output pointer");
  DevScratch sc{(cudaStream_t)stream, {}};
  cudaError_t e;
  double* db = (double*)sc.get(sizeof(double) * nb * 2 * t->d, e);
  CKD_CUDA(e);
  int64_t* off = (int64_t*)sc.get(sizeof(int64_t) * (nb + 1), e);
  CKD_CUDA(e);
  int64_t* di = (int64_t*)sc.get(sizeof(int64_t) * std::max<int64_t>(total, 1), e);
  CKD_CUDA(e);
  CKD_CUDA(cudaMemcpyAsync(db, boxes, sizeof(double) * nb * 2 * t->d, cudaMemcpyHostToDevice, sc.s));
  CKD_CUDA(cudaMemcpyAsync(off, offsets_host, sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice,
                           sc.s));
  if (total > 0) {
    CKD_TRY(box_run(t, db, nb, true, nullptr, off, di, sc.s));
    CKD_CUDA(cudaMemcpyAsync(idx_host, di, sizeof(int64_t) * total, cudaMemcpyDeviceToHost, sc.s));
  }
  CKD_CUDA(cudaStreamSynchronize(sc.s));
  return CKD_OK;
}

ckd_status ckd_exclusive_scan(const int64_t* in, int64_t* out, int64_t n, void* stream) {
  if (n < 0 || !out || (n > 0 && !in)) return fail(CKD_ERR_BAD_ARG, "bad scan arguments");
  return scan_i64(in, out, n, (cudaStream_t)stream);
}

}  // extern "C"

// ------------------------------------------------- persistent forest plans
namespace ckd {
struct ForestPlan;
ckd_status forest_plan_create(const double* pts_dev, const int64_t* offsets, int64_t T, int d,
                              int leaf, const double* boxsize, const double* q_dev,
                              const int64_t* q_offsets, int64_t nq, int k, int sorted,
                              double* dist_dev, int64_t* idx_dev, double node_factor,
                              int qblock, ForestPlan** out);
ckd_status forest_plan_run(ForestPlan* p, cudaStream_t s, int withhold, long long spin_limit);
ckd_status forest_plan_status(ForestPlan* p, cudaStream_t s);
const ckd_tree* forest_plan_tree(const ForestPlan* p);
void forest_plan_release(ForestPlan* p);
}  // namespace ckd

extern "C" {

ckd_status ckd_forest_plan_create(const double* pts_dev, const int64_t* offsets_host,
                                  int64_t n_trees, int d, int leaf, const double* boxsize,
                                  const double* q_dev, const int64_t* q_offsets_host, int64_t nq,
                                  int k, int sorted, double* dist_dev, int64_t* idx_dev,
                                  double node_factor, int queries_per_block,
                                  ckd_forest_plan** out) {
  if (!out) return fail(CKD_ERR_BAD_ARG, "null output handle pointer");
  *out = nullptr;
  int dev = 0;
  CKD_TRY(check_device(&dev));
  ForestPlan* p = nullptr;
  CKD_TRY(forest_plan_create(pts_dev, offsets_host, n_trees, d, leaf, boxsize, q_dev,
                             q_offsets_host, nq, k, sorted, dist_dev, idx_dev, node_factor,
                             queries_per_block, &p));
  *out = reinterpret_cast<ckd_forest_plan*>(p);
  return CKD_OK;
}

ckd_status ckd_forest_plan_run(ckd_forest_plan* plan, void* stream) {
  if (!plan) return fail(CKD_ERR_BAD_ARG, "null plan");
  const long long polls = (long long)g_pk_wait_ms.load() * 2000;
  return forest_plan_run(reinterpret_cast<ForestPlan*>(plan), (cudaStream_t)stream,
                         g_pk_withhold.load(), polls);
}

ckd_status ckd_forest_plan_status(ckd_forest_plan* plan, void* stream) {
  if (!plan) return fail(CKD_ERR_BAD_ARG, "null plan");
  return forest_plan_status(reinterpret_cast<ForestPlan*>(plan), (cudaStream_t)stream);
}

ckd_status ckd_forest_plan_forest(const ckd_forest_plan* plan, const ckd_tree** forest) {
  if (!plan || !forest) return fail(CKD_ERR_BAD_ARG, "null plan or output");
  *forest = forest_plan_tree(reinterpret_cast<const ForestPlan*>(plan));
  return CKD_OK;
}

ckd_status ckd_forest_plan_free(ckd_forest_plan* plan) {
  forest_plan_release(reinterpret_cast<ForestPlan*>(plan));
  return CKD_OK;
}

}  // extern "C"
