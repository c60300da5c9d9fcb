/* ckd.h -- C ABI of libckd, the B200 (sm_100a) k-d tree library.
 *
 * Drop-in boundary for cosmokdtree's build_kdtree / knn_search / ball_search /
 * box_search path.  Every entry point is extern "C", takes plain pointers and
 * sizes, returns a ckd_status and never aborts the process (the reference STOPs:
 * src/cosmokdtree.f90:161,170,190; src/cosmokdtree2py.f90:58,276).  On failure
 * ckd_last_error() returns a message for the calling thread.
 *
 * Pointers suffixed _dev are device pointers on the tree's device; _host
 * variants take host memory and do the copies themselves.  `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).  Device-pointer
 * calls are asynchronous on `stream` unless stated otherwise.
 *
 * Ids are 0-based int64 (the reference returns 1-based ids that
 * src/cosmokdtree/kdtree.py:52,75,86 shift with `idx -= 1`).  A kNN slot with no
 * neighbour (k > n) holds id -2 and distance sqrt(FLT_MAX) = 1.8446743523953730e19,
 * the values the reference's Python API returns.
 */
#ifndef CKD_H_
#define CKD_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ckd_status {
  CKD_OK = 0,
  CKD_ERR_BAD_DIM = 1,     /* dimensionality mismatch / unsupported D */
  CKD_ERR_OUT_OF_BOX = 2,  /* periodic: coordinate outside [-L/2, L/2] */
  CKD_ERR_BAD_ARG = 3,     /* null pointer, k <= 0, radius <= 0, n < 1, NaN, ... */
  CKD_ERR_OOM = 4,         /* device allocation failed */
  CKD_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
  CKD_ERR_CUDA = 6,        /* any other CUDA runtime error */
  CKD_ERR_NO_DEVICE = 7,   /* no usable sm_100 device */
  CKD_ERR_DEPTH = 8        /* tree deeper than the build's level cap */
} ckd_status;

typedef enum ckd_dtype { CKD_F64 = 0, CKD_F32 = 1 } ckd_dtype;

typedef struct ckd_tree ckd_tree; /* opaque handle owning all device buffers */

/* Library version (major*10000 + minor*100 + patch). */
int ckd_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* ckd_last_error(void);

/* Build a tree.
 * Replaces pybuild_kdtree (src/cosmokdtree2py.f90:29-74) / build_kdtree
 * (src/cosmokdtree.f90:124-238).
 * pts: n x d row-major, dtype CKD_F64 or CKD_F32 (FP32 input is widened to FP64).
 * pts_on_device: 1 if pts is a device pointer, 0 if host memory.
 * leaf: leaf size (reference default 16).  boxsize: d box sides for a periodic
 * tree (coordinates must lie in [-L/2, L/2]), or NULL for a non-periodic tree.
 * Synchronises `stream` before returning. */
ckd_status ckd_build(const void* pts, int64_t n, int d, int dtype, int leaf,
                     const double* boxsize, int pts_on_device, void* stream, ckd_tree** out);

/* Free a tree and its device buffers (replaces pydeallocate_tree,
 * src/cosmokdtree2py.f90:80-97).  NULL is accepted.  Waits for the device to
 * finish pending work; the memory returns to the library's device pool, where
 * the next build reuses it. */
ckd_status ckd_free(ckd_tree* tree);

/* Return the memory cached in the current device's pool (freed trees and
 * scratch) to the driver.  No reference counterpart. */
ckd_status ckd_release_cached_memory(void);

/* Scalar properties of a built tree.  Any output pointer may be NULL. */
ckd_status ckd_tree_info(const ckd_tree* tree, int64_t* n, int* d, int* leaf, int* periodic,
                         int32_t* n_nodes, int32_t* n_leaves, int32_t* depth, int* device);

/* Copy the tree structure to host memory, nodes in preorder (left subtree first),
 * for structural comparison.  Each output may be NULL; sizes are n_nodes (per
 * node), n_nodes*2*d (cell, box) and n (ids, leaf order).  axis = -1 marks a leaf.
 * left/right are preorder indices (-1 for leaves).  Synchronous. */
ckd_status ckd_tree_export(const ckd_tree* tree, int32_t* axis, double* split, int64_t* start,
                           int64_t* count, int64_t* left, int64_t* right, double* cell,
                           double* box, int64_t* ids);

/* Exact k nearest neighbours of nq query points (row-major nq x d FP64).
 * Replaces pyknn_search (src/cosmokdtree2py.f90:103-143) / knn_search
 * (src/cosmokdtree.f90:504-540).  Results ranked by (squared distance, id);
 * dist_dev / idx_dev are nq x k row-major.  sorted=0 allows any order inside a row. */
ckd_status ckd_knn(const ckd_tree* tree, const double* q_dev, int64_t nq, int k, int sorted,
                   double* dist_dev, int64_t* idx_dev, void* stream);

/* The two stages of ckd_knn, for callers that reuse a query order or time the
 * search kernel alone.  No reference counterpart (the reference has no query
 * ordering).  ckd_query_order writes order_dev[nq]: a permutation of 0..nq-1 that
 * groups queries by the leaf containing them.  ckd_knn_ordered runs the search in
 * that order (order_dev may be NULL for input order); results still land in the
 * queries' own rows. */
ckd_status ckd_query_order(const ckd_tree* tree, const double* q_dev, int64_t nq,
                           int32_t* order_dev, void* stream);
ckd_status ckd_knn_ordered(const ckd_tree* tree, const double* q_dev, int64_t nq,
                           const int32_t* order_dev, int k, int sorted, double* dist_dev,
                           int64_t* idx_dev, void* stream);

/* Number of CUDA kernels this library has launched in this process. */
int64_t ckd_launch_count(void);

/* Process-wide kNN kernel choice (no reference counterpart): 0 = automatic (8
 * when k <= 64, the coordinates allow the FP32 screen and the tree is shallow
 * enough; 1 otherwise), 1 = FP64 packet
 * traversal, 7 = per-lane traversal with 8-byte heap entries (FP32 key +
 * position, exact tie resolution), 8 = 7 expanding nodes from child-pair records.
 * Every variant returns the same exact result. */
ckd_status ckd_set_knn_variant(int variant);

/* Process-wide launch tuning of the search kernels (no reference counterpart;
 * set by the autotuner).  key 0: kNN variant (as ckd_set_knn_variant);
 * key 1: cap on resident blocks per SM for the per-lane kNN kernel (0 = as many
 * as fit); key 2: warps per block of the per-lane kNN kernel (1..8, default 2,
 * at most 4 used); key 4: search kernel of ckd_knn_learned (0 = bounded per-lane
 * traversal; 3 = 0 with child-pair-record descent, default); key 6: ordering of queries by leaf before kNN and ball
 * searches (0 = automatic, default; 1 = always; 2 = never); key 7: inference of
 * the learned-bound network (0 = FP32 FMAs; 1 = tensor cores, tcgen05 MMAs on
 * BF16 activations, default); key 8: box search of up to 32768 boxes per call
 * on one tree, and of any number on a forest (1 = a warp per box, frontier
 * expanded a level at a time, default; 0 = a lane per box); key 9: cap in MiB on the device memory the library's pool hands out
 * at any time on the current device (0 = none, default): an allocation past it
 * fails with CKD_ERR_OOM and the call returns everything it had taken; key 10:
 * how long (ms, default 20000) an idle CTA of the persistent forest launch waits
 * for work before it gives up with CKD_ERR_TIMEOUT; key 11: number of first work
 * items the host withholds from the persistent forest launch while counting them
 * as pending (default 0; a test of the bounded wait: the launch cannot finish
 * and ends with CKD_ERR_TIMEOUT). */
ckd_status ckd_set_tuning(int key, int value);

/* Bytes of the current device's library pool in use by live allocations (trees,
 * networks, a running call's scratch) and reserved from the driver (no reference
 * counterpart; used to check that failed calls return their scratch). */
ckd_status ckd_pool_usage(int64_t* used, int64_t* reserved);

/* Traversal statistics of the kNN kernels (diagnostics, no reference
 * counterpart).  Copies the counters accumulated since the previous call into
 * out8 (if not NULL), clears them, and turns collection on (enable=1) or off.
 * Per-lane kernels: [0] node expansions, [2] leaf visits, [3] points screened,
 * [5] screen passes (FP64 evaluations), [6] heap inserts (all summed over queries);
 * [4] and [7]: 32 x the largest leaf-visit and node-expansion counts of each
 * warp's lanes, summed over warps (against [2] and [0] they show how long lanes
 * wait for the slowest query of their warp).  Synchronises the device. */
ckd_status ckd_knn_stats(int enable, int64_t* out8);

/* Kernel timing (diagnostics, no reference counterpart).  With enable=1 the kNN
 * entry points record CUDA events around their main search kernel on the
 * caller's stream; ckd_kernel_ms waits for the last recorded pair and returns
 * its elapsed milliseconds (or -1 if none was recorded). */
ckd_status ckd_set_kernel_timing(int enable);
ckd_status ckd_kernel_ms(float* ms);

/* ckd_knn without any device allocation.  No counterpart in the reference: it
 * serves callers that cannot allocate device memory while searching -- a host
 * application that reserves all device memory up front and lets nothing reach
 * the CUDA allocator later, or a latency-critical loop that cannot pay for the
 * implicit synchronisation of an allocation.  Same arguments and exact result as
 * ckd_knn; the search's scratch (query keys, processing order, a histogram of
 * coarse leaf bins) lives in one fixed device array of about 18 MB that every
 * device loading the library holds until exit.  Limits: nq <= 2097152 per call,
 * k <= 64, tree depth < 92; larger requests fail with CKD_ERR_BAD_ARG.  All calls
 * share the array, so calls that overlap on the GPU (other streams or threads)
 * race and must be serialised by the caller.  The first call on a device looks
 * up the array's address (cudaGetSymbolAddress); make it before any stream
 * capture.  The lookup is repeated when the device's current context has changed
 * since (after cudaDeviceReset, or under a context the caller made current), so
 * the first call after such a change should also come before any capture. */
ckd_status ckd_knn_noalloc(const ckd_tree* tree, const double* q_dev, int64_t nq, int k,
                           int sorted, double* dist_dev, int64_t* idx_dev, void* stream);

/* kNN with a k per query in one call (k_dev[nq], each in 1..kmax; no reference
 * counterpart: the reference takes one k per call, src/cosmokdtree.f90:504-540).
 * Outputs are (nq, kmax) row-major; slots past a query's own k hold id -2 and
 * distance sqrt(HUGE(0.0)) = 1.8446743523953730e19, the k > n marker.  Queries
 * are grouped by k on the device and each group takes the ckd_knn path, so rows
 * equal ckd_knn's for their k.  Reads the k histogram back (synchronises). */
ckd_status ckd_knn_multi_k(const ckd_tree* tree, const double* q_dev, int64_t nq,
                           const int32_t* k_dev, int kmax, int sorted, double* dist_dev,
                           int64_t* idx_dev, void* stream);

/* ckd_knn on host buffers (copies in, computes, copies out; synchronous).  From
 * 2^20 queries on, the search runs in 16 row chunks while a second stream copies
 * each finished chunk back.  Pinned output buffers receive the copies directly;
 * pageable ones are filled from a ring of pinned 32 MB slots that the library
 * keeps between calls (released by ckd_release_cached_memory) by up to 16 host
 * threads, while later pieces are in flight. */
ckd_status ckd_knn_host(const ckd_tree* tree, const double* q_host, int64_t nq, int k, int sorted,
                        double* dist_host, int64_t* idx_host, void* stream);

/* Ball search, two-phase CSR protocol.  Replaces pyball_search_call_1/2
 * (src/cosmokdtree2py.f90:153-246) / ball_search (src/cosmokdtree.f90:1015-1212).
 * Phase 1 writes counts_dev[nq] = number of points with d^2 <= radius^2.
 * The caller builds offsets_dev[nq+1] (exclusive prefix; ckd_exclusive_scan helps)
 * and allocates idx/dist of offsets[nq] entries; phase 2 fills them.  sorted=1
 * orders each row by (squared distance, id); sorted=0 keeps traversal order. */
ckd_status ckd_ball_count(const ckd_tree* tree, const double* q_dev, int64_t nq, double radius,
                          int64_t* counts_dev, void* stream);
ckd_status ckd_ball_fill(const ckd_tree* tree, const double* q_dev, int64_t nq, double radius,
                         int sorted, const int64_t* offsets_dev, int64_t* idx_dev,
                         double* dist_dev, void* stream);

/* Box search, two-phase CSR protocol.  Boxes are nb x 2d row-major
 * [lo0, hi0, lo1, hi1, ...].  Replaces pybox_search_call_1/2
 * (src/cosmokdtree2py.f90:252-315) / box_search (src/cosmokdtree.f90:1220-1328),
 * batched over nb boxes.  Descent and inclusion rules are the reference's. */
ckd_status ckd_box_count(const ckd_tree* tree, const double* boxes_dev, int64_t nb,
                         int64_t* counts_dev, void* stream);
ckd_status ckd_box_fill(const ckd_tree* tree, const double* boxes_dev, int64_t nb,
                        const int64_t* offsets_dev, int64_t* idx_dev, void* stream);

/* The same two-phase protocols on host buffers, for callers without device
 * memory of their own (the Fortran module cosmokdtree_gpu, C, other FFIs); the
 * shape of pyball_search_call_1/2 and pybox_search_call_1/2
 * (src/cosmokdtree2py.f90:153-315) with caller-owned rows.  Phase 1 writes the
 * CSR offsets (offsets_host[n+1], n = nq or nb); the caller allocates
 * offsets_host[n] results; phase 2 fills them.  Ids are 0-based.  Synchronous. */
ckd_status ckd_ball_count_host(const ckd_tree* tree, const double* q_host, int64_t nq,
                               double radius, int64_t* offsets_host, void* stream);
ckd_status ckd_ball_fill_host(const ckd_tree* tree, const double* q_host, int64_t nq,
                              double radius, int sorted, const int64_t* offsets_host,
                              int64_t* idx_host, double* dist_host, void* stream);
ckd_status ckd_box_count_host(const ckd_tree* tree, const double* boxes_host, int64_t nb,
                              int64_t* offsets_host, void* stream);
ckd_status ckd_box_fill_host(const ckd_tree* tree, const double* boxes_host, int64_t nb,
                             const int64_t* offsets_host, int64_t* idx_host, void* stream);

/* ---------------------------------------------------------------------------
 * Forests: many independent trees of uneven sizes built and searched together
 * (halo / subvolume catalogues).  No single-call counterpart in the reference,
 * which builds one tree per call (src/cosmokdtree.f90:124-238) and keeps the box
 * side in a module global (src/cosmokdtree.f90:87), so each tree here is
 * exactly the tree ckd_build would make from its points.
 *
 * Tree t owns rows offsets[t] .. offsets[t+1]-1 of pts (host array of n_trees+1
 * entries, offsets[0] = 0, every tree non-empty); all trees share d, leaf and
 * boxsize.  The result is a ckd_tree handle holding all trees; single-tree
 * entry points reject it.  Ids in results are local to their tree (0-based). */
ckd_status ckd_forest_build(const void* pts, const int64_t* offsets_host, int64_t n_trees, int d,
                            int dtype, int leaf, const double* boxsize, int pts_on_device,
                            void* stream, ckd_tree** out);
/* Number of trees and (if not NULL) their host offsets (n_trees + 1 entries). */
ckd_status ckd_forest_info(const ckd_tree* forest, int64_t* n_trees, int64_t* offsets_host);
/* kNN of queries grouped by tree: queries q_offsets_dev[t] .. q_offsets_dev[t+1]-1
 * (device array, n_trees + 1 entries) search tree t.  Results as ckd_knn, rows in
 * query order.  All trees' queries go through one ordering pass and one search
 * launch; no host synchronisation, so the call can be captured in a CUDA graph
 * (after a first uncaptured call has set the kernel attributes).  Needs k <= 64. */
ckd_status ckd_forest_knn(const ckd_tree* forest, const double* q_dev, const int64_t* q_offsets_dev,
                          int64_t nq, int k, int sorted, double* dist_dev, int64_t* idx_dev,
                          void* stream);
/* One persistent launch that builds a whole forest and answers its kNN queries
 * (no reference counterpart: the reference builds one tree per call and searches
 * it query by query, src/cosmokdtree.f90:124-238 and :504-540).  Every CTA of a
 * resident grid takes items from a device work queue: (tree, level) items split
 * the tree's open nodes of that level (the sliding-midpoint rule of
 * src/cosmokdtree.f90:347-410, the same trees as ckd_forest_build), and once a
 * tree is complete its (tree, query block) items search it (exact kNN, k <= 64,
 * rows in query order).  Idle CTAs poll the queue with a bounded wait
 * (ckd_set_tuning key 10); running past it ends the launch with CKD_ERR_TIMEOUT.
 *
 * ckd_forest_plan_create allocates everything once (cudaMalloc; points and
 * queries stay the caller's device arrays, read at every run; offsets on the
 * host; node_factor <= 0 sizes the node arrays for 0.45 nodes per point;
 * queries_per_block 32..2^20, e.g. 128).  ckd_forest_plan_run enqueues the
 * launch without allocating or synchronising, so it can be captured in a CUDA
 * graph (a first uncaptured run sets the kernel attributes).
 * ckd_forest_plan_status synchronises the stream and returns the launch's
 * status (CKD_ERR_OOM: node capacity exceeded, recreate with a larger factor;
 * CKD_ERR_DEPTH: a tree deeper than 126 levels; CKD_ERR_TIMEOUT); after a
 * successful status, ckd_forest_plan_forest gives the built forest (owned by the
 * plan, valid until the next run or ckd_forest_plan_free; never pass it to
 * ckd_free) for the box and ball searches. */
typedef struct ckd_forest_plan ckd_forest_plan;
ckd_status ckd_forest_plan_create(const double* pts_dev, const int64_t* offsets_host,
                                  int64_t n_trees, int d, int leaf, const double* boxsize,
                                  const double* q_dev, const int64_t* q_offsets_host, int64_t nq,
                                  int k, int sorted, double* dist_dev, int64_t* idx_dev,
                                  double node_factor, int queries_per_block,
                                  ckd_forest_plan** out);
ckd_status ckd_forest_plan_run(ckd_forest_plan* plan, void* stream);
ckd_status ckd_forest_plan_status(ckd_forest_plan* plan, void* stream);
ckd_status ckd_forest_plan_forest(const ckd_forest_plan* plan, const ckd_tree** forest);
ckd_status ckd_forest_plan_free(ckd_forest_plan* plan);

/* Box search over a forest, boxes grouped by tree like the kNN queries
 * (b_offsets_dev, device, n_trees + 1 entries); two-phase CSR as ckd_box_*. */
ckd_status ckd_forest_box_count(const ckd_tree* forest, const double* boxes_dev,
                                const int64_t* b_offsets_dev, int64_t nb, int64_t* counts_dev,
                                void* stream);
ckd_status ckd_forest_box_fill(const ckd_tree* forest, const double* boxes_dev,
                               const int64_t* b_offsets_dev, int64_t nb,
                               const int64_t* offsets_dev, int64_t* idx_dev, void* stream);
/* Ball search over a forest, queries grouped by tree as for ckd_forest_knn;
 * two-phase CSR as ckd_ball_* (ids local to each query's tree). */
ckd_status ckd_forest_ball_count(const ckd_tree* forest, const double* q_dev,
                                 const int64_t* q_offsets_dev, int64_t nq, double radius,
                                 int64_t* counts_dev, void* stream);
ckd_status ckd_forest_ball_fill(const ckd_tree* forest, const double* q_dev,
                                const int64_t* q_offsets_dev, int64_t nq, double radius,
                                int sorted, const int64_t* offsets_dev, int64_t* idx_dev,
                                double* dist_dev, void* stream);

/* Save a built tree or forest to a file / load it onto the current device (no
 * counterpart in the reference, which rebuilds on every run).  The file is a raw
 * copy of the handle's arrays, so a loaded tree gives bit-identical results.
 * Synchronous. */
ckd_status ckd_tree_save(const ckd_tree* tree, const char* path);
ckd_status ckd_tree_load(const char* path, ckd_tree** out);

/* out_dev[0] = 0, out_dev[i+1] = in_dev[0] + ... + in_dev[i]  (n+1 outputs). */
ckd_status ckd_exclusive_scan(const int64_t* in_dev, int64_t* out_dev, int64_t n, void* stream);

/* ---------------------------------------------------------------------------
 * Learned k-th-neighbour distance bound (no counterpart in the reference; it
 * speeds up ckd_knn without changing its results).
 *
 * A 12 -> 64 -> 64 -> 1 ReLU network (BF16 weights, FP32 arithmetic) predicts
 * y = log2(distance to the k-th neighbour) of a query from features of its leaf
 * and ancestors (ckd_mlp_features).  ckd_knn_learned seeds each query's heap with
 * the bound r = 2^(y + margin): the traversal prunes from the root, and every
 * query with fewer than k points within r is searched again without a bound, so
 * the result is exactly ckd_knn's.  The parameter vector is FP32, layout
 * W1[64][12], b1[64], W2[64][64], b2[64], W3[64], b3 (CKD_MLP_PARAMS floats);
 * the normalisation vector holds the feature means[12], 1/sigma[12], and the
 * target mean and sigma (CKD_MLP_NORM floats). */
#define CKD_MLP_FEATURES 12
#define CKD_MLP_HIDDEN 64
#define CKD_MLP_PARAMS 5057
#define CKD_MLP_NORM 26
typedef struct ckd_mlp ckd_mlp;

/* New network on the current device, weights initialised from `seed`. */
ckd_status ckd_mlp_create(uint64_t seed, ckd_mlp** out);
ckd_status ckd_mlp_free(ckd_mlp* net);
/* Host copies of the FP32 weights / normalisation / margin / Adam step count;
 * any output may be NULL.  Synchronous. */
ckd_status ckd_mlp_get(const ckd_mlp* net, float* params_host, float* norm_host, float* margin,
                       int64_t* steps);
/* Replace weights (resets Adam) and/or normalisation (either may be NULL) and set
 * the margin (log2 units added to every prediction).  Synchronous. */
ckd_status ckd_mlp_set(ckd_mlp* net, const float* params_host, const float* norm_host,
                       float margin);
/* feat_dev[nq][12] = features of each query for neighbour count k. */
ckd_status ckd_mlp_features(const ckd_tree* tree, const double* q_dev, int64_t nq, int k,
                            float* feat_dev, void* stream);
/* Gradient (grad_host[CKD_MLP_PARAMS]) and value (*loss) of the mean squared error
 * (1/n) sum (z - (t - t_mean) / t_sigma)^2 of the normalised output z over n
 * samples, at the current BF16 weights.  The first use of an untrained network
 * sets the normalisation from these samples.  Synchronous. */
ckd_status ckd_mlp_grad(ckd_mlp* net, const float* feat_dev, const float* target_dev, int64_t n,
                        float* grad_host, float* loss, void* stream);
/* `epochs` passes of Adam (lr, betas 0.9/0.999, eps 1e-8) over the samples in the
 * given order, `batch` samples per step; loss_host[e] (may be NULL) receives the
 * mean loss of epoch e.  Targets are log2 of exact k-th-neighbour distances.
 * Synchronous. */
ckd_status ckd_mlp_train(ckd_mlp* net, const float* feat_dev, const float* target_dev, int64_t n,
                         int batch, int epochs, float lr, float* loss_host, void* stream);
/* y_dev[n] = predicted log2 k-th distance (margin not added). */
ckd_status ckd_mlp_predict(const ckd_mlp* net, const float* feat_dev, int64_t n, float* y_dev,
                           void* stream);
/* ckd_knn with the learned bound.  Same results as ckd_knn; *n_fallback (may be
 * NULL) receives the number of queries that needed the unbounded rerun (all of
 * them when the bounded kernel does not apply: k > 64 or a very deep tree).
 * Synchronises `stream` once to read that count. */
ckd_status ckd_knn_learned(const ckd_tree* tree, const ckd_mlp* net, const double* q_dev,
                           int64_t nq, int k, int sorted, double* dist_dev, int64_t* idx_dev,
                           int64_t* n_fallback, void* stream);

/* ckd_knn_multi_k with the learned bound: the queries are grouped by k on the
 * device as there, and each group takes the ckd_knn_learned search (no
 * reference counterpart).  Rows equal ckd_knn_multi_k's; *n_fallback is the
 * total number of queries that reran without the bound.  Reads the k histogram
 * and each group's rerun count back (synchronises). */
ckd_status ckd_knn_learned_multi_k(const ckd_tree* tree, const ckd_mlp* net, const double* q_dev,
                                   int64_t nq, const int32_t* k_dev, int kmax, int sorted,
                                   double* dist_dev, int64_t* idx_dev, int64_t* n_fallback,
                                   void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CKD_H_ */
