// ckd_oracle.cpp -- CPU restatement of cosmokdtree's build / kNN / ball / box path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
// baseline ("reference algorithm, C++ restatement").  Only the test-suite, the
// smoke check and bench.py's CPU-baseline leg may load it.  The product path
// (cosmokdtree_b200) never calls into it.
//
// The reference is Fortran (src/cosmokdtree.f90 + src/cosmokdtree2py.f90) and
// there is no Fortran compiler in this image, so the reference cannot be run
// here.  Parity pinning: the reference ships no golden vectors; its only result
// checks are the brute-force comparisons inside its demo programs
// (demos/cosmokdtree/periodic/tree_test.f90:79-139,
//  demos/cosmokdtree/box_search/tree_test.f90:85-97).  tests/test_oracle.py
// re-runs those checks seeded and asserted, plus a scipy cKDTree cross-check.
//
// Semantics restated (all arithmetic FP64, never contracted: build with
// -ffp-contract=off):
//   * build: sliding-midpoint rule of cosmokdtree.f90:286-451 (cell bounds,
//     longest-cell-side axis with spread tie-break, midpoint, one-point slides,
//     x < split goes left), root cell from cosmokdtree.f90:218-229.
//   * kNN: best-first queue (cosmokdtree.f90:549-675) when non-periodic,
//     hyperplane DFS (cosmokdtree.f90:782-853) when periodic.
//   * ball: bbox recursion with the fully-inside shortcut
//     (cosmokdtree.f90:1076-1139, 1332-1366) when non-periodic, hyperplane DFS
//     (cosmokdtree.f90:1143-1212) when periodic.
//   * box: cosmokdtree.f90:1258-1328 (strict descent, inclusive leaf test).
//   * distances: cosmokdtree.f90:1441-1546.
//
// Canonicalisations (documented; they only matter at exact ties, where the
// reference result depends on visiting order or on its unstable partition):
//   1. kNN / sorted ball rank by (d2, id) lexicographically, lower id first.
//   2. Partition is stable, so each segment stays sorted by original id and the
//      slide point (first minloc / maxloc) is the lowest id holding the extreme.
//   3. A periodic root cell is written on all D axes (the reference writes 3).
//   4. Hyperplane visit tests are padded by a relative 1e-12 so no candidate
//      whose FP64 distance passes the acceptance test can be skipped by
//      rounding; results equal the brute-force definition.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>
#include <omp.h>

namespace {

constexpr double kHuge = (double)FLT_MAX;  // HUGE(0.0) promoted to FP64 (cosmokdtree.f90:517)
constexpr double kPad = 1e-12;             // canonicalisation 4

struct Node {
  double split = 0.0;
  int axis = -1;
  bool leaf = false;
  int64_t start = 0, count = 0;   // range in the leaf-ordered point array
  std::vector<double> cell;       // [lo0, hi0, lo1, hi1, ...]
  std::unique_ptr<Node> left, right;
};

struct Tree {
  int64_t n = 0;
  int d = 0;
  int leaf = 16;
  bool periodic = false;
  std::vector<double> L;          // box side per axis (periodic only)
  std::vector<double> pts;        // leaf-ordered, row-major (n x d)
  std::vector<int64_t> ids;       // original 0-based index per leaf-ordered point
  // flattened preorder copy of the node graph
  std::vector<double> split;
  std::vector<int> axis;
  std::vector<int64_t> lchild, rchild, start, count;
  std::vector<unsigned char> is_leaf;
  std::vector<double> cell;       // n_nodes x 2d
  int64_t n_nodes = 0;
  int depth = 0;
};

struct BuildCtx {
  Tree* t;
  std::vector<double> tmp_pts;
  std::vector<int64_t> tmp_ids;
  int max_task_depth;
};

// cosmokdtree.f90:286-451 -- one node of the sliding-midpoint recursion.
std::unique_ptr<Node> build_rec(BuildCtx& c, int64_t s, int64_t n, const std::vector<double>& cell,
                                int depth) {
  Tree& t = *c.t;
  const int d = t.d;
  auto node = std::make_unique<Node>();
  node->cell = cell;
  node->start = s;
  node->count = n;
  if (n <= t.leaf) {  // cosmokdtree.f90:327-341
    node->leaf = true;
    return node;
  }
  double* P = &t.pts[s * d];
  int64_t* I = &t.ids[s];
  // cosmokdtree.f90:347-353: per-axis data extent and cell side
  std::vector<double> mn(d, 0.0), mx(d, 0.0), spread(d), side(d);
  for (int j = 0; j < d; ++j) {
    double a = P[j], b = P[j];
    for (int64_t i = 1; i < n; ++i) {
      double v = P[i * d + j];
      if (v < a) a = v;
      if (v > b) b = v;
    }
    mn[j] = a;
    mx[j] = b;
    side[j] = cell[2 * j + 1] - cell[2 * j];
    spread[j] = b - a;
  }
  // cosmokdtree.f90:355-365: longest cell side, ties -> larger spread
  double maxside = side[0];
  int axis = 0;
  for (int j = 1; j < d; ++j) {
    if (side[j] > maxside) {
      maxside = side[j];
      axis = j;
    }
    if (side[j] == maxside && spread[j] > spread[axis]) axis = j;
  }
  double mid = 0.5 * (cell[2 * axis] + cell[2 * axis + 1]);  // :367
  const double minx = mn[axis], maxx = mx[axis];
  // stable partition into tmp, then copy back.  mode 0: x<mid, 1: slide left, 2: slide right
  int mode = 0;
  int64_t ext = -1;  // position (within segment) of the slide point
  if (minx >= mid) {  // :376-388
    mid = minx;
    mode = 1;
    for (int64_t i = 0; i < n; ++i)
      if (P[i * d + axis] == minx) { ext = i; break; }
  } else if (maxx < mid) {  // :391-403
    mid = maxx;
    mode = 2;
    for (int64_t i = 0; i < n; ++i)
      if (P[i * d + axis] == maxx) { ext = i; break; }
  }
  double* TP = &c.tmp_pts[s * d];
  int64_t* TI = &c.tmp_ids[s];
  int64_t nl = 0;
  auto goes_left = [&](int64_t i) -> bool {
    if (mode == 0) return P[i * d + axis] < mid;  // :470
    if (mode == 1) return i == ext;
    return i != ext;
  };
  for (int64_t i = 0; i < n; ++i)
    if (goes_left(i)) {
      std::memcpy(&TP[nl * d], &P[i * d], sizeof(double) * d);
      TI[nl] = I[i];
      ++nl;
    }
  int64_t w = nl;
  for (int64_t i = 0; i < n; ++i)
    if (!goes_left(i)) {
      std::memcpy(&TP[w * d], &P[i * d], sizeof(double) * d);
      TI[w] = I[i];
      ++w;
    }
  std::memcpy(P, TP, sizeof(double) * d * n);
  std::memcpy(I, TI, sizeof(int64_t) * n);

  node->split = mid;
  node->axis = axis;
  std::vector<double> cl = cell, cr = cell;  // :419-422
  cl[2 * axis + 1] = mid;
  cr[2 * axis] = mid;
  if (depth < c.max_task_depth) {  // :424-441, task parallel top levels
    std::unique_ptr<Node> L, R;
#pragma omp task shared(L, c, cl) firstprivate(s, nl, depth)
    L = build_rec(c, s, nl, cl, depth + 1);
#pragma omp task shared(R, c, cr) firstprivate(s, nl, n, depth)
    R = build_rec(c, s + nl, n - nl, cr, depth + 1);
#pragma omp taskwait
    node->left = std::move(L);
    node->right = std::move(R);
  } else {
    node->left = build_rec(c, s, nl, cl, depth + 1);
    node->right = build_rec(c, s + nl, n - nl, cr, depth + 1);
  }
  return node;
}

void flatten(Tree& t, const Node* nd, int depth, int64_t& next) {
  // iterative preorder to survive degenerate (very deep) trees
  struct Item { const Node* n; int64_t parent; int side; int depth; };
  std::vector<Item> st;
  st.push_back({nd, -1, 0, depth});
  while (!st.empty()) {
    Item it = st.back();
    st.pop_back();
    int64_t me = next++;
    const Node* x = it.n;
    t.split.push_back(x->split);
    t.axis.push_back(x->axis);
    t.lchild.push_back(-1);
    t.rchild.push_back(-1);
    t.start.push_back(x->start);
    t.count.push_back(x->count);
    t.is_leaf.push_back(x->leaf ? 1 : 0);
    for (double v : x->cell) t.cell.push_back(v);
    if (it.parent >= 0) (it.side == 0 ? t.lchild : t.rchild)[it.parent] = me;
    if (it.depth > t.depth) t.depth = it.depth;
    if (!x->leaf) {
      st.push_back({x->right.get(), me, 1, it.depth + 1});
      st.push_back({x->left.get(), me, 0, it.depth + 1});
    }
  }
}

void free_rec_iter(std::unique_ptr<Node> root) {
  // avoid recursive destructor depth on degenerate trees
  std::vector<std::unique_ptr<Node>> st;
  st.push_back(std::move(root));
  while (!st.empty()) {
    std::unique_ptr<Node> x = std::move(st.back());
    st.pop_back();
    if (x->left) st.push_back(std::move(x->left));
    if (x->right) st.push_back(std::move(x->right));
  }
}

// ---------------------------------------------------------------- distances
// cosmokdtree.f90:1441-1465 -- squared distance, axis order, minimum image.
inline double dist2(const Tree& t, const double* p, const double* q) {
  double s = 0.0;
  for (int j = 0; j < t.d; ++j) {
    double dx = p[j] - q[j];
    if (t.periodic) {
      double a = std::fabs(dx);
      dx = std::min(a, t.L[j] - a);
    }
    s = s + dx * dx;
  }
  return s;
}

// cosmokdtree.f90:1472-1485
inline double dist1d(const Tree& t, double x1, double x2, int j) {
  double dx = x1 - x2;
  if (t.periodic) {
    double a = std::fabs(dx);
    dx = std::min(a, t.L[j] - a);
  }
  return std::fabs(dx);
}

// Cell min-distance^2.  Non-periodic: cosmokdtree.f90:1525-1546.  Periodic: the
// nearer of the two faces under the minimum image (a safe lower bound; the
// reference does not prune periodic searches with cells at all).
inline double cell_mind2(const Tree& t, const double* cell, const double* q) {
  double s = 0.0;
  for (int j = 0; j < t.d; ++j) {
    double lo = cell[2 * j], hi = cell[2 * j + 1], x = q[j], dm;
    if (x < lo || x > hi) {
      if (t.periodic)
        dm = std::min(dist1d(t, x, lo, j), dist1d(t, x, hi, j));
      else
        dm = (x < lo) ? dist1d(t, x, lo, j) : dist1d(t, x, hi, j);
    } else {
      dm = 0.0;
    }
    s = s + dm * dm;
  }
  return s;
}

// ------------------------------------------------------------- kNN heaps
struct Cand { double d2; int64_t id; };
// canonical order (d2, id); the sentinel id -1 makes (HUGE, -1) beat every real
// candidate at d2 == HUGE, mirroring the strict test of cosmokdtree.f90:658.
inline bool lt(const Cand& a, const Cand& b) { return a.d2 < b.d2 || (a.d2 == b.d2 && a.id < b.id); }

// cosmokdtree.f90:859-905 -- root replaced, sift down (max-heap, 0-based).
inline void heap_replace_root(Cand* h, int k, Cand c) {
  int i = 0;
  for (;;) {
    int l = 2 * i + 1, r = l + 1, big = i;
    Cand cur = (big == i) ? c : h[big];
    if (l < k && lt(cur, h[l])) { big = l; cur = h[l]; }
    if (r < k && lt(cur, h[r])) { big = r; cur = h[r]; }
    if (big == i) break;
    h[i] = h[big];
    i = big;
  }
  h[i] = c;
}

inline void offer(Cand* h, int k, double d2, int64_t id) {
  Cand c{d2, id};
  if (lt(c, h[0])) heap_replace_root(h, k, c);
}

// cosmokdtree.f90:549-675 -- best-first traversal with a min-heap of nodes.
void knn_queue(const Tree& t, const double* q, Cand* h, int k) {
  struct QE { double md; int64_t node; };
  auto qgt = [](const QE& a, const QE& b) { return a.md > b.md; };
  std::vector<QE> pq;
  pq.reserve(128);
  pq.push_back({cell_mind2(t, &t.cell[0], q), 0});
  while (!pq.empty()) {
    std::pop_heap(pq.begin(), pq.end(), qgt);
    QE e = pq.back();
    pq.pop_back();
    double worst = h[0].d2;
    if (e.md > worst) continue;  // :621
    int64_t nd = e.node;
    if (!t.is_leaf[nd]) {
      int64_t L = t.lchild[nd], R = t.rchild[nd];
      double ml = cell_mind2(t, &t.cell[L * 2 * t.d], q);
      double mr = cell_mind2(t, &t.cell[R * 2 * t.d], q);
      if (ml <= worst) { pq.push_back({ml, L}); std::push_heap(pq.begin(), pq.end(), qgt); }  // :634
      if (mr <= worst) { pq.push_back({mr, R}); std::push_heap(pq.begin(), pq.end(), qgt); }  // :642
    } else {
      for (int64_t i = t.start[nd]; i < t.start[nd] + t.count[nd]; ++i)  // :654-664
        offer(h, k, dist2(t, &t.pts[i * t.d], q), t.ids[i]);
    }
  }
}

// cosmokdtree.f90:782-853 -- hyperplane DFS with the periodic face tests.
void knn_hyperp(const Tree& t, int64_t nd, const double* q, Cand* h, int k) {
  if (t.is_leaf[nd]) {
    for (int64_t i = t.start[nd]; i < t.start[nd] + t.count[nd]; ++i)
      offer(h, k, dist2(t, &t.pts[i * t.d], q), t.ids[i]);
    return;
  }
  int ax = t.axis[nd];
  double d1d = q[ax] - t.split[nd];
  bool left_first = d1d < 0;
  knn_hyperp(t, left_first ? t.lchild[nd] : t.rchild[nd], q, h, k);
  double worst = h[0].d2;
  bool look = d1d * d1d <= worst * (1.0 + kPad);  // :828 (canonical: <=, padded)
  if (t.periodic && !look) {
    double half = t.L[ax] / 2.0, s = std::sqrt(worst) * (1.0 + kPad) + kPad * t.L[ax];
    if (left_first)
      look = q[ax] - s <= -half;  // :830
    else
      look = q[ax] + s >= half;   // :842
  }
  if (look) knn_hyperp(t, left_first ? t.rchild[nd] : t.lchild[nd], q, h, k);
}

void knn_one(const Tree& t, const double* q, int k, bool sorted, double* dist, int64_t* idx) {
  std::vector<Cand> h(k, Cand{kHuge, -1});  // :517-518
  if (t.periodic)
    knn_hyperp(t, 0, q, h.data(), k);
  else
    knn_queue(t, q, h.data(), k);
  if (sorted) std::sort(h.begin(), h.end(), lt);  // :529-535, canonical order
  for (int i = 0; i < k; ++i) {
    dist[i] = std::sqrt(h[i].d2);                 // :538
    idx[i] = h[i].id < 0 ? -2 : h[i].id;          // 1-based -1 then kdtree.py:52 "-= 1"
  }
}

// --------------------------------------------------------------- ball search
struct BallOut { std::vector<int64_t> ids; std::vector<double> d2; };

// cosmokdtree.f90:1332-1366
void ball_reduce(const Tree& t, int64_t nd, const double* q, BallOut& o) {
  for (int64_t i = t.start[nd]; i < t.start[nd] + t.count[nd]; ++i) {
    o.ids.push_back(t.ids[i]);
    o.d2.push_back(dist2(t, &t.pts[i * t.d], q));
  }
}

// cosmokdtree.f90:1076-1139 (non-periodic)
void ball_bbox(const Tree& t, int64_t nd, const double* q, double r, BallOut& o) {
  const double* cell = &t.cell[nd * 2 * t.d];
  double mind = 0.0, maxd = 0.0;
  for (int j = 0; j < t.d; ++j) {  // bbox_distance_1D, :1492-1516
    double lo = cell[2 * j], hi = cell[2 * j + 1], x = q[j], dmin;
    if (x < lo) dmin = dist1d(t, x, lo, j);
    else if (x > hi) dmin = dist1d(t, x, hi, j);
    else dmin = 0.0;
    double dmax = std::max(dist1d(t, x, lo, j), dist1d(t, x, hi, j));
    mind = mind + dmin * dmin;
    maxd = maxd + dmax * dmax;
  }
  double r2 = r * r;
  if (mind > r2) return;                   // :1112
  if (maxd <= r2) { ball_reduce(t, nd, q, o); return; }  // :1116-1118
  if (t.is_leaf[nd]) {
    for (int64_t i = t.start[nd]; i < t.start[nd] + t.count[nd]; ++i) {
      double d2 = dist2(t, &t.pts[i * t.d], q);
      if (d2 <= r2) { o.ids.push_back(t.ids[i]); o.d2.push_back(d2); }  // :1126
    }
    return;
  }
  ball_bbox(t, t.lchild[nd], q, r, o);
  ball_bbox(t, t.rchild[nd], q, r, o);
}

// cosmokdtree.f90:1143-1212 (periodic)
void ball_hyperp(const Tree& t, int64_t nd, const double* q, double r, BallOut& o) {
  double r2 = r * r;
  if (t.is_leaf[nd]) {
    for (int64_t i = t.start[nd]; i < t.start[nd] + t.count[nd]; ++i) {
      double d2 = dist2(t, &t.pts[i * t.d], q);
      if (d2 <= r2) { o.ids.push_back(t.ids[i]); o.d2.push_back(d2); }
    }
    return;
  }
  int ax = t.axis[nd];
  double d1d = q[ax] - t.split[nd];
  bool left_first = d1d < 0;
  ball_hyperp(t, left_first ? t.lchild[nd] : t.rchild[nd], q, r, o);
  double rp = r * (1.0 + kPad);
  bool look = std::fabs(d1d) <= rp;
  if (t.periodic && !look) {
    double half = t.L[ax] / 2.0, s = rp + kPad * t.L[ax];
    look = left_first ? (q[ax] - s <= -half) : (q[ax] + s >= half);
  }
  if (look) ball_hyperp(t, left_first ? t.rchild[nd] : t.lchild[nd], q, r, o);
}

void ball_one(const Tree& t, const double* q, double r, BallOut& o) {
  if (t.periodic)
    ball_hyperp(t, 0, q, r, o);
  else
    ball_bbox(t, 0, q, r, o);
}

// ---------------------------------------------------------------- box search
// cosmokdtree.f90:1258-1328
void box_rec(const Tree& t, int64_t nd, const double* box, std::vector<int64_t>& out) {
  if (t.is_leaf[nd]) {
    for (int64_t i = t.start[nd]; i < t.start[nd] + t.count[nd]; ++i) {
      const double* p = &t.pts[i * t.d];
      bool in = true;
      for (int j = 0; j < t.d; ++j)
        if (p[j] < box[2 * j] || p[j] > box[2 * j + 1]) { in = false; break; }  // :1319
      if (in) out.push_back(t.ids[i]);
    }
    return;
  }
  int ax = t.axis[nd];
  if (box[2 * ax] < t.split[nd]) box_rec(t, t.lchild[nd], box, out);      // :1296
  if (box[2 * ax + 1] > t.split[nd]) box_rec(t, t.rchild[nd], box, out);  // :1300
}

int set_threads(int nthreads) {
  int p = nthreads > 0 ? nthreads : omp_get_max_threads();
  return p;
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

// Returns 0 on success; 1 bad dimension / arguments; 2 point outside [-L/2, L/2].
int ora_build(const double* pts, int64_t n, int d, int leaf, const double* boxsize, int nthreads,
              void** out) {
  *out = nullptr;
  if (d < 1 || n < 1 || leaf < 1) return 1;
  auto t = new Tree();
  t->n = n;
  t->d = d;
  t->leaf = leaf;
  t->periodic = boxsize != nullptr;
  if (t->periodic) {
    t->L.assign(boxsize, boxsize + d);
    for (int j = 0; j < d; ++j)
      if (!(t->L[j] > 0)) { delete t; return 1; }
    for (int64_t i = 0; i < n; ++i)  // cosmokdtree.f90:177-190
      for (int j = 0; j < d; ++j) {
        double v = pts[i * d + j];
        if (v < -t->L[j] / 2 || v > t->L[j] / 2) { delete t; return 2; }
      }
  }
  t->pts.assign(pts, pts + n * d);
  t->ids.resize(n);
  for (int64_t i = 0; i < n; ++i) t->ids[i] = i;
  std::vector<double> cell(2 * d);
  for (int j = 0; j < d; ++j) {
    if (t->periodic) {  // :218-224 (all D axes, canonicalisation 3)
      cell[2 * j] = -t->L[j] / 2.;
      cell[2 * j + 1] = t->L[j] / 2.;
    } else {  // :226-229
      double a = pts[j], b = pts[j];
      for (int64_t i = 1; i < n; ++i) {
        a = std::min(a, pts[i * d + j]);
        b = std::max(b, pts[i * d + j]);
      }
      cell[2 * j] = a;
      cell[2 * j + 1] = b;
    }
  }
  BuildCtx c;
  c.t = t;
  c.tmp_pts.resize(n * d);
  c.tmp_ids.resize(n);
  int p = set_threads(nthreads);
  c.max_task_depth = (int)(std::log((double)p + 0.1) / std::log(2.0));  // :273-280
  std::unique_ptr<Node> root;
#pragma omp parallel num_threads(p)
  {
#pragma omp single
    root = build_rec(c, 0, n, cell, 0);
  }
  int64_t next = 0;
  flatten(*t, root.get(), 0, next);
  t->n_nodes = next;
  free_rec_iter(std::move(root));
  *out = t;
  return 0;
}

void ora_free(void* h) { delete static_cast<Tree*>(h); }

int64_t ora_n_nodes(void* h) { return static_cast<Tree*>(h)->n_nodes; }
int ora_depth(void* h) { return static_cast<Tree*>(h)->depth; }

// Preorder node export: axis (-1 for leaves), split, start, count, is_leaf,
// left/right child (preorder index, -1 for leaves), cells (n_nodes x 2d).
void ora_export(void* h, int32_t* axis, double* split, int64_t* start, int64_t* count,
                uint8_t* is_leaf, int64_t* lchild, int64_t* rchild, double* cell, int64_t* ids,
                double* pts) {
  Tree& t = *static_cast<Tree*>(h);
  for (int64_t i = 0; i < t.n_nodes; ++i) {
    if (axis) axis[i] = t.is_leaf[i] ? -1 : t.axis[i];
    if (split) split[i] = t.split[i];
    if (start) start[i] = t.start[i];
    if (count) count[i] = t.count[i];
    if (is_leaf) is_leaf[i] = t.is_leaf[i];
    if (lchild) lchild[i] = t.lchild[i];
    if (rchild) rchild[i] = t.rchild[i];
  }
  if (cell) std::memcpy(cell, t.cell.data(), sizeof(double) * t.cell.size());
  if (ids) std::memcpy(ids, t.ids.data(), sizeof(int64_t) * t.n);
  if (pts) std::memcpy(pts, t.pts.data(), sizeof(double) * t.n * t.d);
}

void ora_knn(void* h, const double* q, int64_t nq, int k, int sorted, double* dist, int64_t* idx,
             int nthreads) {
  const Tree& t = *static_cast<Tree*>(h);
  int p = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) num_threads(p)
  for (int64_t i = 0; i < nq; ++i)
    knn_one(t, &q[i * t.d], k, sorted != 0, &dist[i * k], &idx[i * k]);
}

void ora_ball_count(void* h, const double* q, int64_t nq, double r, int64_t* counts, int nthreads) {
  const Tree& t = *static_cast<Tree*>(h);
  int p = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) num_threads(p)
  for (int64_t i = 0; i < nq; ++i) {
    BallOut o;
    ball_one(t, &q[i * t.d], r, o);
    counts[i] = (int64_t)o.ids.size();
  }
}

// offsets: nq+1 exclusive prefix of the counts.
void ora_ball_fill(void* h, const double* q, int64_t nq, double r, int sorted,
                   const int64_t* offsets, int64_t* idx, double* dist, int nthreads) {
  const Tree& t = *static_cast<Tree*>(h);
  int p = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) num_threads(p)
  for (int64_t i = 0; i < nq; ++i) {
    BallOut o;
    ball_one(t, &q[i * t.d], r, o);
    size_t m = o.ids.size();
    std::vector<Cand> c(m);
    for (size_t j = 0; j < m; ++j) c[j] = Cand{o.d2[j], o.ids[j]};
    if (sorted) std::sort(c.begin(), c.end(), lt);  // :1062-1066, canonical order
    int64_t base = offsets[i];
    for (size_t j = 0; j < m; ++j) {
      idx[base + j] = c[j].id;
      dist[base + j] = std::sqrt(c[j].d2);  // :1070
    }
  }
}

void ora_box_count(void* h, const double* boxes, int64_t nb, int64_t* counts, int nthreads) {
  const Tree& t = *static_cast<Tree*>(h);
  int p = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) num_threads(p)
  for (int64_t i = 0; i < nb; ++i) {
    std::vector<int64_t> o;
    box_rec(t, 0, &boxes[i * 2 * t.d], o);
    counts[i] = (int64_t)o.size();
  }
}

void ora_box_fill(void* h, const double* boxes, int64_t nb, const int64_t* offsets, int64_t* idx,
                  int nthreads) {
  const Tree& t = *static_cast<Tree*>(h);
  int p = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) num_threads(p)
  for (int64_t i = 0; i < nb; ++i) {
    std::vector<int64_t> o;
    box_rec(t, 0, &boxes[i * 2 * t.d], o);
    std::memcpy(&idx[offsets[i]], o.data(), sizeof(int64_t) * o.size());
  }
}

// Algorithmic bytes of an exact cell-pruned kNN search of this tree (the bytes
// any such search must read, no reuse credited), given each query's exact k-th
// squared distance:  D*8 (query) + sum over leaves with cell_mind2 <= dk2 of
// n_leaf*(D*8+4) + (2*D*8+8) per node on those leaves' root paths + k*16.
// Writes the totals: out[0] bytes, out[1] leaves, out[2] nodes, out[3] points.
void ora_knn_algbytes(void* h, const double* q, int64_t nq, int k, const double* kth_d2,
                      double* out, int nthreads) {
  const Tree& t = *static_cast<Tree*>(h);
  int p = set_threads(nthreads);
  double tb = 0, tl = 0, tn = 0, tp = 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(p) reduction(+ : tb, tl, tn, tp)
  for (int64_t i = 0; i < nq; ++i) {
    const double* x = &q[i * t.d];
    double dk2 = kth_d2[i];
    std::vector<int64_t> st{0};
    double nodes = 0, leaves = 0, pts = 0;
    while (!st.empty()) {
      int64_t nd = st.back();
      st.pop_back();
      if (cell_mind2(t, &t.cell[nd * 2 * t.d], x) > dk2) continue;
      nodes += 1;
      if (t.is_leaf[nd]) {
        leaves += 1;
        pts += (double)t.count[nd];
      } else {
        st.push_back(t.rchild[nd]);
        st.push_back(t.lchild[nd]);
      }
    }
    tb += t.d * 8.0 + pts * (t.d * 8.0 + 4.0) + nodes * (2.0 * t.d * 8.0 + 8.0) + k * 16.0;
    tl += leaves;
    tn += nodes;
    tp += pts;
  }
  out[0] = tb;
  out[1] = tl;
  out[2] = tn;
  out[3] = tp;
}

}  // extern "C"
