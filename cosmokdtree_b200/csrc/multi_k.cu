// multi_k.cu -- kNN with a k per query in one call.
//
// The reference takes one k per call (src/cosmokdtree.f90:504-540); catalogues
// that mix k (per-object neighbour counts) call it once per k.  Here the
// queries are grouped by k on the device (histogram over k, counting sort), each
// group is gathered into a contiguous block and searched by the ordinary kNN path
// with its own k, and the rows are scattered back into an (nq, kmax) output.
// Slots past a query's own k hold the missing-neighbour marker (id -2, distance
// sqrt(HUGE(0.0))), like slots past n when k > n.
#include <vector>

#include "ckd_common.cuh"
#include "ckd_mlp.cuh"

namespace ckd {

ckd_status knn_run(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted, double* dist,
                   int64_t* idx, cudaStream_t s);

namespace {

__global__ void k_k_hist(const int32_t* __restrict__ kq, int64_t nq, int kmax,
                         int32_t* __restrict__ hist, int32_t* __restrict__ bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const int32_t k = kq[i];
  if (k < 1 || k > kmax) {
    atomicExch(bad, 1);
    return;
  }
  atomicAdd(&hist[k], 1);
}

// counting sort of query indices by k (order inside a group is the atomics'
// order; every row's result depends only on its own query, so it does not matter)
__global__ void k_k_scatter(const int32_t* __restrict__ kq, int64_t nq,
                            const int32_t* __restrict__ off, int32_t* __restrict__ fill,
                            int32_t* __restrict__ grp) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  const int32_t k = kq[i];
  const int32_t slot = off[k] + atomicAdd(&fill[k], 1);
  grp[slot] = (int32_t)i;
}

template <int D>
__global__ void k_gather_q(const double* __restrict__ q, const int32_t* __restrict__ rows,
                           int64_t n, double* __restrict__ qg) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t r = rows[i];
#pragma unroll
  for (int j = 0; j < D; ++j) qg[i * D + j] = q[r * D + j];
}

// rows of one group (width k) into the (nq, kmax) output, padding the rest
__global__ void k_scatter_rows(const double* __restrict__ dg, const int64_t* __restrict__ ig,
                               const int32_t* __restrict__ rows, int64_t n, int k, int kmax,
                               double* __restrict__ dist, int64_t* __restrict__ idx) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * kmax) return;
  const int64_t i = e / kmax;
  const int j = (int)(e - i * kmax);
  const int64_t r = rows[i];
  if (j < k) {
    dist[r * kmax + j] = dg[i * k + j];
    idx[r * kmax + j] = ig[i * k + j];
  } else {
    dist[r * kmax + j] = sqrt((double)CKD_HUGE);
    idx[r * kmax + j] = -2;
  }
}

template <int D>
ckd_status gather_launch(const double* q, const int32_t* rows, int64_t n, double* qg,
                         cudaStream_t s) {
  k_gather_q<D><<<(unsigned)cdiv(n, 256), 256, 0, s>>>(q, rows, n, qg);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

ckd_status gather_q(int d, const double* q, const int32_t* rows, int64_t n, double* qg,
                    cudaStream_t s) {
  switch (d) {
    case 1: return gather_launch<1>(q, rows, n, qg, s);
    case 2: return gather_launch<2>(q, rows, n, qg, s);
    case 3: return gather_launch<3>(q, rows, n, qg, s);
    case 4: return gather_launch<4>(q, rows, n, qg, s);
    case 5: return gather_launch<5>(q, rows, n, qg, s);
    case 6: return gather_launch<6>(q, rows, n, qg, s);
    case 7: return gather_launch<7>(q, rows, n, qg, s);
    case 8: return gather_launch<8>(q, rows, n, qg, s);
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

}  // namespace

ckd_status knn_learned(const ckd_tree* t, const ckd_mlp* net, const double* q, int64_t nq, int k,
                       int sorted, double* dist, int64_t* idx, int64_t* nfb, cudaStream_t s);

// net != nullptr: every k group takes the learned-bound search (its reruns are
// added to *nfb_out).
ckd_status knn_multi_k(const ckd_tree* t, const double* q, int64_t nq, const int32_t* kq,
                       int kmax, int sorted, double* dist, int64_t* idx, cudaStream_t s,
                       const ckd_mlp* net, int64_t* nfb_out) {
  if (nfb_out) *nfb_out = 0;
  int32_t *hist = nullptr, *off = nullptr, *fill = nullptr, *grp = nullptr, *bad = nullptr;
  // every buffer joins the guard as soon as it exists, so a failed allocation
  // returns the earlier ones to the pool
  struct Free {
    cudaStream_t s;
    std::vector<void*> ps;
    ~Free() {
      for (void* p : ps) dev_free(p, s);
    }
  } fr{s, {}};
  auto take = [&](int32_t** p, size_t bytes) -> cudaError_t {
    const cudaError_t e = dev_alloc((void**)p, bytes, s);
    if (e == cudaSuccess) fr.ps.push_back(*p);
    return e;
  };
  CKD_CUDA(take(&hist, sizeof(int32_t) * (kmax + 1)));
  CKD_CUDA(take(&off, sizeof(int32_t) * (kmax + 2)));
  CKD_CUDA(take(&fill, sizeof(int32_t) * (kmax + 1)));
  CKD_CUDA(take(&grp, sizeof(int32_t) * nq));
  CKD_CUDA(take(&bad, sizeof(int32_t)));
  CKD_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * (kmax + 1), s));
  CKD_CUDA(cudaMemsetAsync(fill, 0, sizeof(int32_t) * (kmax + 1), s));
  CKD_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  const unsigned g = (unsigned)cdiv(nq, 256);
  k_k_hist<<<g, 256, 0, s>>>(kq, nq, kmax, hist, bad);
  CKD_LAUNCH_CHECK();
  std::vector<int32_t> h((size_t)kmax + 1);
  int32_t hbad = 0;
  CKD_CUDA(cudaMemcpyAsync(h.data(), hist, sizeof(int32_t) * (kmax + 1), cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaStreamSynchronize(s));
  if (hbad) return fail(CKD_ERR_BAD_ARG, "every k must lie in 1..kmax");
  std::vector<int32_t> ho((size_t)kmax + 2, 0);
  for (int k = 0; k <= kmax; ++k) ho[k + 1] = ho[k] + h[k];
  CKD_CUDA(cudaMemcpyAsync(off, ho.data(), sizeof(int32_t) * (kmax + 2), cudaMemcpyHostToDevice, s));
  k_k_scatter<<<g, 256, 0, s>>>(kq, nq, off, fill, grp);
  CKD_LAUNCH_CHECK();
  CKD_CUDA(cudaStreamSynchronize(s));  // `ho` is the source of a copy
  for (int k = 1; k <= kmax; ++k) {
    const int64_t n = h[k];
    if (n == 0) continue;
    const int32_t* rows = grp + ho[k];
    double *qg = nullptr, *dg = nullptr;
    int64_t* ig = nullptr;
    CKD_CUDA(dev_alloc((void**)&qg, sizeof(double) * n * t->d, s));
    fr.ps.push_back(qg);
    CKD_CUDA(dev_alloc((void**)&dg, sizeof(double) * n * k, s));
    fr.ps.push_back(dg);
    CKD_CUDA(dev_alloc((void**)&ig, sizeof(int64_t) * n * k, s));
    fr.ps.push_back(ig);
    CKD_TRY(gather_q(t->d, q, rows, n, qg, s));
    if (net) {
      int64_t nfb = 0;
      CKD_TRY(knn_learned(t, net, qg, n, k, sorted, dg, ig, &nfb, s));
      if (nfb_out) *nfb_out += nfb;
    } else {
      CKD_TRY(knn_run(t, qg, n, k, sorted, dg, ig, s));
    }
    k_scatter_rows<<<(unsigned)cdiv(n * kmax, 256), 256, 0, s>>>(dg, ig, rows, n, k, kmax, dist,
                                                                idx);
    CKD_LAUNCH_CHECK();
  }
  return CKD_OK;
}

}  // namespace ckd
