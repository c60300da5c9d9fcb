// host_pipe.cu -- kNN on host buffers in row chunks (ckd_knn_host from 2^20 queries on).
//
// The search runs chunk by chunk on the caller's stream while a second stream
// copies each finished chunk back, two device result buffers in flight.  Output
// buffers that are pinned (page-locked) receive the copies directly.  Pageable
// ones cannot be the target of an asynchronous copy: the chunk is copied in
// 32 MB pieces into a ring of six pinned slots owned by the library, and host
// threads (up to 16) move each landed piece into the caller's arrays while the
// next pieces cross PCIe and the next chunk is searched.  Each chunk's queries are
// uploaded just before its search, so the upload overlaps the previous chunk.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "ckd_common.cuh"

namespace ckd {

ckd_status knn_run(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted, double* dist,
                   int64_t* idx, cudaStream_t s);

namespace {

constexpr int kChunks = 16;
constexpr int kSlots = 6;
constexpr size_t kSlotBytes = size_t(32) << 20;

// The pinned slot ring, kept between calls (one pageable call at a time uses it).
std::mutex g_stage_mu;
unsigned char* g_stage = nullptr;

// Host threads that copy one piece (two arrays) together: the calling thread takes
// share 0, worker w share w; copy() returns when every share is done.
class CopyPool {
 public:
  explicit CopyPool(int n) : n_(std::max(1, n)) {
    for (int w = 1; w < n_; ++w) th_.emplace_back([this, w] { work(w); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      quit_ = true;
    }
    go_.notify_all();
    for (auto& t : th_) t.join();
  }
  void copy(char* d0, const char* s0, size_t b0, char* d1, const char* s1, size_t b1) {
    {
      std::lock_guard<std::mutex> g(mu_);
      dst_[0] = d0, src_[0] = s0, bytes_[0] = b0;
      dst_[1] = d1, src_[1] = s1, bytes_[1] = b1;
      done_ = 0;
      ++gen_;
    }
    go_.notify_all();
    share(0);
    std::unique_lock<std::mutex> g(mu_);
    fin_.wait(g, [this] { return done_ == n_ - 1; });
  }

 private:
  void share(int w) {
    for (int a = 0; a < 2; ++a) {
      const size_t part = (bytes_[a] + n_ - 1) / n_;
      const size_t lo = std::min(bytes_[a], part * w), hi = std::min(bytes_[a], lo + part);
      if (hi > lo) std::memcpy(dst_[a] + lo, src_[a] + lo, hi - lo);
    }
  }
  void work(int w) {
    unsigned seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> g(mu_);
        go_.wait(g, [&] { return quit_ || gen_ != seen; });
        if (quit_) return;
        seen = gen_;
      }
      share(w);
      {
        std::lock_guard<std::mutex> g(mu_);
        ++done_;
      }
      fin_.notify_one();
    }
  }
  int n_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable go_, fin_;
  unsigned gen_ = 0;
  int done_ = 0;
  bool quit_ = false;
  char* dst_[2] = {nullptr, nullptr};
  const char* src_[2] = {nullptr, nullptr};
  size_t bytes_[2] = {0, 0};
};

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

void release_host_staging() {
  std::lock_guard<std::mutex> g(g_stage_mu);
  if (g_stage) cudaFreeHost(g_stage);
  g_stage = nullptr;
}

ckd_status knn_host_pipelined(const ckd_tree* t, const double* q, int64_t nq, int k, int sorted,
                              double* dist, int64_t* idx, cudaStream_t s) {
  const int64_t rows = cdiv(nq, (int64_t)kChunks);
  const int d = t->d;
  bool direct = is_pinned(dist) && is_pinned(idx);
  // pageable outputs go through the pinned slot ring, held for the whole call; if
  // no pinned memory can be had, the copies go straight to the pageable buffers
  // (each then returns when done)
  std::unique_lock<std::mutex> stage_lock(g_stage_mu, std::defer_lock);
  if (!direct) {
    stage_lock.lock();
    if (!g_stage && cudaHostAlloc((void**)&g_stage, kSlotBytes * kSlots, cudaHostAllocDefault) !=
                        cudaSuccess) {
      cudaGetLastError();
      g_stage = nullptr;
      stage_lock.unlock();
      direct = true;
    }
  }
  double *dq = nullptr, *dd[2] = {nullptr, nullptr};
  int64_t* di[2] = {nullptr, nullptr};
  cudaStream_t s2 = nullptr;
  cudaEvent_t ev[4 + kSlots] = {};
  // every exit waits for both streams before the buffers go
  struct Cleanup {
    cudaStream_t s;
    cudaStream_t* s2;
    double** dq;
    double** dd;
    int64_t** di;
    cudaEvent_t* ev;
    ~Cleanup() {
      if (*s2) cudaStreamSynchronize(*s2);
      cudaStreamSynchronize(s);
      dev_free(*dq, s);
      for (int b = 0; b < 2; ++b) {
        dev_free(dd[b], s);
        dev_free(di[b], s);
      }
      for (int e = 0; e < 4 + kSlots; ++e)
        if (ev[e]) cudaEventDestroy(ev[e]);
      if (*s2) cudaStreamDestroy(*s2);
    }
  } cleanup{s, &s2, &dq, dd, di, ev};
  CKD_CUDA(dev_alloc((void**)&dq, sizeof(double) * nq * d, s));
  for (int b = 0; b < 2; ++b) {
    CKD_CUDA(dev_alloc((void**)&dd[b], sizeof(double) * rows * k, s));
    CKD_CUDA(dev_alloc((void**)&di[b], sizeof(int64_t) * rows * k, s));
  }
  CKD_CUDA(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
  for (int e = 0; e < 4 + kSlots; ++e)
    CKD_CUDA(cudaEventCreateWithFlags(&ev[e], cudaEventDisableTiming));
  cudaEvent_t* searched = ev;      // [2]: chunk searched into buffer b
  cudaEvent_t* copied = ev + 2;    // [2]: buffer b copied out
  cudaEvent_t* landed = ev + 4;    // [kSlots]: a piece landed in its pinned slot
  const int64_t nc = cdiv(nq, rows);
  auto search = [&](int64_t c) -> ckd_status {  // upload chunk c's queries, search them
    const int b = (int)(c & 1);
    const int64_t r0 = c * rows, n = std::min(rows, nq - r0);
    CKD_CUDA(cudaMemcpyAsync(dq + r0 * d, q + r0 * d, sizeof(double) * n * d,
                             cudaMemcpyHostToDevice, s));
    if (c >= 2) CKD_CUDA(cudaStreamWaitEvent(s, copied[b], 0));  // buffer b copied out
    CKD_TRY(knn_run(t, dq + r0 * d, n, k, sorted, dd[b], di[b], s));
    CKD_CUDA(cudaEventRecord(searched[b], s));
    return CKD_OK;
  };
  if (direct) {
    CKD_TRY(search(0));
    for (int64_t c = 0; c < nc; ++c) {
      const int b = (int)(c & 1);
      const int64_t r0 = c * rows, n = std::min(rows, nq - r0);
      if (c + 1 < nc) CKD_TRY(search(c + 1));
      CKD_CUDA(cudaStreamWaitEvent(s2, searched[b], 0));
      CKD_CUDA(cudaMemcpyAsync(dist + r0 * k, dd[b], sizeof(double) * n * k,
                               cudaMemcpyDeviceToHost, s2));
      CKD_CUDA(cudaMemcpyAsync(idx + r0 * k, di[b], sizeof(int64_t) * n * k,
                               cudaMemcpyDeviceToHost, s2));
      CKD_CUDA(cudaEventRecord(copied[b], s2));
    }
    CKD_CUDA(cudaStreamSynchronize(s2));
    CKD_CUDA(cudaStreamSynchronize(s));
    return CKD_OK;
  }
  // pageable outputs: pieces of `prow` rows through the pinned slot ring
  const int64_t prow = std::max<int64_t>(1, (int64_t)(kSlotBytes / (16 * (size_t)k)));
  struct Piece {
    int64_t c, r0, n;  // chunk, first row, rows
  };
  std::vector<Piece> pieces;
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t c0 = c * rows, c1 = std::min(nq, c0 + rows);
    for (int64_t r = c0; r < c1; r += prow) pieces.push_back({c, r, std::min(prow, c1 - r)});
  }
  const int64_t np = (int64_t)pieces.size();
  auto slot_dist = [&](int64_t p) {
    return reinterpret_cast<double*>(g_stage + (size_t)(p % kSlots) * kSlotBytes);
  };
  auto slot_idx = [&](int64_t p) {
    return reinterpret_cast<int64_t*>(g_stage + (size_t)(p % kSlots) * kSlotBytes +
                                      (size_t)prow * k * sizeof(double));
  };
  int64_t next_search = 0, issued = 0;
  auto issue = [&](int64_t p) -> ckd_status {  // copy piece p into its slot (stream s2)
    const Piece& pc = pieces[p];
    const int b = (int)(pc.c & 1);
    while (next_search <= pc.c + 1 && next_search < nc) CKD_TRY(search(next_search++));
    if (pc.r0 == pc.c * rows) CKD_CUDA(cudaStreamWaitEvent(s2, searched[b], 0));
    const int64_t off = (pc.r0 - pc.c * rows) * k;
    CKD_CUDA(cudaMemcpyAsync(slot_dist(p), dd[b] + off, sizeof(double) * pc.n * k,
                             cudaMemcpyDeviceToHost, s2));
    CKD_CUDA(cudaMemcpyAsync(slot_idx(p), di[b] + off, sizeof(int64_t) * pc.n * k,
                             cudaMemcpyDeviceToHost, s2));
    CKD_CUDA(cudaEventRecord(landed[p % kSlots], s2));
    const bool last = p + 1 == np || pieces[p + 1].c != pc.c;
    if (last) CKD_CUDA(cudaEventRecord(copied[b], s2));
    return CKD_OK;
  };
  CopyPool pool((int)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency())));
  for (int64_t p = 0; p < np; ++p) {
    while (issued < np && issued < p + kSlots) CKD_TRY(issue(issued++));
    CKD_CUDA(cudaEventSynchronize(landed[p % kSlots]));
    const Piece& pc = pieces[p];
    pool.copy(reinterpret_cast<char*>(dist + pc.r0 * k),
              reinterpret_cast<const char*>(slot_dist(p)), sizeof(double) * pc.n * k,
              reinterpret_cast<char*>(idx + pc.r0 * k), reinterpret_cast<const char*>(slot_idx(p)),
              sizeof(int64_t) * pc.n * k);
  }
  CKD_CUDA(cudaStreamSynchronize(s2));
  CKD_CUDA(cudaStreamSynchronize(s));
  return CKD_OK;
}

}  // namespace ckd
