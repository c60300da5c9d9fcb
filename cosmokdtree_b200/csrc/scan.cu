// scan.cu -- device-wide exclusive prefix sums (reduce, scan partials, downsweep).
// Used for CSR offsets (ball / box results), the build's per-level partition
// ranks and the query bucket order.
#include "ckd_common.cuh"
#include "ckd_scan.cuh"

namespace ckd {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

template <typename Tin, typename Tacc>
__global__ void __launch_bounds__(kThreads) k_tile_reduce(const Tin* __restrict__ in, int64_t n,
                                                          Tacc* __restrict__ partial) {
  int64_t base = (int64_t)blockIdx.x * kTile;
  Tacc s = 0;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    int64_t j = base + (int64_t)i * kThreads + threadIdx.x;
    if (j < n) s += (Tacc)in[j];
  }
  __shared__ Tacc red[kThreads / 32];
  Tacc tot = block_sum<Tacc, kThreads>(s, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// out[j] = offset + exclusive prefix; the last tile also writes out[n] = total.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kThreads) k_tile_scan(const Tin* __restrict__ in, int64_t n,
                                                        const Tout* __restrict__ offs,
                                                        Tout* __restrict__ out) {
  int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
  Tout v[kItems];
  Tout run = 0;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    int64_t j = base + i;
    Tout x = j < n ? (Tout)in[j] : (Tout)0;
    v[i] = run;
    run += x;
  }
  __shared__ Tout tmp[kThreads / 32];
  Tout tot;
  Tout pre = block_exclusive_scan<Tout, kThreads>(run, tmp, tot);
  Tout off = offs ? offs[blockIdx.x] : (Tout)0;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    int64_t j = base + i;
    if (j < n) out[j] = off + pre + v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = off + tot;
}

template <typename Tin, typename Tout>
ckd_status scan_impl(const Tin* in, Tout* out, int64_t n, cudaStream_t s) {
  if (n <= 0) {
    CKD_CUDA(cudaMemsetAsync(out, 0, sizeof(Tout), s));
    return CKD_OK;
  }
  int64_t tiles = cdiv(n, kTile);
  if (tiles == 1) {
    k_tile_scan<Tin, Tout><<<1, kThreads, 0, s>>>(in, n, (const Tout*)nullptr, out);
    CKD_LAUNCH_CHECK();
    return CKD_OK;
  }
  Scratch sc(s);
  Tout* part = nullptr;
  Tout* poff = nullptr;
  CKD_CUDA(sc.alloc(&part, sizeof(Tout) * tiles));
  CKD_CUDA(sc.alloc(&poff, sizeof(Tout) * (tiles + 1)));
  k_tile_reduce<Tin, Tout><<<(unsigned)tiles, kThreads, 0, s>>>(in, n, part);
  CKD_LAUNCH_CHECK();
  CKD_TRY((scan_impl<Tout, Tout>(part, poff, tiles, s)));
  k_tile_scan<Tin, Tout><<<(unsigned)tiles, kThreads, 0, s>>>(in, n, poff, out);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

// owner[i] = the t with off[t] <= i < off[t+1] (CSR rows -> row index)
__global__ void k_csr_owner(const int64_t* __restrict__ off, int32_t n_rows, int64_t n_items,
                            int32_t* __restrict__ owner) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_items) return;
  int32_t lo = 0, hi = n_rows - 1;
  while (lo < hi) {
    int32_t mid = (lo + hi + 1) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  owner[i] = lo;
}

}  // namespace

ckd_status scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, cudaStream_t s) {
  return scan_impl<int32_t, int64_t>(in, out, n, s);
}
ckd_status scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
  return scan_impl<int64_t, int64_t>(in, out, n, s);
}
ckd_status scan_i32(const int32_t* in, int32_t* out, int64_t n, cudaStream_t s) {
  return scan_impl<int32_t, int32_t>(in, out, n, s);
}

ckd_status csr_owner(const int64_t* off_dev, int32_t n_rows, int64_t n_items, int32_t* owner,
                      cudaStream_t s) {
  if (n_items <= 0) return CKD_OK;
  k_csr_owner<<<(unsigned)cdiv(n_items, 256), 256, 0, s>>>(off_dev, n_rows, n_items, owner);
  CKD_LAUNCH_CHECK();
  return CKD_OK;
}

}  // namespace ckd
