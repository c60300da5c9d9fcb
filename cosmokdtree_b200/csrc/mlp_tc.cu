// mlp_tc.cu -- tensor-core (tcgen05) inference of the learned-bound network.
//
// One CTA of 128 threads serves tiles of 128 queries.  Thread t computes the
// standardised features of query t of the tile and stores them (BF16, K padded
// from 12 to 16 with zeros) as row t of the A operand in shared memory; one
// thread then issues
//   layer 1:  D1[128x64] = A1[128x16] . W1^T                  (1 tcgen05.mma, K = 16)
//   layer 2:  D2[128x64] = bf16(relu(D1 + b1))[128x64] . W2^T (4 tcgen05.mma, K = 16 each)
// with FP32 accumulators in tensor memory (128 lanes x 128 columns: D1 in columns
// 0-63, D2 in 64-127).  Each thread reads its own row back with tcgen05.ld (warp w
// owns TMEM lanes 32w..32w+31), applies bias and ReLU in FP32, and evaluates the
// 64-wide output layer in registers.  Completion of the MMAs is signalled through
// an mbarrier by tcgen05.commit; every wait is bounded and reports a timeout.
//
// Operands use the canonical no-swizzle K-major layout of tcgen05 shared-memory
// descriptors: 8-row x 16-byte core matrices, element (r, k) of an R-row operand
// at byte (k / 8) * R * 16 + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, so one
// K-step of 16 covers two 8-column chunks R * 16 bytes apart (leading byte
// offset) and 8-row groups are 128 bytes apart (stride byte offset).
//
// Numerics: BF16 weights and BF16 activations into the MMA, FP32 accumulation,
// FP32 bias / ReLU / output layer.  The prediction only sets a search bound, so
// results of the search do not depend on it.
#include <cuda_bf16.h>

#include <algorithm>

#include "ckd_mlp.cuh"
#include "ckd_traverse.cuh"

namespace ckd {

namespace {

constexpr int kTcRows = 128;  // queries per tile = MMA M
constexpr int kK1 = 16;       // layer-1 K (12 features padded)
// shared-memory layout (bytes)
constexpr int kOffA1 = 0;                               // 128 x 16 bf16
constexpr int kOffA2 = kOffA1 + kTcRows * kK1 * 2;      // 128 x 64 bf16
constexpr int kOffB1 = kOffA2 + kTcRows * kMlpH * 2;    // 64 x 16 bf16
constexpr int kOffB2 = kOffB1 + kMlpH * kK1 * 2;        // 64 x 64 bf16
constexpr int kOffF = kOffB2 + kMlpH * kMlpH * 2;       // b1, b2, w3 (64 each), b3
constexpr int kOffBar = kOffF + (3 * kMlpH + 4) * 4;    // mbarrier (8-byte aligned)
constexpr int kOffSlot = kOffBar + 8;                   // TMEM base address
constexpr int kTcSmem = kOffSlot + 8;
// dynamic shared memory requested per CTA: also caps residency at 3 CTAs per SM,
// so the 3 x 128 allocated TMEM columns never exceed the SM's 512
constexpr int kTcSmemRequest = 64 * 1024;
static_assert(kOffBar % 8 == 0, "mbarrier alignment");
constexpr uint32_t kTmemCols = 128;
constexpr unsigned kWaitLimit = 1u << 24;

// instruction descriptor: D F32, A/B BF16, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMlpH >> 3) << 17) |
                            ((uint32_t)(kTcRows >> 4) << 24);

__device__ __forceinline__ uint32_t core_off(int r, int k, int rows) {
  return (uint32_t)((k >> 3) * rows * 16 + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// no-swizzle K-major shared-memory descriptor (version 1) for K-step s of an
// operand with `rows` rows starting at shared address `base`
__device__ __forceinline__ uint64_t smem_desc(uint32_t base, int rows, int s) {
  const uint32_t start = base + (uint32_t)(2 * s) * rows * 16;
  const uint32_t lbo = (uint32_t)rows * 16, sbo = 128;
  return (uint64_t)((start >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

// bounded wait on an mbarrier phase; false if the limit was reached
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}" : "=r"(done) : "r"(bar), "r"(phase) : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 64 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
  uint32_t r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
      "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
      "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
        "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]),
        "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]),
        "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]),
        "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
        "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]),
        "=r"(r[62]), "=r"(r[63])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 64; ++j) v[j] = __uint_as_float(r[j]);
}

// FROM_FEATURES: inputs are feature rows (ckd_mlp_predict) and the output is y;
// otherwise queries in leaf order and the output is the squared radius r2.
template <int D, bool FROM_FEATURES>
__global__ void __launch_bounds__(kTcRows, 1)
    k_mlp_tc(TreeView tv, const __nv_bfloat16* __restrict__ wb, MlpNorm nm,
             const double* __restrict__ Q, const int32_t* __restrict__ order,
             const int32_t* __restrict__ qleaf, const float* __restrict__ feat, int64_t n, int k,
             double* __restrict__ r2, float* __restrict__ y_out, unsigned* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int t = threadIdx.x, warp = t >> 5;
  float* F = reinterpret_cast<float*>(sm + kOffF);  // b1 | b2 | w3 | b3
  const uint32_t sA1 = smem_u32(sm + kOffA1), sA2 = smem_u32(sm + kOffA2);
  const uint32_t sB1 = smem_u32(sm + kOffB1), sB2 = smem_u32(sm + kOffB2);
  const uint32_t bar = smem_u32(sm + kOffBar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + kOffSlot);

  // ---- setup: TMEM, mbarrier, weights in the operand layouts
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = t; i < kMlpH * kK1; i += kTcRows) {  // W1 [64][12] -> 64 x 16
    const int nn = i / kK1, kk = i % kK1;
    const __nv_bfloat16 v = kk < kMlpF ? wb[kW1 + nn * kMlpF + kk] : __float2bfloat16_rn(0.0f);
    *reinterpret_cast<__nv_bfloat16*>(sm + kOffB1 + core_off(nn, kk, kMlpH)) = v;
  }
  for (int i = t; i < kMlpH * kMlpH; i += kTcRows) {  // W2 [64][64]
    const int nn = i / kMlpH, kk = i % kMlpH;
    *reinterpret_cast<__nv_bfloat16*>(sm + kOffB2 + core_off(nn, kk, kMlpH)) = wb[kW2 + i];
  }
  if (t < kMlpH) {
    F[t] = __bfloat162float(wb[kB1 + t]);
    F[kMlpH + t] = __bfloat162float(wb[kB2 + t]);
    F[2 * kMlpH + t] = __bfloat162float(wb[kW3 + t]);
  }
  if (t == 0) F[3 * kMlpH] = __bfloat162float(wb[kB3]);
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t taddr = *slot;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;
  uint32_t last_commit = 0;  // parity of the last commit thread 0 issued
  bool ok = true;

  for (int64_t base = (int64_t)blockIdx.x * kTcRows; base < n; base += (int64_t)gridDim.x * kTcRows) {
    const int64_t s = base + t;
    const bool valid = s < n;
    // ---- features of this thread's query -> row t of A1
    float f[kMlpF];
    int64_t qi = 0;
    if (FROM_FEATURES) {
#pragma unroll
      for (int j = 0; j < kMlpF; ++j) f[j] = valid ? feat[s * kMlpF + j] : 0.0f;
    } else {
#pragma unroll
      for (int j = 0; j < kMlpF; ++j) f[j] = 0.0f;
      if (valid) {
        qi = order ? (int64_t)order[s] : s;
        double q[D];
#pragma unroll
        for (int j = 0; j < D; ++j) q[j] = Q[qi * D + j];
        const int32_t leaf = qleaf ? qleaf[qi] : locate_leaf<D>(tv.meta, q);
        leaf_features<D>(tv, q, leaf, k, f);
      }
    }
#pragma unroll
    for (int kk = 0; kk < kK1; ++kk) {
      const float x = (kk < kMlpF && valid) ? (f[kk] - nm.mu[kk]) * nm.isg[kk] : 0.0f;
      *reinterpret_cast<__nv_bfloat16*>(sm + kOffA1 + core_off(t, kk, kTcRows)) =
          __float2bfloat16_rn(x);
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    // ---- layer 1
    if (t == 0 && ok) {
      mma_bf16(taddr, smem_desc(sA1, kTcRows, 0), smem_desc(sB1, kMlpH, 0), 0u);
      mma_commit(bar);
      last_commit = phase;
    }
    ok = ok && bar_wait(bar, phase);
    phase ^= 1u;
    fence_after();
    float h[64];
    tmem_ld64(taddr + lane_base, h);
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) {
      const float a = fmaxf(h[j] + F[j], 0.0f);
      *reinterpret_cast<__nv_bfloat16*>(sm + kOffA2 + core_off(t, j, kTcRows)) =
          __float2bfloat16_rn(a);
    }
    fence_async_smem();
    fence_before();
    ok = __syncthreads_and(ok);
    fence_after();
    // ---- layer 2
    if (t == 0 && ok) {
#pragma unroll
      for (int ks = 0; ks < kMlpH / 16; ++ks)
        mma_bf16(taddr + kMlpH, smem_desc(sA2, kTcRows, ks), smem_desc(sB2, kMlpH, ks),
                 ks > 0 ? 1u : 0u);
      mma_commit(bar);
      last_commit = phase;
    }
    ok = ok && bar_wait(bar, phase);
    phase ^= 1u;
    fence_after();
    tmem_ld64(taddr + lane_base + kMlpH, h);
    float z = F[3 * kMlpH];
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) z = fmaf(F[2 * kMlpH + j], fmaxf(h[j] + F[kMlpH + j], 0.0f), z);
    const float yv = nm.y_mu + nm.y_sigma * z;
    if (valid) {
      if (FROM_FEATURES) {
        y_out[s] = yv;
      } else {
        const double rr = exp2(2.0 * (double)(yv + nm.margin));
        // a timed-out wait leaves no usable prediction: an infinite bound makes the
        // search unbounded for this query (exact either way)
        r2[qi] = (ok && isfinite(rr)) ? rr : CKD_HUGE;
      }
    }
    fence_before();
    ok = __syncthreads_and(ok);  // every lane has read D1 / D2 before the next tile's MMAs
    fence_after();
  }
  // After a timed-out wait no further MMA is issued, but the one whose completion
  // was not seen may still be writing tensor memory: thread 0 waits for it once
  // more (bounded) before the columns are released to the next CTA.  A timeout
  // makes every output of the launch invalid (CKD_ERR_TIMEOUT is returned).
  if (!ok && t == 0) {
    atomicExch(err, 1u);
    bar_wait(bar, last_commit);
  }
  fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                 "r"(kTmemCols)
                 : "memory");
}

template <int D, bool FF>
ckd_status launch_tc(const ckd_tree* t, const ckd_mlp* net, const double* q, const int32_t* order,
                     const int32_t* qleaf, const float* feat, int64_t n, int k, double* r2,
                     float* y, cudaStream_t s) {
  static_assert(kTcSmem <= kTcSmemRequest, "shared memory layout exceeds the request");
  int dev = 0, sms = 148;
  CKD_CUDA(cudaGetDevice(&dev));
  CKD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CKD_CUDA(cudaFuncSetAttribute(k_mlp_tc<D, FF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kTcSmemRequest));
  unsigned* err = nullptr;
  CKD_CUDA(dev_alloc((void**)&err, sizeof(unsigned), s));
  CKD_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), s));
  const int64_t grid = std::min<int64_t>(cdiv(n, kTcRows), (int64_t)sms * 3);
  TreeView tv{};
  if (t) tv = t->view();
  k_mlp_tc<D, FF><<<(unsigned)std::max<int64_t>(1, grid), kTcRows, kTcSmemRequest, s>>>(
      tv, net->wb, net->norm, q, order, qleaf, feat, n, k, r2, y, err);
  note_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    dev_free(err, s);
    return cuda_fail(e, "k_mlp_tc");
  }
  unsigned herr = 0;
  CKD_CUDA(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  CKD_CUDA(cudaStreamSynchronize(s));
  dev_free(err, s);
  if (herr) return fail(CKD_ERR_TIMEOUT, "tensor-core MLP: an MMA completion wait timed out");
  return CKD_OK;
}

}  // namespace

ckd_status mlp_radius_tc(const ckd_tree* t, const ckd_mlp* net, const double* q,
                         const int32_t* order, const int32_t* qleaf, int64_t nq, int k, double* r2,
                         cudaStream_t s) {
  switch (t->d) {
#define CKD_TC(DD) \
  case DD: return launch_tc<DD, false>(t, net, q, order, qleaf, nullptr, nq, k, r2, nullptr, s);
    CKD_TC(1) CKD_TC(2) CKD_TC(3) CKD_TC(4) CKD_TC(5) CKD_TC(6) CKD_TC(7) CKD_TC(8)
#undef CKD_TC
  }
  return fail(CKD_ERR_BAD_DIM, "dimensionality must be 1..8");
}

ckd_status mlp_predict_tc(const ckd_mlp* net, const float* feat, int64_t n, float* y,
                          cudaStream_t s) {
  return launch_tc<3, true>(nullptr, net, nullptr, nullptr, nullptr, feat, n, 0, nullptr, y, s);
}

}  // namespace ckd
