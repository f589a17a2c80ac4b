// b2_mlp.cuh -- the learned warm start: a BF16 multilayer perceptron
// 32 -> 128 -> 128 -> 16 (25 contact features plus a constant, 3 outputs),
// GELU activations, FP32 accumulation, on the fifth-generation tensor cores.
//
// Every product is a tcgen05.mma (kind::f16, BF16 operands, FP32 accumulator
// in tensor memory) issued by one thread of a 128-thread CTA; operands sit in
// shared memory in the canonical no-swizzle layout of 8x8 core matrices
// (128 contiguous bytes, 8 rows of 16 bytes). A matrix stored row by row in
// that layout serves as a K-major operand of its natural shape and, through
// an MN-major descriptor, as the transposed operand of the backward products,
// so no transposed copies are kept. Tile = 128 samples = the 128 TMEM lanes:
// thread t of the CTA owns sample t in every epilogue (tcgen05.ld 32x32b).
//
// Training (k_mlp_grad): forward, mean-squared loss over the 3 outputs,
// backward, and per-tile parameter gradients written to a partial array that
// k_mlp_adam sums in tile order (deterministic) before the Adam update.
// Inference (k_mlp_forward): the forward pass over a persistent loop of tiles,
// with a caller-supplied feature source and output sink.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include "b2_common.cuh"

namespace b2 {
namespace mlp {

constexpr int kRows = 128;     // samples per tile: MMA M and TMEM lanes
constexpr int kIn = 32;        // input columns: 25 features, the constant 1 (bias of layer 1), zero padding
constexpr int kFeatures = 25;
constexpr int kBiasCol = 25;
constexpr int kHid = 128;
constexpr int kOut = 16;       // output columns: 3 used, zero padding to the MMA's smallest N
constexpr int kUsedOut = 3;
constexpr int kThreads = 128;

// FP32 parameter vector: W1 [kHid][kIn] (column kBiasCol is b1), W2 [kHid][kHid], b2, W3 [kOut][kHid], b3
constexpr int kPW1 = 0;
constexpr int kPW2 = kPW1 + kHid * kIn;
constexpr int kPB2 = kPW2 + kHid * kHid;
constexpr int kPW3 = kPB2 + kHid;
constexpr int kPB3 = kPW3 + kOut * kHid;
constexpr int kParams = kPB3 + kOut;

// BF16 weights packed in the canonical operand layout (byte offsets)
constexpr int kBW1 = 0;
constexpr int kBW2 = kBW1 + kHid * kIn * 2;
constexpr int kBW3 = kBW2 + kHid * kHid * 2;
constexpr int kPackedBytes = kBW3 + kOut * kHid * 2;

// shared memory of the kernels (byte offsets from a 1024-byte aligned base)
constexpr int kSW = 0;                              // packed weights
constexpr int kSX = kSW + kPackedBytes;             // X  [128 x 32]
constexpr int kSH1 = kSX + kRows * kIn * 2;         // H1 [128 x 128]
constexpr int kSH2 = kSH1 + kRows * kHid * 2;       // H2 [128 x 128], later dZ1
constexpr int kSDY = kSH2 + kRows * kHid * 2;       // dY [128 x 16]
constexpr int kSDZ2 = kSDY + kRows * kOut * 2;      // dZ2 [128 x 128]
constexpr int kSB2 = kSDZ2 + kRows * kHid * 2;      // b2 (float [128])
constexpr int kSB3 = kSB2 + kHid * 4;               // b3 (float [16])
constexpr int kSRed = kSB3 + kOut * 4;              // per-warp column sums of dZ2 (float [4][128])
constexpr int kSRed3 = kSRed + 4 * kHid * 4;        // per-warp column sums of dY (float [4][16])
constexpr int kSLoss = kSRed3 + 4 * kOut * 4;       // per-warp loss sums (float [4])
constexpr int kSBar = kSLoss + 16;                  // mbarriers: [0] MMA completion, [1] weight load
constexpr int kSTmem = kSBar + 16;                  // TMEM base address written by tcgen05.alloc
constexpr int kSmemGrad = kSTmem + 16;
constexpr int kSmemFwd = kSDY;                      // the forward pass uses weights, X, H1, H2 ...
constexpr int kSmemFwdTotal = kSmemGrad;            // ... but keeps the same map for the biases and barriers
constexpr int kSmemAlign = 1024;

// TMEM columns (512 allocated; one CTA per SM by its shared memory)
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kTZ1 = 0, kTZ2 = 128, kTY = 256, kTDH2 = 256, kTDW3 = 384, kTDH1 = 128, kTDW2 = 256, kTDW1 = 0;

constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s per bounded wait

// ---- layout and descriptors -------------------------------------------------

// byte offset of element (r, k) of an [R x K] BF16 matrix in the canonical
// no-swizzle layout: core matrix (r/8, k/8) at ((r/8)(K/8) + k/8) * 128 bytes,
// row r%8 of it at 16-byte stride, element k%8 at 2-byte stride
__host__ __device__ __forceinline__ uint32_t kmaj(int r, int k, int K) {
  return (uint32_t)(((((r >> 3) * (K >> 3)) + (k >> 3)) << 7) | ((r & 7) << 4) | ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor (no swizzle, sm100 version field = 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// K-major operand: an [MN x K] matrix (K = its column count), K-step kk of 16
// elements: the two 8-column core matrices are adjacent (128 bytes apart), the
// 8-row groups K*16 bytes apart
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t base, int K, int kk) {
  return sdesc(base + (uint32_t)kk * 256u, 128u, (uint32_t)K * 16u);
}

// MN-major operand read from a [Kdim x MN] matrix stored row by row (rows are
// the reduction index): K-step kk covers rows 16kk..16kk+15; 8-row groups are
// MN*16 bytes apart (leading offset), 8-column core matrices 128 bytes (stride)
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t base, int MN, int kk) {
  return sdesc(base + (uint32_t)kk * (uint32_t)MN * 32u, (uint32_t)MN * 16u, 128u);
}

// instruction descriptor of kind::f16: BF16 A and B, FP32 D, M x N, majors
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- tcgen05, mbarrier and bulk-copy wrappers -------------------------------

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory made visible to the tensor cores
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity to complete; on timeout the
// error flag is set and false returned (the caller skips the rest of its work).
__device__ __noinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer_ns() - t0 > kWaitLimitNs) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// one-dimensional bulk copy global -> shared, completion counted on the mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {  // one full warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {  // the allocating warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (the load and its
// wait in one statement, so no register is read before it has arrived)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// D (+)= A B^T, M = 128, over ksteps K-steps of 16; A and B in K-major or
// MN-major form (ld = the stored matrix's column count). One thread issues.
__device__ __forceinline__ void gemm(uint32_t d, uint32_t a, int a_mn, int a_ld, uint32_t b, int b_mn, int b_ld, int N,
                                     int ksteps) {
  const uint32_t id = idesc_bf16(kRows, N, a_mn, b_mn);
  for (int kk = 0; kk < ksteps; kk++) {
    const uint64_t ad = a_mn ? desc_mnmajor(a, a_ld, kk) : desc_kmajor(a, a_ld, kk);
    const uint64_t bd = b_mn ? desc_mnmajor(b, b_ld, kk) : desc_kmajor(b, b_ld, kk);
    umma_bf16(d, ad, bd, id, kk > 0 ? 1u : 0u);
  }
}

// ---- activation ---------------------------------------------------------------

// tanh by the SFU's approximate instruction (relative error about 2^-11,
// below the BF16 rounding of the activations it feeds): the epilogues evaluate
// 256 activations per sample and tile, which the accurate libm tanhf made the
// bottleneck of the forward pass
__device__ __forceinline__ float tanh_sfu(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// GELU, tanh form: g(x) = x/2 (1 + tanh(c (x + a x^3)))
__device__ __forceinline__ float gelu(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  return 0.5f * x * (1.0f + tanh_sfu(u));
}

__device__ __forceinline__ float gelu_grad(float x) {
  const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
  const float t = tanh_sfu(u);
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * x * x);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// 8 consecutive columns (c0 multiple of 8) of row r into an [R x K] operand
__device__ __forceinline__ void store8(unsigned char* base, int r, int c0, int K, const float* v) {
  uint4 q;
  q.x = pack_bf16x2(v[0], v[1]);
  q.y = pack_bf16x2(v[2], v[3]);
  q.z = pack_bf16x2(v[4], v[5]);
  q.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4*>(base + kmaj(r, c0, K)) = q;
}

// ---- kernels ------------------------------------------------------------------

struct Shared {
  unsigned char* base;
  uint32_t s;  // shared address of base
  __device__ uint32_t at(int off) const { return s + (uint32_t)off; }
};

__device__ __forceinline__ Shared shared_base(unsigned char* raw) {
  const uint32_t s0 = smem_u32(raw);
  const uint32_t pad = (kSmemAlign - (s0 & (kSmemAlign - 1))) & (kSmemAlign - 1);
  Shared sh;
  sh.base = raw + pad;
  sh.s = s0 + pad;
  return sh;
}

// CTA set-up: barriers, TMEM, weights (bulk copy) and biases. Returns the TMEM base.
__device__ __forceinline__ uint32_t setup(const Shared& sh, const unsigned char* wpacked, const float* P, int* err,
                                          bool& ok) {
  const int tid = threadIdx.x;
  const uint32_t bar_mma = sh.at(kSBar), bar_ld = sh.at(kSBar + 8);
  if (tid == 0) {
    mbar_init(bar_mma, 1);
    mbar_init(bar_ld, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < kWarp) tmem_alloc(sh.at(kSTmem), kTmemCols);
  float* b2 = reinterpret_cast<float*>(sh.base + kSB2);
  float* b3 = reinterpret_cast<float*>(sh.base + kSB3);
  b2[tid] = P[kPB2 + tid];
  if (tid < kOut) b3[tid] = P[kPB3 + tid];
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(bar_ld, kPackedBytes);
    bulk_g2s(sh.at(kSW + kBW1), wpacked + kBW1, kBW2 - kBW1, bar_ld);
    bulk_g2s(sh.at(kSW + kBW2), wpacked + kBW2, kBW3 - kBW2, bar_ld);
    bulk_g2s(sh.at(kSW + kBW3), wpacked + kBW3, kPackedBytes - kBW3, bar_ld);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sh.base + kSTmem);
  ok = __syncthreads_and(mbar_wait(bar_ld, 0, err)) != 0;
  return tmem;
}

__device__ __forceinline__ void teardown(uint32_t tmem) {
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < kWarp) {
    tc_fence_after();
    tmem_free(tmem, kTmemCols);
  }
}

// shared-memory writes of all threads -> one thread issues products -> commit;
// every thread waits for the products. Returns false on a timed-out wait.
template <class Issue>
__device__ __forceinline__ bool run_mma(const Shared& sh, uint32_t& phase, int* err, Issue issue) {
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_fence_after();
    issue();
    umma_commit(sh.at(kSBar));
  }
  const bool ok = mbar_wait(sh.at(kSBar), phase, err);
  phase ^= 1u;
  tc_fence_after();
  return __syncthreads_and(ok) != 0;  // the same outcome in every thread
}

// Forward pass of one tile whose X is in shared memory: Z1 -> H1 -> Z2 -> H2 ->
// Y. On return thread t holds y[0..2] of sample t (biases added).
__device__ __forceinline__ bool forward_tile(const Shared& sh, uint32_t tmem, uint32_t& phase, int* err, float (&y)[3]) {
  const int tid = threadIdx.x;
  const int r = tid;
  const uint32_t lane_off = (uint32_t)((tid & ~31) << 16);  // this warp's TMEM lane quarter
  const uint32_t sW = sh.at(kSW), sX = sh.at(kSX), sH1 = sh.at(kSH1), sH2 = sh.at(kSH2);
  const float* b2 = reinterpret_cast<const float*>(sh.base + kSB2);
  const float* b3 = reinterpret_cast<const float*>(sh.base + kSB3);
  // Z1 = X W1^T (b1 through the constant column)
  if (!run_mma(sh, phase, err, [&] { gemm(tmem + kTZ1, sX, 0, kIn, sW + kBW1, 0, kIn, kHid, kIn / 16); })) return false;
#pragma unroll 1
  for (int c = 0; c < kHid; c += 16) {
    float v[16];
    tmem_ld16(tmem + lane_off + kTZ1 + c, v);
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = gelu(v[i]);
    store8(sh.base + kSH1, r, c, kHid, v);
    store8(sh.base + kSH1, r, c + 8, kHid, v + 8);
  }
  // Z2 = H1 W2^T, + b2
  if (!run_mma(sh, phase, err, [&] { gemm(tmem + kTZ2, sH1, 0, kHid, sW + kBW2, 0, kHid, kHid, kHid / 16); }))
    return false;
#pragma unroll 1
  for (int c = 0; c < kHid; c += 16) {
    float v[16];
    tmem_ld16(tmem + lane_off + kTZ2 + c, v);
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = gelu(v[i] + b2[c + i]);
    store8(sh.base + kSH2, r, c, kHid, v);
    store8(sh.base + kSH2, r, c + 8, kHid, v + 8);
  }
  // Y = H2 W3^T, + b3
  if (!run_mma(sh, phase, err, [&] { gemm(tmem + kTY, sH2, 0, kHid, sW + kBW3, 0, kHid, kOut, kHid / 16); }))
    return false;
  float v[16];
  tmem_ld16(tmem + lane_off + kTY, v);
#pragma unroll
  for (int o = 0; o < kUsedOut; o++) y[o] = v[o] + b3[o];
  return true;
}

// Gradient of the mean-squared loss over one tile of 128 samples (rows
// tile*128 .. of the dataset, those >= nrows masked). Writes the tile's
// parameter gradient to gpart[blockIdx.x][kParams] and its loss sum to
// lpart[blockIdx.x]. inv_n = 1 / (samples in the minibatch).
__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_grad(const unsigned char* __restrict__ wpacked, const float* __restrict__ P, const float* __restrict__ feat,
               const float* __restrict__ target, const int* __restrict__ tiles, int nrows, float inv_n,
               float* __restrict__ gpart, float* __restrict__ lpart, int* err) {
  extern __shared__ unsigned char mlp_smem_raw[];
  const Shared sh = shared_base(mlp_smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t lane_off = (uint32_t)((tid & ~31) << 16);
  bool ok = true;
  const uint32_t tmem = setup(sh, wpacked, P, err, ok);
  uint32_t phase = 0;
  float* g = gpart + (size_t)blockIdx.x * kParams;
  const float* b2 = reinterpret_cast<const float*>(sh.base + kSB2);
  float* red = reinterpret_cast<float*>(sh.base + kSRed);
  float* red3 = reinterpret_cast<float*>(sh.base + kSRed3);
  float* lsum = reinterpret_cast<float*>(sh.base + kSLoss);

  const int tile = tiles ? tiles[blockIdx.x] : (int)blockIdx.x;
  const long long row = (long long)tile * kRows + tid;
  const bool live = row < nrows;
  float t[3] = {0.f, 0.f, 0.f};
  {  // X tile (FP32 dataset -> BF16 operand)
    float x[kIn];
#pragma unroll
    for (int k = 0; k < kIn; k++) x[k] = live ? feat[row * kIn + k] : 0.f;
#pragma unroll
    for (int k = 0; k < kIn; k += 8) store8(sh.base + kSX, tid, k, kIn, x + k);
    if (live) {
#pragma unroll
      for (int o = 0; o < 3; o++) t[o] = target[row * 3 + o];
    }
  }
  float y[3] = {0.f, 0.f, 0.f};
  if (ok) ok = forward_tile(sh, tmem, phase, err, y);

  // loss and dY = 2 (y - t) / n (masked rows contribute nothing)
  float dy[kOut];
#pragma unroll
  for (int o = 0; o < kOut; o++) dy[o] = 0.f;
  float loss = 0.f;
  if (live) {
#pragma unroll
    for (int o = 0; o < kUsedOut; o++) {
      const float e = y[o] - t[o];
      loss += e * e;
      dy[o] = 2.0f * e * inv_n;
    }
  }
  store8(sh.base + kSDY, tid, 0, kOut, dy);
  store8(sh.base + kSDY, tid, 8, kOut, dy + 8);
  // column sums over the tile (bias gradients), warp shuffles then per-warp slots
#pragma unroll
  for (int o = 0; o < kOut; o++) {
    float sdy = dy[o];
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) sdy += __shfl_xor_sync(0xffffffffu, sdy, d);
    if (lane == 0) red3[warp * kOut + o] = sdy;
  }
  {
    float sl = loss;
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) sl += __shfl_xor_sync(0xffffffffu, sl, d);
    if (lane == 0) lsum[warp] = sl;
  }

  // dH2 = dY W3 (B = W3 as MN-major [in x out]); dW3^T = H2^T dY (contraction over samples)
  const uint32_t sW = sh.at(kSW), sX = sh.at(kSX), sH1 = sh.at(kSH1), sH2 = sh.at(kSH2), sDY = sh.at(kSDY),
                 sDZ2 = sh.at(kSDZ2);
  if (ok) ok = run_mma(sh, phase, err, [&] {
    gemm(tmem + kTDH2, sDY, 0, kOut, sW + kBW3, 1, kHid, kHid, kOut / 16);
    gemm(tmem + kTDW3, sH2, 1, kHid, sDY, 1, kOut, kOut, kRows / 16);
  });
  // dZ2 = dH2 * gelu'(Z2 + b2); dW3 out of TMEM (lane = input unit i, column = output o)
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < kHid; c += 16) {
      float dh[16], z[16];
      tmem_ld16(tmem + lane_off + kTDH2 + c, dh);
      tmem_ld16(tmem + lane_off + kTZ2 + c, z);
#pragma unroll
      for (int i = 0; i < 16; i++) dh[i] = live ? dh[i] * gelu_grad(z[i] + b2[c + i]) : 0.f;
      store8(sh.base + kSDZ2, tid, c, kHid, dh);
      store8(sh.base + kSDZ2, tid, c + 8, kHid, dh + 8);
#pragma unroll
      for (int i = 0; i < 16; i++) {
        float s = dh[i];
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
        if (lane == 0) red[warp * kHid + c + i] = s;
      }
    }
    float w3[16];
    tmem_ld16(tmem + lane_off + kTDW3, w3);
#pragma unroll
    for (int o = 0; o < kOut; o++) g[kPW3 + o * kHid + tid] = w3[o];
  }
  // dH1 = dZ2 W2 (B = W2 as MN-major); dW2 = dZ2^T H1
  if (ok) ok = run_mma(sh, phase, err, [&] {
    gemm(tmem + kTDH1, sDZ2, 0, kHid, sW + kBW2, 1, kHid, kHid, kHid / 16);
    gemm(tmem + kTDW2, sDZ2, 1, kHid, sH1, 1, kHid, kHid, kRows / 16);
  });
  // dZ1 = dH1 * gelu'(Z1) into the H2 buffer; dW2 out of TMEM (lane = output unit o)
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < kHid; c += 16) {
      float dh[16], z[16];
      tmem_ld16(tmem + lane_off + kTDH1 + c, dh);
      tmem_ld16(tmem + lane_off + kTZ1 + c, z);
#pragma unroll
      for (int i = 0; i < 16; i++) dh[i] = live ? dh[i] * gelu_grad(z[i]) : 0.f;
      store8(sh.base + kSH2, tid, c, kHid, dh);
      store8(sh.base + kSH2, tid, c + 8, kHid, dh + 8);
      float w2[16];
      tmem_ld16(tmem + lane_off + kTDW2 + c, w2);
#pragma unroll
      for (int i = 0; i < 16; i++) g[kPW2 + tid * kHid + c + i] = w2[i];
    }
  }
  // dW1 = dZ1^T X
  if (ok) ok = run_mma(sh, phase, err, [&] { gemm(tmem + kTDW1, sH2, 1, kHid, sX, 1, kIn, kIn, kRows / 16); });
  if (ok) {
#pragma unroll
    for (int c = 0; c < kIn; c += 16) {
      float w1[16];
      tmem_ld16(tmem + lane_off + kTDW1 + c, w1);
#pragma unroll
      for (int i = 0; i < 16; i++) g[kPW1 + tid * kIn + c + i] = w1[i];
    }
    g[kPB2 + tid] = red[tid] + red[kHid + tid] + red[2 * kHid + tid] + red[3 * kHid + tid];
    if (tid < kOut) g[kPB3 + tid] = red3[tid] + red3[kOut + tid] + red3[2 * kOut + tid] + red3[3 * kOut + tid];
    if (tid == 0) lpart[blockIdx.x] = lsum[0] + lsum[1] + lsum[2] + lsum[3];
  }
  teardown(tmem);
}

// Adam step on the FP32 parameters from the tile gradients (summed in tile
// order), then the BF16 operand copy. Step size lr, moments beta1/beta2,
// bias corrections bc1 = 1 - beta1^t, bc2 = 1 - beta2^t.
__global__ void k_mlp_adam(float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ gpart, int ntiles, float lr, float beta1, float beta2, float eps,
                           float bc1, float bc2, unsigned char* __restrict__ wpacked, const float* __restrict__ lpart,
                           double* loss_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && loss_out) {
    double s = 0.0;
    for (int t = 0; t < ntiles; t++) s += (double)lpart[t];
    *loss_out = s;
  }
  if (p >= kParams) return;
  float gsum = 0.f;
  for (int t = 0; t < ntiles; t++) gsum += gpart[(size_t)t * kParams + p];
  const float mm = beta1 * m[p] + (1.0f - beta1) * gsum;
  const float vv = beta2 * v[p] + (1.0f - beta2) * gsum * gsum;
  m[p] = mm;
  v[p] = vv;
  const float w = P[p] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
  P[p] = w;
  __nv_bfloat16 h = __float2bfloat16_rn(w);
  if (p < kPW2) {
    *reinterpret_cast<__nv_bfloat16*>(wpacked + kBW1 + kmaj((p - kPW1) / kIn, (p - kPW1) % kIn, kIn)) = h;
  } else if (p < kPB2) {
    *reinterpret_cast<__nv_bfloat16*>(wpacked + kBW2 + kmaj((p - kPW2) / kHid, (p - kPW2) % kHid, kHid)) = h;
  } else if (p >= kPW3 && p < kPB3) {
    *reinterpret_cast<__nv_bfloat16*>(wpacked + kBW3 + kmaj((p - kPW3) / kHid, (p - kPW3) % kHid, kHid)) = h;
  }
}

// BF16 operand copy of the FP32 parameters (after they are set)
__global__ void k_mlp_pack(const float* __restrict__ P, unsigned char* __restrict__ wpacked) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  const __nv_bfloat16 h = __float2bfloat16_rn(P[p]);
  if (p < kPW2) {
    *reinterpret_cast<__nv_bfloat16*>(wpacked + kBW1 + kmaj((p - kPW1) / kIn, (p - kPW1) % kIn, kIn)) = h;
  } else if (p < kPB2) {
    *reinterpret_cast<__nv_bfloat16*>(wpacked + kBW2 + kmaj((p - kPW2) / kHid, (p - kPW2) % kHid, kHid)) = h;
  } else if (p >= kPW3 && p < kPB3) {
    *reinterpret_cast<__nv_bfloat16*>(wpacked + kBW3 + kmaj((p - kPW3) / kHid, (p - kPW3) % kHid, kHid)) = h;
  }
}

// Inference over ntiles tiles of 128 samples, persistent CTAs. Src fills the
// 32 inputs of one sample (and returns false for a sample past the end); Dst
// consumes the 3 outputs.
template <class Src, class Dst>
__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_forward(const unsigned char* __restrict__ wpacked, const float* __restrict__ P, int ntiles, Src src, Dst dst,
                  int* err) {
  extern __shared__ unsigned char mlp_smem_raw[];
  const Shared sh = shared_base(mlp_smem_raw);
  const int tid = threadIdx.x;
  bool ok = true;
  const uint32_t tmem = setup(sh, wpacked, P, err, ok);
  uint32_t phase = 0;
  for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
    const long long row = (long long)tile * kRows + tid;
    float x[kIn];
    const bool live = src(row, x);
#pragma unroll
    for (int k = 0; k < kIn; k += 8) store8(sh.base + kSX, tid, k, kIn, x + k);
    float y[3];
    ok = forward_tile(sh, tmem, phase, err, y);
    if (ok && live) dst(row, y);
  }
  teardown(tmem);
}

// feature source / output sink of the plain forward (a dataset in global memory)
struct ArraySrc {
  const float* feat;
  long long n;
  __device__ bool operator()(long long row, float (&x)[kIn]) const {
    const bool live = row < n;
#pragma unroll
    for (int k = 0; k < kIn; k++) x[k] = live ? feat[row * kIn + k] : 0.f;
    return live;
  }
};

struct ArrayDst {
  float* out;
  __device__ void operator()(long long row, const float (&y)[3]) const {
#pragma unroll
    for (int o = 0; o < 3; o++) out[row * 3 + o] = y[o];
  }
};

}  // namespace mlp
}  // namespace b2
