// Training gradient of the edge-scoring MLP on the fifth-generation tensor cores (tcgen05,
// accumulators in tensor memory).
//
// The same network and rounding points as mlp.cu: BF16 operands, FP32 accumulation,
//   h1 = bf16(relu(x W1 + b1)), h2 = relu(h1 W2 + b2), logit = h2 . bf16(w3) + b3,
//   d = (sigmoid(logit) - y) / count, dh2 = bf16(d bf16(w3) [h2 > 0]),
//   dh1 = (dh2 W2^T) [h1 > 0],
// except that dh1 enters its weight-gradient contraction rounded to BF16 (it is a tensor-core
// operand there). A CTA of 128 threads takes 128 edges at a time, one edge row per thread
// and per TMEM lane, and issues from one thread:
//   D  = X W1             (M 128, N 64, K 16)   then, reusing D's columns,
//   D  = H1 W2            (M 128, N 64, K 64)
//   D  = dH2 W2^T         (M 128, N 64, K 64)
//   G2 += H1^T dH2        (M 64, N 64, K 128)   dW2, accumulated over the CTA's chunks
//   GX += X^T dH2         (M 64, N 64, K 128)   its row 15 is db2 (feature 15 is set to 1)
//   G1 += X^T dH1         (M 64, N 64, K 128)   rows 0..4 are dW1, row 15 is db1
// Each result is read back with tcgen05.ld by the thread that owns the row and turned into
// the next operand in shared memory (ReLU, bias, BF16) while the next MMA waits on an
// mbarrier that tcgen05.commit arrives on. dw3 and db3 are FP32 column sums of h2 d in shared
// memory. At exit the accumulators go to the global gradient with atomicAdd.
//
// Operands sit in shared memory without swizzling, as 16-byte units of eight consecutive
// BF16 values. A tile with rows r (edges, or weight columns) and 8-wide column blocks b
// keeps unit (r, b) at r * 16 + b * stride_b. The same bytes then serve as
//   - a K-major operand (rows = M or N, columns = K): 8-row groups 128 B apart (SBO), the two
//     8-column halves of a 16-wide K step stride_b apart (LBO);
//   - an MN-major operand (rows = K, columns = M or N): 8-column groups stride_b apart (SBO),
//     8-row groups of K 128 B apart (LBO).
// The descriptor and instruction-descriptor encodings follow the PTX ISA's tcgen05
// matrix and instruction descriptors (bit layouts as in CUTLASS's UMMA::SmemDescriptor and
// UMMA::InstrDescriptor).
#include <cuda_bf16.h>

#include "common.cuh"
#include "mlp.cuh"

namespace tspb {
namespace tc {

constexpr int ROWS = 128;       // edges per chunk: the M of the row-wise MMAs, one per thread
constexpr int TMEM_COLS = 256;  // D, G2, GX, G1: 64 FP32 columns each
constexpr int COL_D = 0, COL_G2 = 64, COL_GX = 128, COL_G1 = 192;

// shared-memory layout (bytes)
constexpr int S_X = 0;              // X: units (edge, fb), fb 0..7 (2..7 zero), 2048 B per block; two slots
constexpr int X_SLOT = 16384;       // tile t uses slot t % 2 (its column sums may still read it during t + 1)
constexpr int S_W1T = S_X + 2 * X_SLOT;  // W1 as N = hidden, K = feature: units (i, fb), 1024 B per block
constexpr int S_W2T = S_W1T + 2048;  // W2 as N = j, K = i: units (j, ib)
constexpr int S_W2 = S_W2T + 8192;   // W2 as N = i, K = j: units (i, jb)
constexpr int S_H1 = S_W2 + 8192;    // h1: units (edge, ib)
constexpr int S_DH2 = S_H1 + 16384;  // dh2: units (edge, jb)
constexpr int S_DH1 = S_DH2 + 16384;  // dh1: units (edge, ib)
constexpr int RED_STRIDE = 65;        // h2 d per edge row, padded against bank conflicts
constexpr int S_RED = S_DH1 + 16384;
constexpr int S_D = S_RED + ROWS * RED_STRIDE * 4;
constexpr int S_BAR = S_D + ROWS * 4;  // mbarrier (8 B)
constexpr int S_TMEM = S_BAR + 8;      // TMEM base address written by tcgen05.alloc
constexpr int S_BYTES = S_TMEM + 8;
static_assert(S_BAR % 8 == 0, "mbarrier alignment");

constexpr uint32_t idesc(int M, int N, bool a_mn, bool b_mn) {
  // bits 4-5 D format (1: F32), 7-9 A format and 10-12 B format (1: BF16), 15/16 A/B major
  // (1: MN-major), 17-22 N >> 3, 24-28 M >> 4
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
constexpr uint32_t ID_ROWS = idesc(128, 64, false, false);  // row-wise products, both K-major
constexpr uint32_t ID_SUMS = idesc(64, 64, true, true);     // sums over edges, both MN-major

// shared-memory matrix descriptor without swizzle: start, LBO and SBO in 16-byte units,
// version 1 (bit 46); base offset, LBO mode and layout type 0
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// Waits for the mbarrier phase with the given parity; false after about a second of SM
// cycles without it (the caller then records an error and stops issuing work).
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > (1LL << 31)) return false;
  }
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane; the wait names the registers so
// that no use of them is scheduled before the load completes.
__device__ __forceinline__ void tmem_load16(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])::"memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void tmem_load64(uint32_t addr, float (&v)[64]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) tmem_load16(addr + 16 * q, v + 16 * q);
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// A row of 64 values as eight 16-byte units (row, b) at base + row * 16 + b * 2048.
__device__ __forceinline__ void store_row(unsigned char* sm, int base, int row, const float (&v)[64]) {
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    uint4 u;
    u.x = pack2(v[8 * b + 0], v[8 * b + 1]);
    u.y = pack2(v[8 * b + 2], v[8 * b + 3]);
    u.z = pack2(v[8 * b + 4], v[8 * b + 5]);
    u.w = pack2(v[8 * b + 6], v[8 * b + 7]);
    *reinterpret_cast<uint4*>(sm + base + row * 16 + b * 2048) = u;
  }
}

__global__ void __launch_bounds__(ROWS, 1)
    mlp_train_tc_kernel(const float* __restrict__ P, const uint4* __restrict__ X4, const float* __restrict__ y,
                        long long E, float inv_count, float* __restrict__ grad, float* __restrict__ loss,
                        int32_t* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ float s_b1[MLP_H], s_b2[MLP_H], s_w3[MLP_H];
  __shared__ float s_b3;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long chunks = (E + ROWS - 1) / ROWS;
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t bar = base + S_BAR;

  // weights as K-major operands, biases, the zero X blocks, the mbarrier, tensor memory
  for (int q = tid; q < MLP_H; q += ROWS) {
    s_b1[q] = P[OFF_B1 + q];
    s_b2[q] = P[OFF_B2 + q];
    s_w3[q] = bf16_round(P[OFF_W3 + q]);
  }
  if (tid == 0) s_b3 = P[OFF_B3];
  for (int q = tid; q < MLP_H * 2; q += ROWS) {  // W1 as (N = i, K = f): unit (i, fb) = W1[8 fb + t][i]
    const int i = q & 63, fb = q >> 6;
    const float* w = P + OFF_W1 + 8 * fb * MLP_H + i;
    uint4 u;
    u.x = pack2(w[0], w[MLP_H]);
    u.y = pack2(w[2 * MLP_H], w[3 * MLP_H]);
    u.z = pack2(w[4 * MLP_H], w[5 * MLP_H]);
    u.w = pack2(w[6 * MLP_H], w[7 * MLP_H]);
    *reinterpret_cast<uint4*>(sm + S_W1T + i * 16 + fb * 1024) = u;
  }
  for (int q = tid; q < MLP_H * 8; q += ROWS) {
    const int r = q & 63, b = q >> 6;
    const float* wt = P + OFF_W2 + 8 * b * MLP_H + r;  // W2 as (N = j, K = i): unit (j, ib) = W2[8 ib + t][j]
    uint4 u;
    u.x = pack2(wt[0], wt[MLP_H]);
    u.y = pack2(wt[2 * MLP_H], wt[3 * MLP_H]);
    u.z = pack2(wt[4 * MLP_H], wt[5 * MLP_H]);
    u.w = pack2(wt[6 * MLP_H], wt[7 * MLP_H]);
    *reinterpret_cast<uint4*>(sm + S_W2T + r * 16 + b * 1024) = u;
    const float* w = P + OFF_W2 + r * MLP_H + 8 * b;  // W2 as (N = i, K = j): unit (i, jb) = W2[i][8 jb + t]
    u.x = pack2(w[0], w[1]);
    u.y = pack2(w[2], w[3]);
    u.z = pack2(w[4], w[5]);
    u.w = pack2(w[6], w[7]);
    *reinterpret_cast<uint4*>(sm + S_W2 + r * 16 + b * 1024) = u;
  }
  for (int q = tid; q < 12 * ROWS; q += ROWS)  // X blocks 2..7 of both slots: the zero rows 16..63 of X^T
    *reinterpret_cast<uint4*>(sm + S_X + (q / (6 * ROWS)) * X_SLOT + (q % ROWS) * 16 + (2 + (q / ROWS) % 6) * 2048) =
        make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(base + S_TMEM),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + S_TMEM);
  const uint32_t row_addr = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's quarter of the lanes
  float* red = reinterpret_cast<float*>(sm + S_RED);
  float* dsh = reinterpret_cast<float*>(sm + S_D);
  uint32_t phase = 0;
  float gw3 = 0.f, gb3 = 0.f, lsum = 0.f;
  int iter = 0;
  bool ok = true;
  // every MMA group ends with a commit on the mbarrier that all threads then wait for
  auto wait_mma = [&]() {
    const bool got = wait_phase(bar, phase);
    phase ^= 1u;
    fence_after();
    ok = __syncthreads_and(got) != 0;
  };
  auto publish = [&]() {  // generic shared-memory writes -> visible to the next MMA
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
  };
  float v[64];

  for (long long c = blockIdx.x; c < chunks; c += gridDim.x, ++iter) {
    const long long e = c * ROWS + tid;
    const bool valid = e < E;
    uint4 u0 = make_uint4(0, 0, 0, 0), u1 = u0;
    if (valid) {
      u0 = __ldg(X4 + 2 * e);
      u1 = __ldg(X4 + 2 * e + 1);
    }
    u1.w = (u1.w & 0xFFFFu) | (0x3F80u << 16);  // feature 15 = 1: the rows of X^T dH at index 15 sum dH
    const int sx = S_X + (iter & 1) * X_SLOT;  // the previous tile's column sums may still read the other slot
    *reinterpret_cast<uint4*>(sm + sx + tid * 16) = u0;
    *reinterpret_cast<uint4*>(sm + sx + tid * 16 + 2048) = u1;
    const float yv = valid ? __ldg(y + e) : 0.f;
    publish();
    // h1 = bf16(relu(X W1 + b1))
    if (tid == 0) {
      mma(tmem + COL_D, sdesc(base + sx, 2048, 128), sdesc(base + S_W1T, 1024, 128), ID_ROWS, 0);
      commit(bar);  // also the previous tile's column sums, issued before this MMA
    }
    wait_mma();
    if (!ok) break;
    tmem_load64(row_addr + COL_D, v);
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = bf16_round(fmaxf(v[i] + s_b1[i], 0.f));
    store_row(sm, S_H1, tid, v);
    publish();
    // h2 = relu(h1 W2 + b2), the logit, the loss and dh2
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 4; ++s)
        mma(tmem + COL_D, sdesc(base + S_H1 + s * 4096, 2048, 128), sdesc(base + S_W2T + s * 2048, 1024, 128), ID_ROWS,
            s > 0 ? 1u : 0u);
      commit(bar);
    }
    wait_mma();
    if (!ok) break;
    tmem_load64(row_addr + COL_D, v);
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < 64; ++i) {
      v[i] = fmaxf(v[i] + s_b2[i], 0.f);
      acc += v[i] * s_w3[i];
    }
    const float logit = acc + s_b3;
    float d = 0.f;
    if (valid) {
      lsum += fmaxf(logit, 0.f) - logit * yv + log1pf(__expf(-fabsf(logit)));
      d = (1.f / (1.f + __expf(-logit)) - yv) * inv_count;
    }
    dsh[tid] = d;
#pragma unroll
    for (int i = 0; i < 64; ++i) {
      red[tid * RED_STRIDE + i] = v[i] * d;
      v[i] = v[i] > 0.f ? d * s_w3[i] : 0.f;
    }
    store_row(sm, S_DH2, tid, v);
    publish();
    // dh1 = dh2 W2^T (masked below), committed alone; then dW2 += h1^T dh2 and db2 (row 15
    // of X^T dh2), which run on while the threads mask dh1. Nothing rewrites h1, dh2 or this
    // X slot before the next tile's first commit, which also covers these sums.
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 4; ++s)
        mma(tmem + COL_D, sdesc(base + S_DH2 + s * 4096, 2048, 128), sdesc(base + S_W2 + s * 2048, 1024, 128), ID_ROWS,
            s > 0 ? 1u : 0u);
      commit(bar);
#pragma unroll
      for (int s = 0; s < 8; ++s)
        mma(tmem + COL_G2, sdesc(base + S_H1 + s * 256, 128, 2048), sdesc(base + S_DH2 + s * 256, 128, 2048), ID_SUMS,
            (iter > 0 || s > 0) ? 1u : 0u);
#pragma unroll
      for (int s = 0; s < 8; ++s)
        mma(tmem + COL_GX, sdesc(base + sx + s * 256, 128, 2048), sdesc(base + S_DH2 + s * 256, 128, 2048), ID_SUMS,
            (iter > 0 || s > 0) ? 1u : 0u);
    }
    // dw3 and db3 in FP32 while the tensor cores run
    if (tid < 64) {
      float s_ = 0.f;
      for (int r = 0; r < ROWS; ++r) s_ += red[r * RED_STRIDE + tid];
      gw3 += s_;
    } else if (warp == 2) {
      float s_ = 0.f;
      for (int r = lane; r < ROWS; r += 32) s_ += dsh[r];
      s_ = warp_sum(s_);
      if (lane == 0) gb3 += s_;
    }
    wait_mma();
    if (!ok) break;
    tmem_load64(row_addr + COL_D, v);
#pragma unroll
    for (int b = 0; b < 8; ++b) {  // mask with this row's h1 > 0
      const uint4 h = *reinterpret_cast<const uint4*>(sm + S_H1 + tid * 16 + b * 2048);
      v[8 * b + 0] = bf16_lo(h.x) > 0.f ? v[8 * b + 0] : 0.f;
      v[8 * b + 1] = bf16_hi(h.x) > 0.f ? v[8 * b + 1] : 0.f;
      v[8 * b + 2] = bf16_lo(h.y) > 0.f ? v[8 * b + 2] : 0.f;
      v[8 * b + 3] = bf16_hi(h.y) > 0.f ? v[8 * b + 3] : 0.f;
      v[8 * b + 4] = bf16_lo(h.z) > 0.f ? v[8 * b + 4] : 0.f;
      v[8 * b + 5] = bf16_hi(h.z) > 0.f ? v[8 * b + 5] : 0.f;
      v[8 * b + 6] = bf16_lo(h.w) > 0.f ? v[8 * b + 6] : 0.f;
      v[8 * b + 7] = bf16_hi(h.w) > 0.f ? v[8 * b + 7] : 0.f;
    }
    store_row(sm, S_DH1, tid, v);
    publish();
    // dW1 (rows 0..4) and db1 (row 15) += X^T dh1: not waited for here. The next tile loads
    // its X into the other slot meanwhile, and its first commit covers these MMAs before it
    // rewrites dh1.
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 8; ++s)
        mma(tmem + COL_G1, sdesc(base + sx + s * 256, 128, 2048), sdesc(base + S_DH1 + s * 256, 128, 2048), ID_SUMS,
            (iter > 0 || s > 0) ? 1u : 0u);
    }
  }
  if (ok && iter > 0) {  // the last tile's column sums
    if (tid == 0) commit(bar);
    wait_mma();
  }

  fence_before();
  __syncthreads();
  fence_after();
  if (ok && iter > 0) {
    // M = 64 accumulators: row m lives in lane (m % 16) + 32 (m / 16), i.e. lanes 0..15 of
    // each warp's quarter hold rows 16 w .. 16 w + 15
    const int m = 16 * warp + lane;
    tmem_load64(row_addr + COL_G2, v);
    if (lane < 16)
      for (int j = 0; j < 64; ++j) atomicAdd(grad + OFF_W2 + m * MLP_H + j, v[j]);
    tmem_load64(row_addr + COL_G1, v);
    if (lane < 16 && m < MLP_F)
      for (int i = 0; i < 64; ++i) atomicAdd(grad + OFF_W1 + m * MLP_H + i, v[i]);
    if (lane < 16 && m == 15)
      for (int i = 0; i < 64; ++i) atomicAdd(grad + OFF_B1 + i, v[i]);
    tmem_load64(row_addr + COL_GX, v);
    if (lane < 16 && m == 15)
      for (int j = 0; j < 64; ++j) atomicAdd(grad + OFF_B2 + j, v[j]);
    if (tid < 64) atomicAdd(grad + OFF_W3 + tid, gw3);
    if (warp == 2 && lane == 0) atomicAdd(grad + OFF_B3, gb3);
    lsum = warp_sum(lsum);
    if (lane == 0) atomicAdd(loss, lsum);
  }
  if (!ok && tid == 0 && status) *status = TSPB_ERR_BUDGET;
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

}  // namespace tc
}  // namespace tspb

using namespace tspb;

extern "C" int tspb_mlp_train_grad_tc(const float* params, const uint16_t* x, const float* labels, int64_t num_edges,
                                      float* grad, float* loss, int32_t* status, void* stream) {
  if (num_edges < 0) return TSPB_ERR_ARG;
  if (num_edges == 0) return TSPB_OK;
  if (!params || !x || !labels || !grad || !loss) return TSPB_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(x) & 15u) != 0) return TSPB_ERR_ARG;  // rows are read as two 16-byte vectors
  int dev = 0, sms = 0;
  TSPB_CUDA_CHECK(cudaGetDevice(&dev));
  TSPB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  TSPB_CUDA_CHECK(cudaFuncSetAttribute(tc::mlp_train_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::S_BYTES));
  const long long chunks = (num_edges + tc::ROWS - 1) / tc::ROWS;
  const int blocks = chunks < sms ? (int)chunks : sms;
  tc::mlp_train_tc_kernel<<<blocks, tc::ROWS, tc::S_BYTES, reinterpret_cast<cudaStream_t>(stream)>>>(
      params, reinterpret_cast<const uint4*>(x), labels, num_edges, (float)(1.0 / (double)num_edges), grad, loss, status);
  return tspb_launch_status();
}
