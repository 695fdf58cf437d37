// Edge-scoring MLP for learned 2-opt candidate lists: features, inference, training.
//
// Network: 5 edge features -> 64 (ReLU) -> 64 (ReLU) -> 1 logit. Weights are kept as FP32
// master copies and used in BF16; every product accumulates in FP32.
//   x  = bf16(features), padded to 16 columns
//   h1 = relu(x @ bf16(W1) + b1)          tensor cores (mma.sync m16n8k16, bf16 -> f32)
//   h2 = relu(bf16(h1) @ bf16(W2) + b2)   tensor cores; layer-1 outputs stay in registers:
//                                         the f32 accumulator fragment of layer 1 is the
//                                         bf16 A fragment of layer 2 after packing
//   logit = h2 . bf16(w3) + b3            f32, reduced across the four lanes of a row
// Training minimises the mean binary cross-entropy with logits; the backward pass
//   dlogit = (sigmoid(logit) - y) / count
//   dh2 = dlogit * bf16(w3) * [h2 > 0]
//   dh1 = (bf16(dh2) @ bf16(W2)^T) * [h1 > 0]   tensor cores
// and the weight gradients (sums over the 16 edges of a warp tile of outer products) run
// in FP32 on CUDA cores from per-warp shared-memory staging, then reduce to global FP32
// gradient buffers. Adam updates the FP32 masters.
//
// Parameter block (FP32, `TSPB_MLP_PARAMS` floats): W1[16][64] (rows >= 5 unused, kept
// zero), b1[64], W2[64][64], b2[64], w3[64], b3[1].
#include <cuda_bf16.h>

#include "common.cuh"
#include "mlp.cuh"

namespace tspb {

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// B fragments of the three weight operands, laid out per lane, plus biases (shared memory).
struct MlpShared {
  uint2 b1[8][32];      // W1  (k 16, n 64)
  uint2 b2[4][8][32];   // W2  (k 64, n 64)
  uint2 b2t[4][8][32];  // W2^T
  float bias1[64], bias2[64], w3[64];
  float b3;
};

// Fragment (k-tile t, n-tile j) of B[k][n] = W[k * ldw + n] for this lane.
__device__ __forceinline__ uint2 frag_b(const float* W, int ldw, int t, int j, int lane, bool transpose) {
  const int g = lane >> 2, tg = lane & 3;
  const int k0 = 16 * t + tg * 2, n = 8 * j + g;
  auto at = [&](int k) { return transpose ? W[n * ldw + k] : W[k * ldw + n]; };
  uint2 r;
  r.x = pack_bf16(at(k0), at(k0 + 1));
  r.y = pack_bf16(at(k0 + 8), at(k0 + 9));
  return r;
}

__device__ void mlp_load_shared(const float* __restrict__ P, MlpShared& S) {
  const int tid = threadIdx.x, T = blockDim.x;
  for (int q = tid; q < 8 * 32; q += T) S.b1[q >> 5][q & 31] = frag_b(P + OFF_W1, MLP_H, 0, q >> 5, q & 31, false);
  for (int q = tid; q < 4 * 8 * 32; q += T) {
    const int t = q >> 8, j = (q >> 5) & 7, l = q & 31;
    S.b2[t][j][l] = frag_b(P + OFF_W2, MLP_H, t, j, l, false);
    S.b2t[t][j][l] = frag_b(P + OFF_W2, MLP_H, t, j, l, true);
  }
  for (int q = tid; q < 64; q += T) {
    S.bias1[q] = P[OFF_B1 + q];
    S.bias2[q] = P[OFF_B2 + q];
    S.w3[q] = bf16r(P[OFF_W3 + q]);
  }
  if (tid == 0) S.b3 = P[OFF_B3];
}

// Forward of one 16-edge tile starting at e0. Fills h1 (bf16-rounded) and h2 in f32
// fragment layout [n-tile][4] and the two row logits of this lane's group.
__device__ __forceinline__ void mlp_forward_tile(const MlpShared& S, const uint32_t* __restrict__ X32, long long e0,
                                                 long long E, int lane, float (&h1)[8][4], float (&h2)[8][4],
                                                 float& logit_lo, float& logit_hi) {
  const int g = lane >> 2, tg = lane & 3;
  const long long r0 = e0 + g, r1 = e0 + g + 8;
  uint32_t a[4];
  a[0] = r0 < E ? X32[r0 * 8 + tg] : 0u;
  a[1] = r1 < E ? X32[r1 * 8 + tg] : 0u;
  a[2] = r0 < E ? X32[r0 * 8 + 4 + tg] : 0u;
  a[3] = r1 < E ? X32[r1 * 8 + 4 + tg] : 0u;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    mma_bf16(acc, a, S.b1[j][lane]);
    const int c = 8 * j + tg * 2;
    h1[j][0] = bf16r(fmaxf(acc[0] + S.bias1[c], 0.f));
    h1[j][1] = bf16r(fmaxf(acc[1] + S.bias1[c + 1], 0.f));
    h1[j][2] = bf16r(fmaxf(acc[2] + S.bias1[c], 0.f));
    h1[j][3] = bf16r(fmaxf(acc[3] + S.bias1[c + 1], 0.f));
  }
  float acc2[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc2[j][0] = acc2[j][1] = acc2[j][2] = acc2[j][3] = 0.f;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    uint32_t a2[4];
    a2[0] = pack_bf16(h1[2 * t][0], h1[2 * t][1]);
    a2[1] = pack_bf16(h1[2 * t][2], h1[2 * t][3]);
    a2[2] = pack_bf16(h1[2 * t + 1][0], h1[2 * t + 1][1]);
    a2[3] = pack_bf16(h1[2 * t + 1][2], h1[2 * t + 1][3]);
#pragma unroll
    for (int j = 0; j < 8; ++j) mma_bf16(acc2[j], a2, S.b2[t][j][lane]);
  }
  float lo = 0.f, hi = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = 8 * j + tg * 2;
    h2[j][0] = fmaxf(acc2[j][0] + S.bias2[c], 0.f);
    h2[j][1] = fmaxf(acc2[j][1] + S.bias2[c + 1], 0.f);
    h2[j][2] = fmaxf(acc2[j][2] + S.bias2[c], 0.f);
    h2[j][3] = fmaxf(acc2[j][3] + S.bias2[c + 1], 0.f);
    lo += h2[j][0] * S.w3[c] + h2[j][1] * S.w3[c + 1];
    hi += h2[j][2] * S.w3[c] + h2[j][3] * S.w3[c + 1];
  }
  lo += __shfl_xor_sync(FULL, lo, 1);
  lo += __shfl_xor_sync(FULL, lo, 2);
  hi += __shfl_xor_sync(FULL, hi, 1);
  hi += __shfl_xor_sync(FULL, hi, 2);
  logit_lo = lo + S.b3;
  logit_hi = hi + S.b3;
}

__global__ void __launch_bounds__(256) mlp_infer_kernel(const float* __restrict__ P, const uint32_t* __restrict__ X32,
                                                        long long E, float* __restrict__ logits) {
  __shared__ MlpShared S;
  mlp_load_shared(P, S);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long tile = warp; tile * 16 < E; tile += nwarps) {
    const long long e0 = tile * 16;
    float h1[8][4], h2[8][4], lo, hi;
    mlp_forward_tile(S, X32, e0, E, lane, h1, h2, lo, hi);
    if ((lane & 3) == 0) {
      const long long r0 = e0 + (lane >> 2), r1 = r0 + 8;
      if (r0 < E) logits[r0] = lo;
      if (r1 < E) logits[r1] = hi;
    }
  }
}

// Per-warp staging for the weight gradients of one tile (f32, row = edge of the tile).
struct WarpStage {
  float h1[16][64];
  float dh1[16][64];
  float h2[16][64];
  float dh2[16][64];
  float x[16][MLP_F];
  float d[16];
};

constexpr int TRAIN_WARPS = 4;

// One pass over E labelled edges: accumulates d(mean BCE)/dparams into grad (f32, same
// layout as P) and the summed loss into loss[0]. `inv_count` = 1 / (edges in the batch).
__global__ void __launch_bounds__(TRAIN_WARPS * 32) mlp_train_kernel(const float* __restrict__ P,
                                                                     const uint32_t* __restrict__ X32,
                                                                     const float* __restrict__ y, long long E,
                                                                     float inv_count, float* __restrict__ grad,
                                                                     float* __restrict__ loss) {
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ MlpShared S;
  mlp_load_shared(P, S);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  WarpStage& W = reinterpret_cast<WarpStage*>(dyn)[wid];
  float* gW2 = reinterpret_cast<float*>(dyn + sizeof(WarpStage) * TRAIN_WARPS) + wid * 64 * 64;  // per warp
  for (int q = lane; q < 64 * 64; q += 32) gW2[q] = 0.f;
  __syncthreads();
  const int g = lane >> 2, tg = lane & 3;
  const int i0 = 2 * lane, i1 = 2 * lane + 1;  // the hidden columns this lane owns for the sums
  float gb1[2] = {0.f, 0.f}, gb2[2] = {0.f, 0.f}, gw3[2] = {0.f, 0.f}, gw1[MLP_F][2];
#pragma unroll
  for (int f = 0; f < MLP_F; ++f) gw1[f][0] = gw1[f][1] = 0.f;
  float gb3 = 0.f, lsum = 0.f;
  const long long warp = ((long long)blockIdx.x * TRAIN_WARPS) + wid;
  const long long nwarps = (long long)gridDim.x * TRAIN_WARPS;
  for (long long tile = warp; tile * 16 < E; tile += nwarps) {
    const long long e0 = tile * 16;
    float h1[8][4], h2[8][4], lo, hi;
    mlp_forward_tile(S, X32, e0, E, lane, h1, h2, lo, hi);
    const long long r0 = e0 + g, r1 = r0 + 8;
    const bool v0 = r0 < E, v1 = r1 < E;
    const float y0 = v0 ? y[r0] : 0.f, y1 = v1 ? y[r1] : 0.f;
    const float d0 = v0 ? (1.f / (1.f + __expf(-lo)) - y0) * inv_count : 0.f;
    const float d1 = v1 ? (1.f / (1.f + __expf(-hi)) - y1) * inv_count : 0.f;
    if (tg == 0) {
      if (v0) lsum += fmaxf(lo, 0.f) - lo * y0 + log1pf(__expf(-fabsf(lo)));
      if (v1) lsum += fmaxf(hi, 0.f) - hi * y1 + log1pf(__expf(-fabsf(hi)));
    }
    // dh2 in fragment layout, then dh1 = bf16(dh2) @ W2^T on tensor cores
    float dh2[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + tg * 2;
      dh2[j][0] = h2[j][0] > 0.f ? d0 * S.w3[c] : 0.f;
      dh2[j][1] = h2[j][1] > 0.f ? d0 * S.w3[c + 1] : 0.f;
      dh2[j][2] = h2[j][2] > 0.f ? d1 * S.w3[c] : 0.f;
      dh2[j][3] = h2[j][3] > 0.f ? d1 * S.w3[c + 1] : 0.f;
    }
    float dh1[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) dh1[j][0] = dh1[j][1] = dh1[j][2] = dh1[j][3] = 0.f;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      uint32_t a[4];
      a[0] = pack_bf16(dh2[2 * t][0], dh2[2 * t][1]);
      a[1] = pack_bf16(dh2[2 * t][2], dh2[2 * t][3]);
      a[2] = pack_bf16(dh2[2 * t + 1][0], dh2[2 * t + 1][1]);
      a[3] = pack_bf16(dh2[2 * t + 1][2], dh2[2 * t + 1][3]);
#pragma unroll
      for (int j = 0; j < 8; ++j) mma_bf16(dh1[j], a, S.b2t[t][j][lane]);
    }
    // stage the tile for the outer-product sums
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + tg * 2;
      W.h1[g][c] = h1[j][0];
      W.h1[g][c + 1] = h1[j][1];
      W.h1[g + 8][c] = h1[j][2];
      W.h1[g + 8][c + 1] = h1[j][3];
      W.h2[g][c] = h2[j][0];
      W.h2[g][c + 1] = h2[j][1];
      W.h2[g + 8][c] = h2[j][2];
      W.h2[g + 8][c + 1] = h2[j][3];
      W.dh2[g][c] = bf16r(dh2[j][0]);
      W.dh2[g][c + 1] = bf16r(dh2[j][1]);
      W.dh2[g + 8][c] = bf16r(dh2[j][2]);
      W.dh2[g + 8][c + 1] = bf16r(dh2[j][3]);
      W.dh1[g][c] = h1[j][0] > 0.f ? dh1[j][0] : 0.f;
      W.dh1[g][c + 1] = h1[j][1] > 0.f ? dh1[j][1] : 0.f;
      W.dh1[g + 8][c] = h1[j][2] > 0.f ? dh1[j][2] : 0.f;
      W.dh1[g + 8][c + 1] = h1[j][3] > 0.f ? dh1[j][3] : 0.f;
    }
    if (tg == 0) {
      W.d[g] = d0;
      W.d[g + 8] = d1;
    }
    if (lane < 16) {
      const long long r = e0 + lane;
      const __nv_bfloat16* xr = reinterpret_cast<const __nv_bfloat16*>(X32 + r * 8);
#pragma unroll
      for (int f = 0; f < MLP_F; ++f) W.x[lane][f] = r < E ? __bfloat162float(xr[f]) : 0.f;
    }
    __syncwarp();
#pragma unroll 4
    for (int e = 0; e < 16; ++e) {
      const float de = W.d[e];
      gb3 += lane == 0 ? de : 0.f;
      gw3[0] += W.h2[e][i0] * de;
      gw3[1] += W.h2[e][i1] * de;
      gb2[0] += W.dh2[e][i0];
      gb2[1] += W.dh2[e][i1];
      const float q0 = W.dh1[e][i0], q1 = W.dh1[e][i1];
      gb1[0] += q0;
      gb1[1] += q1;
#pragma unroll
      for (int f = 0; f < MLP_F; ++f) {
        gw1[f][0] += W.x[e][f] * q0;
        gw1[f][1] += W.x[e][f] * q1;
      }
    }
    // dW2[i][j] = sum_e h1[e][i] * dh2[e][j]; this lane owns rows i0 and i1
    for (int j = 0; j < 64; ++j) {
      float s0 = 0.f, s1 = 0.f;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const float dj = W.dh2[e][j];
        s0 += W.h1[e][i0] * dj;
        s1 += W.h1[e][i1] * dj;
      }
      gW2[i0 * 64 + j] += s0;
      gW2[i1 * 64 + j] += s1;
    }
    __syncwarp();
  }
  // reduce to the global gradient
  atomicAdd(grad + OFF_B1 + i0, gb1[0]);
  atomicAdd(grad + OFF_B1 + i1, gb1[1]);
  atomicAdd(grad + OFF_B2 + i0, gb2[0]);
  atomicAdd(grad + OFF_B2 + i1, gb2[1]);
  atomicAdd(grad + OFF_W3 + i0, gw3[0]);
  atomicAdd(grad + OFF_W3 + i1, gw3[1]);
#pragma unroll
  for (int f = 0; f < MLP_F; ++f) {
    atomicAdd(grad + OFF_W1 + f * MLP_H + i0, gw1[f][0]);
    atomicAdd(grad + OFF_W1 + f * MLP_H + i1, gw1[f][1]);
  }
  if (lane == 0) atomicAdd(grad + OFF_B3, gb3);
  for (int q = lane; q < 64 * 64; q += 32) atomicAdd(grad + OFF_W2 + q, gW2[q]);
  lsum = warp_sum(lsum);
  if (lane == 0) atomicAdd(loss, lsum);
}

__global__ void adam_kernel(float* __restrict__ P, float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                            int count, float lr, float b1, float b2, float eps, float c1, float c2, float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  if (i >= OFF_W1 + MLP_F * MLP_H && i < OFF_B1) {  // padding rows of W1 stay zero
    grad[i] = 0.f;
    return;
  }
  const float gi = grad[i] + wd * P[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  grad[i] = 0.f;
}

// Features of candidate edge (u, pool[u][s]) in the pool of the P nearest neighbours:
//   d(u,v)/s_u, s/P, rank of u in pool[v] / P (1 when absent), (x_v-x_u)/s_u, (y_v-y_u)/s_u
// with s_u = max(d(u, pool[u][P-1]), 1). Labels (optional): 1 when v follows or precedes u
// in `tour_pos` order (tour_pos[node] = position), else 0.
__global__ void edge_features_kernel(const double2* __restrict__ coords, int n, const int32_t* __restrict__ pool, int PK,
                                     DistSrc ds, const int32_t* __restrict__ tour_pos, uint32_t* __restrict__ X32,
                                     float* __restrict__ y) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * PK) return;
  const int u = (int)(e / PK), s = (int)(e - (long long)u * PK);
  const int v = pool[e];
  float f[MLP_F] = {0.f, 0.f, 0.f, 0.f, 0.f};
  float label = 0.f;
  if ((unsigned)v < (unsigned)n) {
    const int far = pool[(long long)u * PK + PK - 1];
    const float su = fmaxf((float)ds(u, (unsigned)far < (unsigned)n ? far : u), 1.f);
    int rvu = PK;
    for (int q = 0; q < PK; ++q)
      if (pool[(long long)v * PK + q] == u) {
        rvu = q;
        break;
      }
    const double2 pu = coords[u], pv = coords[v];
    f[0] = (float)ds(u, v) / su;
    f[1] = (float)s / (float)PK;
    f[2] = (float)rvu / (float)PK;
    f[3] = (float)(pv.x - pu.x) / su;
    f[4] = (float)(pv.y - pu.y) / su;
    if (tour_pos) {
      const int pu_ = tour_pos[u], pv_ = tour_pos[v];
      const int dpos = pu_ > pv_ ? pu_ - pv_ : pv_ - pu_;
      label = (dpos == 1 || dpos == n - 1) ? 1.f : 0.f;
    }
  }
  uint32_t* row = X32 + e * 8;
  row[0] = pack_bf16(f[0], f[1]);
  row[1] = pack_bf16(f[2], f[3]);
  row[2] = pack_bf16(f[4], 0.f);
#pragma unroll
  for (int q = 3; q < 8; ++q) row[q] = 0u;
  if (y) y[e] = label;
}

// Top-k of each node's pool by descending score (ties: lower pool slot first).
__global__ void select_topk_kernel(const int32_t* __restrict__ pool, const float* __restrict__ score, int n, int PK, int k,
                                   int32_t* __restrict__ out) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  const int32_t* p = pool + (long long)u * PK;
  const float* sc = score + (long long)u * PK;
  unsigned long long taken[2] = {0ull, 0ull};  // PK <= 128
  for (int r = 0; r < k; ++r) {
    int best = -1;
    float bs = 0.f;
    for (int q = 0; q < PK; ++q) {
      if (taken[q >> 6] & (1ull << (q & 63))) continue;
      const float s = sc[q];
      if (best < 0 || s > bs) {
        best = q;
        bs = s;
      }
    }
    taken[best >> 6] |= 1ull << (best & 63);
    out[(long long)u * k + r] = p[best];
  }
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_mlp_param_count(void) { return MLP_PARAMS; }

extern "C" int tspb_edge_features(const double* coords, int32_t n, const int32_t* pool, int32_t pool_k,
                                  const int32_t* dist, int64_t dist_stride, const int32_t* tour_pos, uint16_t* x,
                                  float* labels, void* stream) {
  if (n < 1 || pool_k < 1 || pool_k > 128) return TSPB_ERR_ARG;
  if (!coords || !pool || !x) return TSPB_ERR_ARG;
  DistSrc ds;
  ds.dist = dist;
  ds.stride = dist_stride;
  ds.coords = reinterpret_cast<const double2*>(coords);
  const long long total = (long long)n * pool_k;
  edge_features_kernel<<<(int)((total + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const double2*>(coords), n, pool, pool_k, ds, tour_pos, reinterpret_cast<uint32_t*>(x), labels);
  return tspb_launch_status();
}

extern "C" int tspb_mlp_infer(const float* params, const uint16_t* x, int64_t num_edges, float* logits, void* stream) {
  if (num_edges < 0) return TSPB_ERR_ARG;
  if (num_edges == 0) return TSPB_OK;
  if (!params || !x || !logits) return TSPB_ERR_ARG;
  const long long tiles = (num_edges + 15) / 16;
  const int blocks = (int)((tiles + 7) / 8) < 148 * 8 ? (int)((tiles + 7) / 8) : 148 * 8;
  mlp_infer_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      params, reinterpret_cast<const uint32_t*>(x), num_edges, logits);
  return tspb_launch_status();
}

extern "C" int tspb_mlp_train_grad(const float* params, const uint16_t* x, const float* labels, int64_t num_edges,
                                   float* grad, float* loss, void* stream) {
  if (num_edges < 0) return TSPB_ERR_ARG;
  if (num_edges == 0) return TSPB_OK;
  if (!params || !x || !labels || !grad || !loss) return TSPB_ERR_ARG;
  const size_t smem = sizeof(WarpStage) * TRAIN_WARPS + sizeof(float) * 64 * 64 * TRAIN_WARPS;
  TSPB_CUDA_CHECK(cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long tiles = (num_edges + 15) / 16;
  const long long want = (tiles + TRAIN_WARPS - 1) / TRAIN_WARPS;
  const int blocks = want < 148 ? (int)want : 148;
  mlp_train_kernel<<<blocks, TRAIN_WARPS * 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      params, reinterpret_cast<const uint32_t*>(x), labels, num_edges, (float)(1.0 / (double)num_edges), grad, loss);
  return tspb_launch_status();
}

extern "C" int tspb_mlp_adam(float* params, float* grad, float* m, float* v, int32_t step, float lr, float beta1,
                             float beta2, float eps, float weight_decay, void* stream) {
  if (step < 1 || !params || !grad || !m || !v) return TSPB_ERR_ARG;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<(MLP_PARAMS + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      params, grad, m, v, MLP_PARAMS, lr, beta1, beta2, eps, c1, c2, weight_decay);
  return tspb_launch_status();
}

extern "C" int tspb_select_topk(const int32_t* pool, const float* scores, int32_t n, int32_t pool_k, int32_t k,
                                int32_t* out, void* stream) {
  if (n < 0 || pool_k < 1 || pool_k > 128 || k < 1 || k > pool_k) return TSPB_ERR_ARG;
  if (n == 0) return TSPB_OK;
  if (!pool || !scores || !out) return TSPB_ERR_ARG;
  select_topk_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(pool, scores, n, pool_k, k, out);
  return tspb_launch_status();
}
