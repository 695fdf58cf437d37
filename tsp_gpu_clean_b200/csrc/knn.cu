// k-nearest-neighbour candidate table on the device, one CTA per node.
//
// out[u][0..k) = the k nodes closest to u, self excluded, ordered by (distance, node id).
// Distances come from the int32 matrix or are rebuilt from FP64 coordinates (TSPLIB
// EUC_2D). The reference builds this table on the host with argpartition + lexsort
// (src/distances/matrix.py:140-211), where a distance tie at the k-th boundary is resolved
// by NumPy's partition; this kernel resolves it by the lower node id, a fixed and
// documented policy. tspb_knn_ties also reports the rows with such a boundary tie: every
// other row is exactly the reference's, and the context's table (device.candidate_list)
// takes the reference's own host procedure for the flagged rows only.
#include "common.cuh"

namespace tspb {

constexpr int KNN_MAX_K = 64;

__device__ __forceinline__ unsigned long long knn_key(int d, int v) {
  return ((unsigned long long)(unsigned)d << 32) | (unsigned)v;
}

// Each thread keeps its own sorted top-k (ascending keys) over its strided share of the
// row; the CTA then extracts the k smallest keys by k rounds of a block-wide minimum over
// the threads' list heads.
// With `ties`, the kernel selects k + 1 keys, writes the first k and sets ties[u] when the
// k-th and (k+1)-th distances are equal (a tie at the k-th boundary).
template <int K>
__global__ void __launch_bounds__(128) knn_kernel(int n, int k, DistSrc ds, int32_t* __restrict__ out,
                                                  int32_t* __restrict__ ties = nullptr) {
  const int u = blockIdx.x;
  const int tid = threadIdx.x;
  __shared__ unsigned long long red[32];
  unsigned long long top[K];
#pragma unroll
  for (int q = 0; q < K; ++q) top[q] = ~0ull;
  for (int v = tid; v < n; v += blockDim.x) {
    if (v == u) continue;
    const unsigned long long key = knn_key(ds(u, v), v);
    if (key >= top[K - 1]) continue;
    // insertion into the sorted local list
    unsigned long long cur = key;
#pragma unroll
    for (int q = 0; q < K; ++q) {
      const unsigned long long t = top[q];
      const bool sw = cur < t;
      top[q] = sw ? cur : t;
      cur = sw ? t : cur;
    }
  }
  int head = 0;
  const int rounds = ties ? k + 1 : k;
  unsigned long long last = ~0ull;
  for (int r = 0; r < rounds; ++r) {
    unsigned long long mine = ~0ull;
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (q == head) mine = top[q];
    const unsigned long long m = block_min(mine, red);
    if (r == k) {  // the (k+1)-th key: compare distances with the k-th
      if (tid == 0) ties[u] = (m != ~0ull && (m >> 32) == (last >> 32)) ? 1 : 0;
      break;
    }
    last = m;
    if (m == ~0ull) {
      if (tid == 0) out[(long long)u * k + r] = -1;
      continue;
    }
    if (mine == m) ++head;  // keys are unique (node id in the low word)
    if (tid == 0) out[(long long)u * k + r] = (int32_t)(unsigned)(m & 0xffffffffu);
  }
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_knn(const int32_t* dist, int64_t dist_stride, const double* coords, int32_t n, int32_t k,
                        int32_t* out, void* stream) {
  if (n < 0 || k < 0 || k > KNN_MAX_K) return TSPB_ERR_ARG;
  if (n == 0 || k == 0) return TSPB_OK;
  if (!out || (!dist && !coords)) return TSPB_ERR_ARG;
  if (k > n - 1) return TSPB_ERR_ARG;
  DistSrc ds;
  ds.dist = dist;
  ds.stride = dist_stride;
  ds.coords = reinterpret_cast<const double2*>(coords);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (k <= 8) knn_kernel<8><<<n, 128, 0, st>>>(n, k, ds, out);
  else if (k <= 16) knn_kernel<16><<<n, 128, 0, st>>>(n, k, ds, out);
  else if (k <= 32) knn_kernel<32><<<n, 128, 0, st>>>(n, k, ds, out);
  else knn_kernel<64><<<n, 128, 0, st>>>(n, k, ds, out);
  return tspb_launch_status();
}

extern "C" int tspb_knn_ties(const int32_t* dist, int64_t dist_stride, const double* coords, int32_t n, int32_t k,
                             int32_t* out, int32_t* ties, void* stream) {
  if (n < 0 || k < 0 || k + 1 > KNN_MAX_K) return TSPB_ERR_ARG;
  if (n == 0 || k == 0) return TSPB_OK;
  if (!out || !ties || (!dist && !coords)) return TSPB_ERR_ARG;
  if (k > n - 1) return TSPB_ERR_ARG;
  DistSrc ds;
  ds.dist = dist;
  ds.stride = dist_stride;
  ds.coords = reinterpret_cast<const double2*>(coords);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (k + 1 <= 8) knn_kernel<8><<<n, 128, 0, st>>>(n, k, ds, out, ties);
  else if (k + 1 <= 16) knn_kernel<16><<<n, 128, 0, st>>>(n, k, ds, out, ties);
  else if (k + 1 <= 32) knn_kernel<32><<<n, 128, 0, st>>>(n, k, ds, out, ties);
  else knn_kernel<64><<<n, 128, 0, st>>>(n, k, ds, out, ties);
  return tspb_launch_status();
}
