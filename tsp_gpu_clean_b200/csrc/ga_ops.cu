// Population operators for sm_100a: tour cost, tournament selection, row gather, PMX,
// inversion mutation, stable survival ranking, permutation validation, the EUC_2D
// matrix and the candidate-distance table. Each kernel states the reference code whose
// result it reproduces bit for bit.
#include "generation.cuh"

namespace tspb {

// Warp per tour; int64 accumulation is exact, then one conversion to float64
// (evaluate_tour_cpu sums int32 gathers in float64, exact below 2^53:
// src/algorithms/strategies/evaluation/tour_cost.py:17-29).
__global__ void tour_cost_kernel(const int32_t* __restrict__ tours, int num_tours, int n, DistSrc ds,
                                 int return_to_depot, double* __restrict__ costs) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= num_tours) return;
  const int32_t* t = tours + (long long)warp * n;
  long long acc = 0;
  int bad = 0;
  for (int p = lane; p + 1 < n; p += 32) {
    const int a = __ldg(t + p), b = __ldg(t + p + 1);
    if ((unsigned)a >= (unsigned)n || (unsigned)b >= (unsigned)n) {
      bad = 1;
      continue;
    }
    acc += ds(a, b);
  }
  acc = warp_sum(acc);
  bad = __any_sync(FULL, bad);
  if (lane == 0) {
    if (return_to_depot && n > 1) {
      const int a = __ldg(t + n - 1), b = __ldg(t);
      if ((unsigned)a < (unsigned)n && (unsigned)b < (unsigned)n) acc += ds(a, b); else bad = 1;
    }
    costs[warp] = n <= 1 ? 0.0 : (bad ? __longlong_as_double(0x7ff8000000000000LL) : (double)acc);
  }
}

// Thread per parent: first argmin of fitness over the k competitors with strict `<`
// (np.argmin semantics, tournament_selection.py:125-127).
__global__ void tournament_kernel(const double* __restrict__ fitness, int pop_size, const int32_t* __restrict__ cand,
                                  int num_parents, int k, int32_t* __restrict__ winners) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= num_parents) return;
  const int32_t* c = cand + (long long)p * k;
  int best = __ldg(c);
  if ((unsigned)best >= (unsigned)pop_size) best = 0;
  double bf = __ldg(fitness + best);
  for (int q = 1; q < k; ++q) {
    const int v = __ldg(c + q);
    if ((unsigned)v >= (unsigned)pop_size) continue;
    const double f = __ldg(fitness + v);
    if (f < bf) {
      bf = f;
      best = v;
    }
  }
  winners[p] = best;
}

// CTA per output row, int4-vectorised when n is a multiple of 4.
__global__ void gather_rows_kernel(const int32_t* __restrict__ src, int src_rows, int n, const int32_t* __restrict__ rows,
                                   int32_t* __restrict__ out) {
  const int r = blockIdx.x;
  const int sr = __ldg(rows + r);
  if ((unsigned)sr >= (unsigned)src_rows) return;
  const long long s = (long long)sr * n;
  const long long d = (long long)r * n;
  if ((n & 3) == 0) {
    const int4* s4 = reinterpret_cast<const int4*>(src + s);
    int4* d4 = reinterpret_cast<int4*>(out + d);
    for (int q = threadIdx.x; q < (n >> 2); q += blockDim.x) d4[q] = __ldg(s4 + q);
  } else {
    for (int q = threadIdx.x; q < n; q += blockDim.x) out[d + q] = __ldg(src + s + q);
  }
}

// CTA per source row: dst[rows[r], :] = src[r, :] (the elite scatter-back).
__global__ void scatter_rows_kernel(const int32_t* __restrict__ src, int n, const int32_t* __restrict__ rows, int dst_rows,
                                    int32_t* __restrict__ dst) {
  const int r = blockIdx.x;
  const int dr = __ldg(rows + r);
  if ((unsigned)dr >= (unsigned)dst_rows) return;
  const long long s = (long long)r * n, d = (long long)dr * n;
  for (int q = threadIdx.x; q < n; q += blockDim.x) dst[d + q] = __ldg(src + s + q);
}

// CTA per child. Child 2q+h takes p1 = parents[2q+h], p2 = parents[2q+1-h] and the
// shared cuts; the mapping chains of values p2[c1..c2] that are not in p1[c1..c2] are
// independent, so they run one per thread (_apply_pmx, pmx_crossover.py:49-105).
__global__ void pmx_kernel(const int32_t* __restrict__ parents, int num_routes, int n,
                           const int32_t* __restrict__ cut_first, const int32_t* __restrict__ cut_second,
                           int32_t* __restrict__ children, int32_t* __restrict__ status) {
  extern __shared__ int sm[];
  int* inv_p2 = sm;        // n
  int* child = sm + n;     // n
  unsigned* in_seg = reinterpret_cast<unsigned*>(sm + 2 * n);  // (n+31)/32 words
  __shared__ int bad;
  const int row = blockIdx.x;
  const int tid = threadIdx.x, T = blockDim.x;
  const int pairs = num_routes >> 1;
  int32_t* out = children + (long long)row * n;
  if (row >= 2 * pairs) {  // odd tail copied unchanged (pmx_crossover.py:168-169)
    for (int p = tid; p < n; p += T) out[p] = __ldg(parents + (long long)row * n + p);
    if (tid == 0 && status) status[row] = 0;
    return;
  }
  const int q = row >> 1, h = row & 1;
  const int32_t* p1 = parents + (long long)(2 * q + h) * n;
  const int32_t* p2 = parents + (long long)(2 * q + 1 - h) * n;
  int c1 = __ldg(cut_first + q), c2 = __ldg(cut_second + q);
  if (c1 > c2) {
    const int tmp = c1;
    c1 = c2;
    c2 = tmp;
  }
  const int words = (n + 31) >> 5;
  if (tid == 0) bad = 0;
  for (int p = tid; p < n; p += T) {
    inv_p2[p] = -1;
    child[p] = -1;
  }
  for (int w = tid; w < words; w += T) in_seg[w] = 0u;
  __syncthreads();
  if (c1 < 0 || c2 >= n) bad = 1;
  for (int p = tid; p < n; p += T) {
    const int v2 = __ldg(p2 + p);
    const int v1 = __ldg(p1 + p);
    if ((unsigned)v2 >= (unsigned)n || (unsigned)v1 >= (unsigned)n) {
      bad = 1;
      continue;
    }
    if (atomicExch(&inv_p2[v2], p) != -1) bad = 1;
    if (p >= c1 && p <= c2) {
      child[p] = v1;
      atomicOr(&in_seg[v1 >> 5], 1u << (v1 & 31));
    }
  }
  __syncthreads();
  if (bad) {
    for (int p = tid; p < n; p += T) out[p] = __ldg(p1 + p);
    if (tid == 0 && status) status[row] = TSPB_ERR_NOT_PERMUTATION;
    return;
  }
  const int seg_len = c2 - c1 + 1;
  for (int idx = c1 + tid; idx <= c2; idx += T) {
    const int val = __ldg(p2 + idx);
    if (in_seg[val >> 5] & (1u << (val & 31))) continue;
    int pos = idx, steps = 0;
    while (pos >= c1 && pos <= c2 && steps <= seg_len) {
      pos = inv_p2[__ldg(p1 + pos)];
      ++steps;
    }
    if (pos < c1 || pos > c2) child[pos] = val;
  }
  __syncthreads();
  for (int p = tid; p < n; p += T) {
    const int v = child[p];
    out[p] = v == -1 ? __ldg(p2 + p) : v;
  }
  if (tid == 0 && status) status[row] = 0;
}

// CTA per child, Order Crossover with validated parents (order_crossover.py:52-83).
// Shared memory: child[n], in_seg, and the seen-bitmaps of p1 and p2.
__global__ void ox_kernel(const int32_t* __restrict__ parents, int num_routes, int n,
                          const int32_t* __restrict__ cut_first, const int32_t* __restrict__ cut_second,
                          int32_t* __restrict__ children, int32_t* __restrict__ status) {
  extern __shared__ int sm[];
  const int words = (n + 31) >> 5;
  int* child = sm;                                                // n
  unsigned* in_seg = reinterpret_cast<unsigned*>(sm + n);         // words
  unsigned* seen1 = in_seg + words;                               // words
  unsigned* seen2 = seen1 + words;                                // words
  __shared__ int bad;
  __shared__ int red[32];
  const int row = blockIdx.x;
  const int tid = threadIdx.x, T = blockDim.x;
  const int pairs = num_routes >> 1;
  int32_t* out = children + (long long)row * n;
  if (row >= 2 * pairs) {  // odd tail copied unchanged (order_crossover.py:167-168)
    for (int p = tid; p < n; p += T) out[p] = __ldg(parents + (long long)row * n + p);
    if (tid == 0 && status) status[row] = 0;
    return;
  }
  const int q = row >> 1, h = row & 1;
  const int32_t* p1 = parents + (long long)(2 * q + h) * n;
  const int32_t* p2 = parents + (long long)(2 * q + 1 - h) * n;
  int c1 = __ldg(cut_first + q), c2 = __ldg(cut_second + q);
  if (c1 > c2) {
    const int tmp = c1;
    c1 = c2;
    c2 = tmp;
  }
  if (tid == 0) bad = (c1 < 0 || c2 >= n) ? 1 : 0;
  for (int w = tid; w < 3 * words; w += T) in_seg[w] = 0u;
  __syncthreads();
  for (int p = tid; p < n; p += T) {
    const int v1 = __ldg(p1 + p), v2 = __ldg(p2 + p);
    if ((unsigned)v1 >= (unsigned)n || (unsigned)v2 >= (unsigned)n) {
      bad = 1;
      continue;
    }
    if (atomicOr(&seen1[v1 >> 5], 1u << (v1 & 31)) & (1u << (v1 & 31))) bad = 1;
    if (atomicOr(&seen2[v2 >> 5], 1u << (v2 & 31)) & (1u << (v2 & 31))) bad = 1;
  }
  __syncthreads();
  if (bad) {
    for (int p = tid; p < n; p += T) out[p] = __ldg(p1 + p);
    if (tid == 0 && status) status[row] = TSPB_ERR_NOT_PERMUTATION;
    return;
  }
  for (int p = c1 + tid; p <= c2; p += T) {
    const int v1 = __ldg(p1 + p);
    child[p] = v1;
    atomicOr(&in_seg[v1 >> 5], 1u << (v1 & 31));
  }
  __syncthreads();
  ox_fill(p2, n, c2, child, in_seg, red);
  __syncthreads();
  for (int p = tid; p < n; p += T) out[p] = child[p];
  if (tid == 0 && status) status[row] = 0;
}

// Thread per route: exchange of positions p1, p2 when u < rate (swap_mutation.py:94-99).
__global__ void swap_kernel(int32_t* __restrict__ routes, int num_routes, int n, const double* __restrict__ u,
                            double rate, const int32_t* __restrict__ pos1, const int32_t* __restrict__ pos2) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= num_routes) return;
  if (!(__ldg(u + r) < rate)) return;
  const int a = __ldg(pos1 + r), b = __ldg(pos2 + r);
  if ((unsigned)a >= (unsigned)n || (unsigned)b >= (unsigned)n) return;
  int32_t* t = routes + (long long)r * n;
  const int x = t[a];
  t[a] = t[b];
  t[b] = x;
}

// Warp per route, reversal of [min(p1,p2), max(p1,p2)] when u < rate
// (inversion_mutation.py:93-97).
__global__ void inversion_kernel(int32_t* __restrict__ routes, int num_routes, int n, const double* __restrict__ u,
                                 double rate, const int32_t* __restrict__ pos1, const int32_t* __restrict__ pos2) {
  const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= num_routes) return;
  if (!(__ldg(u + r) < rate)) return;
  const int a = __ldg(pos1 + r), b = __ldg(pos2 + r);
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  if (lo < 0 || hi >= n) return;
  int32_t* t = routes + (long long)r * n;
  const int half = (hi - lo + 1) >> 1;
  for (int q = lane; q < half; q += 32) {
    const int x = t[lo + q], y = t[hi - q];
    t[lo + q] = y;
    t[hi - q] = x;
  }
}

// Thread per element: rank by (value, index); ranks below `keep` scatter the index
// (a stable ascending sort, np.lexsort of genetic_algorithm.py:682-689).
__global__ void stable_rank_kernel(const double* __restrict__ f, int count, int keep, int32_t* __restrict__ order) {
  __shared__ double tile[1024];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double fi = i < count ? f[i] : 0.0;
  int rank = 0;
  for (int base = 0; base < count; base += blockDim.x) {
    const int j = base + threadIdx.x;
    if (j < count) tile[threadIdx.x] = f[j];
    __syncthreads();
    const int lim = min((int)blockDim.x, count - base);
    if (i < count) {
      for (int q = 0; q < lim; ++q) {
        const double fj = tile[q];
        const int jj = base + q;
        rank += (fj < fi) || (fj == fi && jj < i);
      }
    }
    __syncthreads();
  }
  if (i < count && rank < keep) order[rank] = i;
}

__global__ void validate_perm_kernel(const int32_t* __restrict__ tours, int n, int32_t* __restrict__ bad_out) {
  extern __shared__ unsigned seen[];
  __shared__ int bad;
  const int r = blockIdx.x;
  const int words = (n + 31) >> 5;
  if (threadIdx.x == 0) bad = 0;
  for (int w = threadIdx.x; w < words; w += blockDim.x) seen[w] = 0u;
  __syncthreads();
  const int32_t* t = tours + (long long)r * n;
  for (int p = threadIdx.x; p < n; p += blockDim.x) {
    const int v = __ldg(t + p);
    if ((unsigned)v >= (unsigned)n) {
      bad = 1;
      continue;
    }
    const unsigned bit = 1u << (v & 31);
    if (atomicOr(&seen[v >> 5], bit) & bit) bad = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) bad_out[r] = bad;
}

__global__ void euc2d_matrix_kernel(const double2* __restrict__ coords, int n, int32_t* __restrict__ dist, long long stride) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y;
  if (c >= n) return;
  dist[(long long)a * stride + c] = a == c ? 0 : euc2d(__ldg(coords + a), __ldg(coords + c));
}

__global__ void cand_dist_kernel(const int32_t* __restrict__ cand, int n, int k, DistSrc ds, int32_t* __restrict__ out) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * k) return;
  const int a = (int)(e / k);
  const int c = __ldg(cand + e);
  out[e] = (unsigned)c < (unsigned)n ? ds(a, c) : 0;
}

}  // namespace tspb

using namespace tspb;

static DistSrc make_ds(const int32_t* dist, int64_t stride, const double* coords) {
  DistSrc d;
  d.dist = dist;
  d.stride = stride;
  d.coords = reinterpret_cast<const double2*>(coords);
  return d;
}

extern "C" int tspb_tour_cost(const int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                              const double* coords, int32_t return_to_depot, double* costs, void* stream) {
  if (num_tours < 0 || n < 0) return TSPB_ERR_ARG;
  if (num_tours == 0) return TSPB_OK;
  if (costs == nullptr || (n > 0 && tours == nullptr) || (dist == nullptr && coords == nullptr)) return TSPB_ERR_ARG;
  const int threads = 256;
  const long long warps = num_tours;
  const int blocks = (int)((warps * 32 + threads - 1) / threads);
  tour_cost_kernel<<<blocks, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      tours, num_tours, n, make_ds(dist, dist_stride, coords), return_to_depot, costs);
  return tspb_launch_status();
}

extern "C" int tspb_tournament(const double* fitness, int32_t pop_size, const int32_t* cand, int32_t num_parents, int32_t k,
                               int32_t* winners, void* stream) {
  if (num_parents < 0 || k < 1 || pop_size < 1) return TSPB_ERR_ARG;
  if (num_parents == 0) return TSPB_OK;
  if (!fitness || !cand || !winners) return TSPB_ERR_ARG;
  tournament_kernel<<<(num_parents + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      fitness, pop_size, cand, num_parents, k, winners);
  return tspb_launch_status();
}

extern "C" int tspb_gather_rows(const int32_t* src, int32_t src_rows, int32_t n, const int32_t* rows, int32_t num_rows,
                                int32_t* out, void* stream) {
  if (num_rows < 0 || n < 0 || src_rows < 0) return TSPB_ERR_ARG;
  if (num_rows == 0 || n == 0) return TSPB_OK;
  if (!src || !rows || !out) return TSPB_ERR_ARG;
  gather_rows_kernel<<<num_rows, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(src, src_rows, n, rows, out);
  return tspb_launch_status();
}

extern "C" int tspb_scatter_rows(const int32_t* src, int32_t num_rows, int32_t n, const int32_t* rows, int32_t* dst,
                                 int32_t dst_rows, void* stream) {
  if (num_rows < 0 || n < 0 || dst_rows < 0) return TSPB_ERR_ARG;
  if (num_rows == 0 || n == 0) return TSPB_OK;
  if (!src || !rows || !dst) return TSPB_ERR_ARG;
  scatter_rows_kernel<<<num_rows, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(src, n, rows, dst_rows, dst);
  return tspb_launch_status();
}

extern "C" int tspb_pmx(const int32_t* parents, int32_t num_routes, int32_t n, const int32_t* cut_first,
                        const int32_t* cut_second, int32_t* children, int32_t* status, void* stream) {
  if (num_routes < 0 || n < 0) return TSPB_ERR_ARG;
  if (num_routes == 0 || n == 0) return TSPB_OK;
  if (!parents || !children || (num_routes >= 2 && (!cut_first || !cut_second))) return TSPB_ERR_ARG;
  const size_t smem = (size_t)8 * n + (size_t)((n + 31) / 32) * 4;
  if (smem > 200 * 1024) return TSPB_ERR_UNSUPPORTED;
  if (smem > 48 * 1024) TSPB_CUDA_CHECK(cudaFuncSetAttribute(pmx_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int threads = n >= 1024 ? 512 : (n >= 256 ? 256 : 128);
  pmx_kernel<<<num_routes, threads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(parents, num_routes, n, cut_first,
                                                                                    cut_second, children, status);
  return tspb_launch_status();
}

extern "C" int tspb_ox(const int32_t* parents, int32_t num_routes, int32_t n, const int32_t* cut_first,
                       const int32_t* cut_second, int32_t* children, int32_t* status, void* stream) {
  if (num_routes < 0 || n < 0) return TSPB_ERR_ARG;
  if (num_routes == 0 || n == 0) return TSPB_OK;
  if (!parents || !children || (num_routes >= 2 && (!cut_first || !cut_second))) return TSPB_ERR_ARG;
  const size_t smem = (size_t)4 * n + (size_t)3 * ((n + 31) / 32) * 4;
  if (smem > 200 * 1024) return TSPB_ERR_UNSUPPORTED;
  if (smem > 48 * 1024) TSPB_CUDA_CHECK(cudaFuncSetAttribute(ox_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int threads = n >= 1024 ? 512 : (n >= 256 ? 256 : 128);
  ox_kernel<<<num_routes, threads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(parents, num_routes, n, cut_first,
                                                                                   cut_second, children, status);
  return tspb_launch_status();
}

extern "C" int tspb_swap(int32_t* routes, int32_t num_routes, int32_t n, const double* u, double rate,
                         const int32_t* pos1, const int32_t* pos2, void* stream) {
  if (num_routes < 0 || n < 0) return TSPB_ERR_ARG;
  if (num_routes == 0 || n == 0) return TSPB_OK;
  if (!routes || !u || !pos1 || !pos2) return TSPB_ERR_ARG;
  const int threads = 128;
  swap_kernel<<<(num_routes + threads - 1) / threads, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      routes, num_routes, n, u, rate, pos1, pos2);
  return tspb_launch_status();
}

extern "C" int tspb_inversion(int32_t* routes, int32_t num_routes, int32_t n, const double* u, double rate,
                              const int32_t* pos1, const int32_t* pos2, void* stream) {
  if (num_routes < 0 || n < 0) return TSPB_ERR_ARG;
  if (num_routes == 0 || n == 0) return TSPB_OK;
  if (!routes || !u || !pos1 || !pos2) return TSPB_ERR_ARG;
  const int threads = 256;
  const int blocks = (int)(((long long)num_routes * 32 + threads - 1) / threads);
  inversion_kernel<<<blocks, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(routes, num_routes, n, u, rate, pos1, pos2);
  return tspb_launch_status();
}

extern "C" int tspb_stable_rank(const double* fitness, int32_t count, int32_t keep, int32_t* order, void* stream) {
  if (count < 0 || keep < 0 || keep > count) return TSPB_ERR_ARG;
  if (count == 0 || keep == 0) return TSPB_OK;
  if (!fitness || !order) return TSPB_ERR_ARG;
  const int threads = 256;
  stable_rank_kernel<<<(count + threads - 1) / threads, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(fitness, count,
                                                                                                               keep, order);
  return tspb_launch_status();
}

extern "C" int tspb_validate_perm(const int32_t* tours, int32_t num_tours, int32_t n, int32_t* bad, void* stream) {
  if (num_tours < 0 || n < 0) return TSPB_ERR_ARG;
  if (num_tours == 0) return TSPB_OK;
  if (!bad || (n > 0 && !tours)) return TSPB_ERR_ARG;
  const size_t smem = (size_t)((n + 31) / 32) * 4;
  if (smem > 200 * 1024) return TSPB_ERR_UNSUPPORTED;
  if (smem > 48 * 1024)
    TSPB_CUDA_CHECK(cudaFuncSetAttribute(validate_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  validate_perm_kernel<<<num_tours, 256, smem, reinterpret_cast<cudaStream_t>(stream)>>>(tours, n, bad);
  return tspb_launch_status();
}

extern "C" int tspb_euc2d_matrix(const double* coords, int32_t n, int32_t* dist, int64_t dist_stride, void* stream) {
  if (n < 0 || dist_stride < n) return TSPB_ERR_ARG;
  if (n == 0) return TSPB_OK;
  if (!coords || !dist) return TSPB_ERR_ARG;
  if (n > 65535) return TSPB_ERR_UNSUPPORTED;
  dim3 grid((n + 255) / 256, n);
  euc2d_matrix_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const double2*>(coords), n,
                                                                                  dist, dist_stride);
  return tspb_launch_status();
}

extern "C" int tspb_candidate_distances(const int32_t* cand, int32_t n, int32_t k, const int32_t* dist, int64_t dist_stride,
                                        const double* coords, int32_t* cand_dist, void* stream) {
  if (n < 0 || k < 0) return TSPB_ERR_ARG;
  if (n == 0 || k == 0) return TSPB_OK;
  if (!cand || !cand_dist || (dist == nullptr && coords == nullptr)) return TSPB_ERR_ARG;
  const long long total = (long long)n * k;
  cand_dist_kernel<<<(int)((total + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      cand, n, k, make_ds(dist, dist_stride, coords), cand_dist);
  return tspb_launch_status();
}

extern "C" int tspb_version(void) { return 100; }

extern "C" const char* tspb_status_string(int status) {
  switch (status) {
    case TSPB_OK: return "ok";
    case TSPB_ERR_ARG: return "invalid argument";
    case TSPB_ERR_CUDA: return "CUDA launch or runtime error";
    case TSPB_ERR_NOT_PERMUTATION: return "input tour is not a permutation of 0..n-1";
    case TSPB_ERR_RANGE: return "value outside the kernel's integer range";
    case TSPB_ERR_UNSUPPORTED: return "unsupported configuration";
    case TSPB_ERR_WORKSPACE: return "workspace too small";
    case TSPB_ERR_BUDGET: return "device watchdog expired before convergence";
    case TSPB_ERR_DEVICE_MEMORY: return "the device could not provide memory held by the library";
    default: return "unknown status";
  }
}
