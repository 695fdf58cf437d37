// GRASP nearest-neighbour initial tours, one thread per row, bit-identical to the
// reference's `_nearest_neighbor_row_cpu`
// (src/algorithms/strategies/initialization/nearest_neighbor_init.py:31-99) with the
// SplitMix64 stream of src/utils/splitmix64.py:38-51:
//   - the start city is unvisited[bounded(rem)], swapped to the end of the unvisited list;
//   - each next city is the first still-unvisited candidate met by an incremental
//     Fisher-Yates shuffle of the current city's k-NN ranks (one bounded draw per rank
//     tried), else a uniform unvisited city.
// Each row needs n + (max_node + 1) + k ints of workspace (unvisited list, its inverse
// map, the shuffled ranks).
#include "common.cuh"

namespace tspb {

__device__ __forceinline__ unsigned long long splitmix64_bounded(unsigned long long& state, unsigned bound) {
  state += 0x9E3779B97F4A7C15ull;
  unsigned long long z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return ((z >> 32) * (unsigned long long)bound) >> 32;
}

__global__ void nn_init_kernel(const int32_t* __restrict__ customers, int n, const int32_t* __restrict__ cand, int cand_rows,
                               int k, const unsigned long long* __restrict__ seeds, int pop, int max_node,
                               int32_t* __restrict__ ws, int32_t* __restrict__ out) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= pop) return;
  const long long per = (long long)n + (max_node + 1) + k;
  int32_t* unv = ws + (long long)row * per;
  int32_t* pmap = unv + n;
  int32_t* order = pmap + (max_node + 1);
  int32_t* dst = out + (long long)row * n;
  for (int q = 0; q <= max_node; ++q) pmap[q] = -1;
  for (int q = 0; q < n; ++q) {
    const int c = __ldg(customers + q);
    unv[q] = c;
    pmap[c] = q;
  }
  unsigned long long st = seeds[row];
  int rem = n;
  int s = (int)splitmix64_bounded(st, (unsigned)rem);
  int cur = unv[s];
  dst[0] = cur;
  int last = rem - 1;
  int ln = unv[last];
  unv[s] = ln;
  unv[last] = cur;
  pmap[ln] = s;
  pmap[cur] = last;
  rem = last;
  for (int step = 1; step < n; ++step) {
    int chosen = -1;
    if (cur >= 0 && cur < cand_rows && k > 0) {
      for (int i = 0; i < k; ++i) order[i] = i;
      const int32_t* crow = cand + (long long)cur * k;
      for (int i = 0; i < k; ++i) {
        const int j = i + (int)splitmix64_bounded(st, (unsigned)(k - i));
        const int tmp = order[i];
        order[i] = order[j];
        order[j] = tmp;
        const int nb = __ldg(crow + order[i]);
        if (nb >= 0 && nb <= max_node) {
          const int p = pmap[nb];
          if (p >= 0 && p < rem) {
            chosen = nb;
            break;
          }
        }
      }
    }
    if (chosen < 0) chosen = unv[(int)splitmix64_bounded(st, (unsigned)rem)];
    dst[step] = chosen;
    const int p = pmap[chosen];
    last = rem - 1;
    ln = unv[last];
    unv[p] = ln;
    unv[last] = chosen;
    pmap[ln] = p;
    pmap[chosen] = last;
    rem = last;
    cur = chosen;
  }
}

// One thread per (job, row): the same procedure with customers 0..n-1 of each job, all
// jobs in one launch (the rows of every instance of a batch start together).
__global__ void nn_init_jobs_kernel(const tspb_nn_job* __restrict__ jobs, int num_jobs, int32_t* __restrict__ ws,
                                    const long long* __restrict__ ws_offsets) {
  const int j = blockIdx.y;
  if (j >= num_jobs) return;
  const tspb_nn_job J = jobs[j];
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= J.rows) return;
  const int n = J.n, k = J.k;
  if (n <= 0) return;
  const long long per = 2LL * n + k;
  int32_t* unv = ws + ws_offsets[j] + (long long)row * per;
  int32_t* pmap = unv + n;
  int32_t* order = pmap + n;
  int32_t* dst = J.out + (long long)row * n;
  for (int q = 0; q < n; ++q) {
    unv[q] = q;
    pmap[q] = q;
  }
  unsigned long long st = J.seeds[row];
  int rem = n;
  int s = (int)splitmix64_bounded(st, (unsigned)rem);
  int cur = unv[s];
  dst[0] = cur;
  int last = rem - 1;
  int ln = unv[last];
  unv[s] = ln;
  unv[last] = cur;
  pmap[ln] = s;
  pmap[cur] = last;
  rem = last;
  for (int step = 1; step < n; ++step) {
    int chosen = -1;
    if (k > 0) {
      for (int i = 0; i < k; ++i) order[i] = i;
      const int32_t* crow = J.cand + (long long)cur * k;
      for (int i = 0; i < k; ++i) {
        const int jj = i + (int)splitmix64_bounded(st, (unsigned)(k - i));
        const int tmp = order[i];
        order[i] = order[jj];
        order[jj] = tmp;
        const int nb = __ldg(crow + order[i]);
        if (nb >= 0 && nb < n) {
          const int p = pmap[nb];
          if (p >= 0 && p < rem) {
            chosen = nb;
            break;
          }
        }
      }
    }
    if (chosen < 0) chosen = unv[(int)splitmix64_bounded(st, (unsigned)rem)];
    dst[step] = chosen;
    const int p = pmap[chosen];
    last = rem - 1;
    ln = unv[last];
    unv[p] = ln;
    unv[last] = chosen;
    pmap[ln] = p;
    pmap[chosen] = last;
    rem = last;
    cur = chosen;
  }
}

// The jobs kernel with each row's unvisited list, position map and rank order in shared
// memory (16-bit entries: 4 n + 2 k bytes per row): the walk's dependent accesses become
// shared-memory accesses instead of L2/HBM round trips. One warp per (job, row): the warp
// fills the arrays, lane 0 walks exactly as nn_init_jobs_kernel does.
__global__ void __launch_bounds__(32) nn_init_jobs_smem_kernel(const tspb_nn_job* __restrict__ jobs, int num_jobs,
                                                               int stride_u16) {
  extern __shared__ __align__(16) uint16_t smu[];
  const int j = blockIdx.y;
  if (j >= num_jobs) return;
  const tspb_nn_job J = jobs[j];
  const int row = blockIdx.x;
  if (row >= J.rows) return;
  const int n = J.n, k = J.k;
  if (n <= 0) return;
  uint16_t* unv = smu;
  uint16_t* pmap = smu + stride_u16;
  uint16_t* order = pmap + stride_u16;
  for (int q = threadIdx.x; q < n; q += 32) {
    unv[q] = (uint16_t)q;
    pmap[q] = (uint16_t)q;
  }
  __syncwarp();
  if (threadIdx.x != 0) return;
  int32_t* dst = J.out + (long long)row * n;
  unsigned long long st = J.seeds[row];
  int rem = n;
  int s = (int)splitmix64_bounded(st, (unsigned)rem);
  int cur = unv[s];
  dst[0] = cur;
  int last = rem - 1;
  int ln = unv[last];
  unv[s] = (uint16_t)ln;
  unv[last] = (uint16_t)cur;
  pmap[ln] = (uint16_t)s;
  pmap[cur] = (uint16_t)last;
  rem = last;
  for (int step = 1; step < n; ++step) {
    int chosen = -1;
    if (k > 0) {
      for (int i = 0; i < k; ++i) order[i] = (uint16_t)i;
      const int32_t* crow = J.cand + (long long)cur * k;
      for (int i = 0; i < k; ++i) {
        const int jj = i + (int)splitmix64_bounded(st, (unsigned)(k - i));
        const uint16_t tmp = order[i];
        order[i] = order[jj];
        order[jj] = tmp;
        const int nb = __ldg(crow + order[i]);
        if (nb >= 0 && nb < n && (int)pmap[nb] < rem) {
          chosen = nb;
          break;
        }
      }
    }
    if (chosen < 0) chosen = unv[(int)splitmix64_bounded(st, (unsigned)rem)];
    dst[step] = chosen;
    const int p = pmap[chosen];
    last = rem - 1;
    ln = unv[last];
    unv[p] = (uint16_t)ln;
    unv[last] = (uint16_t)chosen;
    pmap[ln] = (uint16_t)p;
    pmap[chosen] = (uint16_t)last;
    rem = last;
    cur = chosen;
  }
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_nn_init_jobs(const tspb_nn_job* jobs, int32_t num_jobs, int32_t max_rows, int32_t* workspace,
                                 const int64_t* ws_offsets, void* stream) {
  if (num_jobs < 0 || max_rows < 0) return TSPB_ERR_ARG;
  if (num_jobs == 0 || max_rows == 0) return TSPB_OK;
  if (!jobs || !workspace || !ws_offsets) return TSPB_ERR_ARG;
  if (num_jobs > 65535) return TSPB_ERR_UNSUPPORTED;
  const int threads = 64;
  const dim3 grid((max_rows + threads - 1) / threads, num_jobs);
  nn_init_jobs_kernel<<<grid, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      jobs, num_jobs, workspace, reinterpret_cast<const long long*>(ws_offsets));
  return tspb_launch_status();
}

extern "C" int tspb_nn_init_jobs_smem(const tspb_nn_job* jobs, int32_t num_jobs, int32_t max_rows, int32_t max_n,
                                      int32_t max_k, void* stream) {
  if (num_jobs < 0 || max_rows < 0 || max_n < 0 || max_k < 0) return TSPB_ERR_ARG;
  if (num_jobs == 0 || max_rows == 0 || max_n == 0) return TSPB_OK;
  if (!jobs) return TSPB_ERR_ARG;
  if (num_jobs > 65535 || max_n > 65535) return TSPB_ERR_UNSUPPORTED;
  const int stride = (max_n + 7) & ~7;  // 16-byte aligned sub-arrays
  const size_t smem = (size_t)2 * (2 * (size_t)stride + (size_t)((max_k + 7) & ~7));
  if (smem > 200 * 1024) return TSPB_ERR_UNSUPPORTED;
  if (smem > 48 * 1024)
    TSPB_CUDA_CHECK(cudaFuncSetAttribute(nn_init_jobs_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  nn_init_jobs_smem_kernel<<<dim3(max_rows, num_jobs), 32, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      jobs, num_jobs, stride);
  return tspb_launch_status();
}

extern "C" int tspb_nn_init(const int32_t* customers, int32_t n, const int32_t* cand, int32_t cand_rows, int32_t k,
                            const uint64_t* seeds, int32_t pop, int32_t max_node, int32_t* workspace,
                            size_t workspace_bytes, int32_t* out, void* stream) {
  if (n < 0 || pop < 0 || k < 0 || cand_rows < 0 || max_node < -1) return TSPB_ERR_ARG;
  if (pop == 0 || n == 0) return TSPB_OK;
  if (!customers || !seeds || !out || !workspace || (k > 0 && !cand)) return TSPB_ERR_ARG;
  const size_t need = (size_t)pop * ((size_t)n + (size_t)(max_node + 1) + (size_t)k) * sizeof(int32_t);
  if (workspace_bytes < need) return TSPB_ERR_WORKSPACE;
  const int threads = 64;
  nn_init_kernel<<<(pop + threads - 1) / threads, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      customers, n, cand, cand_rows, k, reinterpret_cast<const unsigned long long*>(seeds), pop, max_node, workspace, out);
  return tspb_launch_status();
}
