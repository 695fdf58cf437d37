// Uniform random-permutation initial population, bit-identical to the reference's
// InitializationCPUPermRandom.initialize
// (src/algorithms/strategies/initialization/random_init.py:30-55): row r starts as the
// customer list and is shuffled by Fisher-Yates from the last position down to 1, position
// i swapped with position splitmix64_bounded(i + 1) of the SplitMix64 stream seeded with
// seeds[r] (src/utils/splitmix64.py:28-51).
//
// The swaps of one row form a dependent chain, so one thread performs them; the row is
// staged in shared memory when it fits (one CTA per row, coalesced load and store by the
// whole CTA). SplitMix64's state advances by a constant, so the draw of step t depends only
// on seed + (t + 1) * increment: the CTA computes all draws in parallel first, and the
// chain is left with two shared-memory accesses per step.
#include "common.cuh"

namespace tspb {

__device__ __forceinline__ unsigned splitmix64_draw(unsigned long long seed, unsigned long long step, unsigned bound) {
  unsigned long long z = seed + (step + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (unsigned)(((z >> 32) * (unsigned long long)bound) >> 32);
}

// Largest n whose row and draws (8 n bytes) are staged in shared memory.
constexpr int kRandomInitSmemN = 24 * 1024;

// CTA per row. `customers` == nullptr means 0..n-1. With n <= stage_max the row and its
// draws sit in shared memory (row[n], draw[n] ints; the launch provides 8 * stage_max
// bytes); otherwise the row is shuffled in place in `out`.
__device__ __forceinline__ void random_init_row(const int32_t* __restrict__ customers, int n, unsigned long long seed,
                                                int32_t* __restrict__ out, int* sm, int stage_max) {
  const int tid = threadIdx.x, T = blockDim.x;
  const bool staged = n <= stage_max;
  int* row = staged ? sm : out;
  int* draw = staged ? sm + n : nullptr;
  for (int p = tid; p < n; p += T) row[p] = customers ? __ldg(customers + p) : p;
  if (staged)  // step t (t = 0 for position n-1) swaps position n-1-t with draw[t]
    for (int t = tid; t < n - 1; t += T) draw[t] = (int)splitmix64_draw(seed, (unsigned long long)t, (unsigned)(n - t));
  __syncthreads();
  if (tid == 0) {
    for (int t = 0; t < n - 1; ++t) {
      const int i = n - 1 - t;
      const int j = staged ? draw[t] : (int)splitmix64_draw(seed, (unsigned long long)t, (unsigned)(i + 1));
      const int a = row[i];
      row[i] = row[j];
      row[j] = a;
    }
  }
  __syncthreads();
  if (staged)
    for (int p = tid; p < n; p += T) out[p] = row[p];
}

__global__ void random_init_kernel(const int32_t* __restrict__ customers, int n,
                                   const unsigned long long* __restrict__ seeds, int32_t* __restrict__ out,
                                   int stage_max) {
  extern __shared__ int sm[];
  const int r = blockIdx.x;
  random_init_row(customers, n, __ldg(seeds + r), out + (long long)r * n, sm, stage_max);
}

// grid (max_rows, jobs): CTA per (job, row), customers 0..n-1 of each job.
__global__ void random_init_jobs_kernel(const tspb_nn_job* __restrict__ jobs, int stage_max) {
  extern __shared__ int sm[];
  const tspb_nn_job J = jobs[blockIdx.y];
  const int r = blockIdx.x;
  if (r >= J.rows || J.n <= 0) return;
  random_init_row(nullptr, J.n, J.seeds[r], J.out + (long long)r * J.n, sm, stage_max);
}

// Rows up to this n are staged (0: none); the launch provides 8 bytes per staged city.
static int random_init_stage_max(int max_n) { return max_n <= kRandomInitSmemN ? max_n : 0; }

template <typename K>
static int set_smem(K kernel, size_t smem) {
  if (smem > 48 * 1024) TSPB_CUDA_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return TSPB_OK;
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_random_init(const uint64_t* seeds, int32_t rows, int32_t n, const int32_t* customers, int32_t* out,
                                void* stream) {
  if (rows < 0 || n < 0) return TSPB_ERR_ARG;
  if (rows == 0 || n == 0) return TSPB_OK;
  if (!seeds || !out) return TSPB_ERR_ARG;
  const int stage_max = random_init_stage_max(n);
  const size_t smem = (size_t)8 * stage_max;
  const int rc = set_smem(random_init_kernel, smem);
  if (rc != TSPB_OK) return rc;
  random_init_kernel<<<rows, 128, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      customers, n, reinterpret_cast<const unsigned long long*>(seeds), out, stage_max);
  return tspb_launch_status();
}

extern "C" int tspb_random_init_jobs(const tspb_nn_job* jobs, int32_t num_jobs, int32_t max_rows, int32_t max_n,
                                     void* stream) {
  if (num_jobs < 0 || max_rows < 0 || max_n < 0) return TSPB_ERR_ARG;
  if (num_jobs == 0 || max_rows == 0 || max_n == 0) return TSPB_OK;
  if (!jobs) return TSPB_ERR_ARG;
  if (num_jobs > 65535) return TSPB_ERR_UNSUPPORTED;
  const int stage_max = random_init_stage_max(max_n);
  const size_t smem = (size_t)8 * stage_max;
  const int rc = set_smem(random_init_jobs_kernel, smem);
  if (rc != TSPB_OK) return rc;
  random_init_jobs_kernel<<<dim3(max_rows, num_jobs), 128, smem, reinterpret_cast<cudaStream_t>(stream)>>>(jobs,
                                                                                                         stage_max);
  return tspb_launch_status();
}
