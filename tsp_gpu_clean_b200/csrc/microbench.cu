// Roofline microbenchmarks for the 2-opt scan's two ceilings.
//
// The candidate 2-opt keeps its distance matrix (4 MB at n = 1000) resident in L2 and
// spends its time on dependent shared-memory lookups, L2 gathers and integer arithmetic,
// so neither the HBM copy rate nor the tensor-core rate bounds it. These two kernels
// measure the ceilings that do:
//
// - l2_gather_kernel: random 4-byte loads (ld.global.cg, L1 bypassed like the scan's
//   matrix gathers) from a table that fits L2, eight independent chains per thread so the
//   memory system, not latency, is the limit. Every load touches one 32-byte L2 sector.
// - int32_issue_kernel: eight independent chains of alternating add.s32 / xor.b32 per
//   thread (written in PTX so each source operation is one integer instruction), enough
//   warps per SM that issue, not dependency latency, is the limit.
//
// The host times each launch with CUDA events and divides the operations the source
// performs by the time.
#include "common.cuh"

namespace tspb {

__global__ void __launch_bounds__(256) l2_gather_kernel(const int32_t* __restrict__ table, unsigned mask, int iters,
                                                        int32_t* __restrict__ sink) {
  const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned s[8];
  int acc = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) s[c] = (tid * 8u + (unsigned)c) * 2654435761u + 12345u;
  for (int it = 0; it < iters; ++it) {
    int v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      s[c] = s[c] * 1664525u + 1013904223u;  // LCG: the next index does not wait for the load
      v[c] = __ldcg(table + ((s[c] >> 7) & mask));
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) acc += v[c];
  }
  if (acc == 0x7fffffff) sink[0] = acc;  // keeps the loads; practically never stores
}

__global__ void __launch_bounds__(256) int32_issue_kernel(int iters, int seed, int32_t* __restrict__ sink) {
  int x[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) x[c] = seed + (int)threadIdx.x * 8 + c;
  const int a = seed * 3 + 1, b = seed ^ 0x5bd1e995;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        asm volatile("add.s32 %0, %0, %1;" : "+r"(x[c]) : "r"(a));
        asm volatile("xor.b32 %0, %0, %1;" : "+r"(x[c]) : "r"(b));
      }
    }
  }
  int acc = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) acc ^= x[c];
  if (acc == 0x7fffffff) sink[0] = acc;
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_microbench_l2_gather(const int32_t* table, int64_t table_len, int32_t iters, int32_t blocks,
                                         int32_t* sink, void* stream) {
  if (!table || !sink || iters <= 0 || blocks <= 0) return TSPB_ERR_ARG;
  if (table_len <= 0 || (table_len & (table_len - 1)) != 0 || table_len > (1LL << 31)) return TSPB_ERR_ARG;
  l2_gather_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(table, (unsigned)(table_len - 1),
                                                                               iters, sink);
  return tspb_launch_status();
}

extern "C" int tspb_microbench_int32(int32_t iters, int32_t blocks, int32_t seed, int32_t* sink, void* stream) {
  if (!sink || iters <= 0 || blocks <= 0) return TSPB_ERR_ARG;
  int32_issue_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(iters, seed, sink);
  return tspb_launch_status();
}
