// Shared declarations of the 2-opt kernels (full-scan and cached variants).
#pragma once

#include "common.cuh"

namespace tspb {

struct TwoOptArgs {
  int32_t* tours;
  int num_tours;
  int n;
  DistSrc ds;
  const int32_t* cand;
  const int32_t* cand_dist;
  int k;
  long long max_iter;
  long long* stats;
  int32_t* status;
  unsigned char* ws;
  size_t ws_tour_bytes;
  size_t ws_keys_off;  // offset of the multi_move key buffer inside a tour's slice
  int arrays_in_smem;
  const int32_t* rev_off;  // cached kernel: CSR offsets of the reverse k-NN index (n + 1)
  const int32_t* rev_idx;  // cached kernel: flat entries a * k + r grouped by candidate node
  const uint32_t* cand_packed;  // scan kernel: c | d(a, c) << 16 per entry (optional)
  const int32_t* skip;          // optional device flag: non-zero makes the launch a no-op
  long long budget;             // watchdog: SM cycles a tour may run (watchdog_cycles())
  int symmetric;                // scan kernel: symmetric distances (TSPB_MODE_SYMMETRIC)
};

// Order-preserving u64 key: negative int32 gain in the high word, scan index low.
__device__ __forceinline__ unsigned long long gain_key(int gain, unsigned idx) {
  return ((unsigned long long)((unsigned)gain ^ 0x80000000u) << 32) | idx;
}
__device__ __forceinline__ int key_gain(unsigned long long key) {
  return (int)((unsigned)(key >> 32) ^ 0x80000000u);
}

constexpr unsigned long long NO_KEY = ~0ull;
constexpr unsigned NO_IDX = ~0u;

// Watchdog: a tour that has not converged after this many SM cycles (about 35 s at
// 1.9 GHz) ends with TSPB_ERR_BUDGET instead of running on. This is the default;
// tspb_set_watchdog_cycles changes the budget that later launches are given.
constexpr long long BUDGET_CYCLES = 1LL << 36;
long long watchdog_cycles();

int smem_optin();
size_t align256(size_t v);
int launch_two_opt_cached(const TwoOptArgs& a, int mode, int threads, cudaStream_t st);
size_t two_opt_cached_tour_bytes(int n, int mode);
int launch_two_opt_scan(const TwoOptArgs& a, int mode, int threads, cudaStream_t st);
size_t two_opt_scan_tour_bytes(int n, int mode);
int carveout_for(int ctas_per_sm, size_t smem_per_cta);

}  // namespace tspb
