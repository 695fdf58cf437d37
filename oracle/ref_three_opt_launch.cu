// Host launchers for the reference's 3-opt grid kernels, compiled together with the
// reference's own kernel sources (three_opt_batch.cu, three_opt_multi_move.cu and the
// headers they include, where they lie in the reference checkout) by oracle/build_ref.py
// into oracle/_ref/libref3opt.so.
//
// TEST INFRASTRUCTURE ONLY: it runs the reference's code to record the golden outputs that
// pin oracle/three_opt_kernel.py (tests/golden/make_three_opt_kernel_golden.py). Nothing in
// the product links or loads it.
//
// The launch follows LocalSearchGPUThreeOpt._improve_grid (benchmark_scripts/
// experiments-and-examples/experiment-comparing-3opt-and-2opt/gpu_three_opt.py:452-537):
// one block of `block` threads per tour, dynamic shared memory of 5 ints per thread plus
// the tour and its edge costs (2 n ints, tours up to 4096 cities), an int32 distance
// matrix with stride n, open tours, one launch per pass.
#include <cuda_runtime.h>

#include "three_opt_batch.cu"
#include "three_opt_multi_move.cu"

extern "C" int ref3_passes(int multi_move, int* population, const int* distances, int n, int population_size,
                           int block, const int* candidates, int cand_k, int inner_k, int* positions, int passes) {
  if (n < 4 || n > 4096 || population_size <= 0 || block < 1 || block > 256 || passes < 0) return 1;
  if ((block & (block - 1)) != 0) return 1;
  if (cand_k > 0 && (candidates == nullptr || positions == nullptr)) return 1;
  const size_t smem = (size_t)block * 5 * sizeof(int) + (size_t)2 * n * sizeof(int);
  if (smem > 48 * 1024) return 1;
  for (int p = 0; p < passes; ++p) {
    if (multi_move)
      three_opt_multi_move_batch_kernel<<<population_size, block, smem>>>(
          population, distances, nullptr, n, n, population_size, 0, 0, 1, cand_k > 0 ? candidates : nullptr, cand_k,
          inner_k, cand_k > 0 ? positions : nullptr, nullptr);
    else
      three_opt_batch_kernel<<<population_size, block, smem>>>(
          population, distances, nullptr, n, n, population_size, 0, 0, 1, cand_k > 0 ? candidates : nullptr, cand_k,
          inner_k, cand_k > 0 ? positions : nullptr, nullptr);
    if (cudaGetLastError() != cudaSuccess) return 2;
  }
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}
