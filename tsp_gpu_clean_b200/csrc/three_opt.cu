// Exhaustive steepest-descent 3-opt on open (cyclic TSP) tours, bit-identical to the
// reference's CPU 3-opt (cpu_three_opt_best_move / cpu_three_opt_refine of its 3-opt
// experiment, benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/
// gpu_three_opt.py:143-277):
//   - cuts 0 <= i < j < k <= n-1 remove (t[i], t[i+1]), (t[j], t[j+1]), (t[k], t[(k+1) % n]);
//   - scan order i, j, then the pure 2-opt case 1 at k = j (j > i + 1), then k ascending with
//     cases 2..7; case 2 needs k > j + 1, case 3 is skipped for i = 0, k = n - 1;
//   - the move applied is the first in scan order with the smallest negative delta, i.e.
//     the minimum of (delta, key) with key = ((i n + j) n + k) 8 + case;
//   - a move is up to three reversals: [i+1, j] (cases 1, 4, 5, 7), [j+1, k] (2, 4, 5, 6),
//     [i+1, k] (3, 5, 6, 7).
//
// Layout: one CTA per tour (persistent over tours). Each pass first builds the tour-ordered
// matrix M[p][q] = d(t[p], t[q]) (n^2 gathers, under 1 % of the n^3/6 triples of a pass), so
// that the six distances of a triple are coalesced reads of the rows M[i], M[i+1], M[j],
// M[j+1] at columns k and k+1. M lives in shared memory for n <= kThreeOptSmemN, else in a
// per-CTA HBM workspace (L1/L2-resident rows). Warps take (i, j) rows of the scan, lanes
// stride over k; deltas are int64 (three distances below 2^30 each).
#include "common.cuh"
#include "two_opt.cuh"

namespace tspb {

constexpr int kThreeOptSmemN = 220;  // 4 n^2 + 12 n bytes of shared memory at most ~190 KB
constexpr int kThreeOptMaxN = 4096;
constexpr unsigned long long kNoKey = ~0ull;

struct MoveKey {
  long long delta;
  unsigned long long key;
};

__device__ __forceinline__ void consider(MoveKey& m, long long delta, unsigned long long key) {
  if (delta < 0 && (delta < m.delta || (delta == m.delta && key < m.key))) {
    m.delta = delta;
    m.key = key;
  }
}

__device__ __forceinline__ MoveKey warp_min_move(MoveKey m) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long od = __shfl_xor_sync(FULL, m.delta, o);
    const unsigned long long ok = __shfl_xor_sync(FULL, m.key, o);
    if (od < m.delta || (od == m.delta && ok < m.key)) {
      m.delta = od;
      m.key = ok;
    }
  }
  return m;
}

// Reverse tour[lo..hi] with the whole CTA.
__device__ __forceinline__ void reverse_segment(int* tour, int lo, int hi) {
  const int half = (hi - lo + 1) >> 1;
  for (int t = threadIdx.x; t < half; t += blockDim.x) {
    const int x = tour[lo + t], y = tour[hi - t];
    tour[lo + t] = y;
    tour[hi - t] = x;
  }
  __syncthreads();
}

template <bool SMEM_M>
__global__ void __launch_bounds__(512) three_opt_kernel(int32_t* __restrict__ tours, int num_tours, int n, DistSrc ds,
                                                        long long max_iter, int32_t* __restrict__ workspace,
                                                        int32_t* __restrict__ status, long long* __restrict__ stats,
                                                        long long budget) {
  extern __shared__ __align__(16) int sm3[];
  int* tour = sm3;                                      // n
  long long* edge = reinterpret_cast<long long*>(sm3 + ((n + 1) & ~1));  // n int64
  int* M = SMEM_M ? reinterpret_cast<int*>(edge + n) : workspace + (long long)blockIdx.x * n * n;
  __shared__ MoveKey warp_best[32];
  __shared__ MoveKey cta_best;
  __shared__ unsigned long long ev_sum;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = (int)(blockDim.x >> 5);
  const int kmax = n - 1;
  const long long pairs = n >= 4 ? (long long)(n - 2) * (n - 1) / 2 : 0;  // (i, j) rows: i <= n-3, i < j <= n-2
  for (int r = blockIdx.x; r < num_tours; r += gridDim.x) {
    int32_t* g = tours + (long long)r * n;
    for (int p = tid; p < n; p += blockDim.x) tour[p] = g[p];
    __syncthreads();
    long long passes = 0, moves = 0, evaluated = 0;
    int code = 0;
    const long long start = clock64();
    for (long long it = 0; it < max_iter && n >= 4; ++it) {
      if (clock64() - start > budget) {  // the watchdog of the 2-opt kernels (uniform per CTA)
        code = TSPB_ERR_BUDGET;
        break;
      }
      // tour-ordered matrix (warp per row, coalesced stores) and edge lengths
      for (int p = wid; p < n; p += nw) {
        const int a = tour[p];
        int* row = M + (long long)p * n;
        for (int c = lane; c < n; c += 32) row[c] = ds(a, tour[c]);
      }
      __syncthreads();
      for (int p = tid; p < n; p += blockDim.x) edge[p] = M[(long long)p * n + (p + 1 == n ? 0 : p + 1)];
      __syncthreads();
      MoveKey best{0, kNoKey};
      long long ev = 0;
      for (long long t = wid; t < pairs; t += nw) {
        // row t of the scan -> (i, j): row i holds j = i+1 .. n-2, i.e. n-2-i pairs
        int i = 0;
        {
          // off(i) = i (n-2) - i (i-1) / 2 pairs precede row i; binary search the last off(i) <= t
          int lo = 0, hi = n - 3;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            const long long off = (long long)mid * (n - 2) - (long long)mid * (mid - 1) / 2;
            if (off <= t) lo = mid; else hi = mid - 1;
          }
          i = lo;
        }
        const long long off_i = (long long)i * (n - 2) - (long long)i * (i - 1) / 2;
        const int j = i + 1 + (int)(t - off_i);
        const int* Ra = M + (long long)i * n;
        const int* Rb = M + (long long)(i + 1) * n;
        const int* Rc = M + (long long)j * n;
        const int* Rd = M + (long long)(j + 1) * n;
        const long long dab = edge[i], dcd = edge[j];
        const long long dac = Ra[j], dad = Ra[j + 1], dbd = Rb[j + 1];
        const unsigned long long base = ((unsigned long long)i * n + j) * n;
        if (lane == 0 && j > i + 1) {
          consider(best, dac + dbd - dab - dcd, (base + j) * 8ull + 1ull);
          ++ev;
        }
        for (int k = j + 1 + lane; k <= kmax; k += 32) {
          const int kp = k + 1 == n ? 0 : k + 1;
          const long long def = edge[k];
          const long long old3 = dab + dcd + def;
          const long long dce = Rc[k], ddf = Rd[kp], dae = Ra[k], dbf = Rb[kp], dbe = Rb[k], dcf = Rc[kp];
          const unsigned long long key = (base + k) * 8ull;
          if (k > j + 1) consider(best, dce + ddf - dcd - def, key + 2);
          if (!(i == 0 && k == n - 1)) consider(best, dae + dbf - dab - def, key + 3);
          consider(best, dac + dbe + ddf - old3, key + 4);
          consider(best, dad + dbe + dcf - old3, key + 5);
          consider(best, dad + dce + dbf - old3, key + 6);
          consider(best, dae + dbd + dcf - old3, key + 7);
          ev += 4 + (k > j + 1) + !(i == 0 && k == n - 1);
        }
      }
      best = warp_min_move(best);
      ev = warp_sum(ev);
      if (lane == 0) warp_best[wid] = best;
      if (tid == 0) ev_sum = 0;
      __syncthreads();
      if (lane == 0) atomicAdd(&ev_sum, (unsigned long long)ev);
      if (tid == 0) {
        MoveKey b = warp_best[0];
        for (int w = 1; w < nw; ++w) {
          const MoveKey o = warp_best[w];
          if (o.delta < b.delta || (o.delta == b.delta && o.key < b.key)) b = o;
        }
        cta_best = b;
      }
      __syncthreads();
      evaluated += (long long)ev_sum;
      ++passes;
      const MoveKey b = cta_best;
      if (b.key == kNoKey) break;  // no improving move: a 3-opt local optimum
      const int kase = (int)(b.key & 7ull);
      const unsigned long long ijk = b.key >> 3;
      const int k = (int)(ijk % (unsigned long long)n);
      const int j = (int)((ijk / (unsigned long long)n) % (unsigned long long)n);
      const int i = (int)(ijk / ((unsigned long long)n * n));
      if (kase == 1 || kase == 4 || kase == 5 || kase == 7) reverse_segment(tour, i + 1, j);
      if (kase == 2 || kase == 4 || kase == 5 || kase == 6) reverse_segment(tour, j + 1, k);
      if (kase == 3 || kase == 5 || kase == 6 || kase == 7) reverse_segment(tour, i + 1, k);
      ++moves;
      __syncthreads();
    }
    for (int p = tid; p < n; p += blockDim.x) g[p] = tour[p];
    if (tid == 0) {
      if (status) status[r] = code;
      if (stats) {
        stats[(long long)r * 3 + 0] = passes;
        stats[(long long)r * 3 + 1] = moves;
        stats[(long long)r * 3 + 2] = evaluated;
      }
    }
    __syncthreads();
  }
}

static size_t three_opt_smem(int n, bool smem_m) {
  const size_t base = (size_t)4 * ((n + 1) & ~1) + (size_t)8 * n;
  return base + (smem_m ? (size_t)4 * n * n : 0);
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_three_opt_workspace_bytes(int32_t n, int32_t ctas, size_t* bytes) {
  if (n < 0 || ctas < 0 || !bytes) return TSPB_ERR_ARG;
  *bytes = n <= kThreeOptSmemN ? 0 : (size_t)ctas * n * n * sizeof(int32_t);
  return TSPB_OK;
}

extern "C" int tspb_three_opt(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                              const double* coords, int64_t max_iterations, int32_t threads, int32_t* workspace,
                              size_t workspace_bytes, int32_t* status, int64_t* stats, void* stream) {
  if (num_tours < 0 || n < 0 || max_iterations < 0) return TSPB_ERR_ARG;
  if (num_tours == 0 || n == 0) return TSPB_OK;
  if (!tours || (!dist && !coords) || (dist && dist_stride < n)) return TSPB_ERR_ARG;
  if (threads != 128 && threads != 256 && threads != 512) return TSPB_ERR_ARG;
  // one exhaustive pass is n^3 / 6 triples on one CTA; the watchdog runs between passes,
  // so n is capped where a pass stays around a second
  if (n > kThreeOptMaxN) return TSPB_ERR_UNSUPPORTED;
  DistSrc ds;
  ds.dist = dist;
  ds.stride = dist_stride;
  ds.coords = reinterpret_cast<const double2*>(coords);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const bool smem_m = n <= kThreeOptSmemN;
  const size_t smem = three_opt_smem(n, smem_m);
  if (smem > (size_t)smem_optin() - 1024) return TSPB_ERR_UNSUPPORTED;
  int ctas = num_tours;
  if (!smem_m) {
    const size_t per = (size_t)n * n * sizeof(int32_t);
    if (!workspace || workspace_bytes < per) return TSPB_ERR_WORKSPACE;
    const size_t fit = workspace_bytes / per;
    if ((size_t)ctas > fit) ctas = (int)fit;
  }
  if (smem_m) {
    TSPB_CUDA_CHECK(cudaFuncSetAttribute(three_opt_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    three_opt_kernel<true><<<ctas, threads, smem, st>>>(tours, num_tours, n, ds, max_iterations, nullptr, status,
                                                        reinterpret_cast<long long*>(stats), watchdog_cycles());
  } else {
    if (smem > 48 * 1024)
      TSPB_CUDA_CHECK(cudaFuncSetAttribute(three_opt_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    three_opt_kernel<false><<<ctas, threads, smem, st>>>(tours, num_tours, n, ds, max_iterations, workspace, status,
                                                         reinterpret_cast<long long*>(stats), watchdog_cycles());
  }
  return tspb_launch_status();
}
