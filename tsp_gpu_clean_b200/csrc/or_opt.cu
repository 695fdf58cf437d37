// Candidate-list Or-opt, best improvement, one CTA per tour (persistent over tours).
//
// The reference has no Or-opt strategy; this operator widens its local-search family next
// to the candidate 2-opt (src/algorithms/strategies/local_search/two_opt.py:347-367: k-NN
// candidates, open cyclic tours with position 0 fixed, exact integer deltas, the first move
// in scan order among equal gains). A move (i, L, r, o) relocates the segment
// S = t[i .. i+L-1] (1 <= L <= max_segment, i >= 1) between c and its successor e, forward
// (o = 0, c = N[t[i]][r]) or reversed (o = 1, L >= 2, c = N[t[i+L-1]][r]); it is valid when
// pos[c] lies outside [i-1, i+L-1]. With p = t[i-1], q = t[(i+L) % n] and (x, y) = (s0, sl)
// forward or (sl, s0) reversed:
//   delta = d(p,q) - d(p,s0) - d(sl,q) + d(x,c) + d(y,e) - d(c,e)
// A pass applies the smallest negative delta, the smallest key
// (((i-1) * max_segment + (L-1)) * k + r) * 2 + o among equal deltas.
//
// Layout: tour[p], pos[a], eout[a] = d(a, succ a) and a rebuild buffer in shared memory
// (16 n bytes). A thread evaluates four consecutive candidates of one (i, L, o): the
// candidate ids and d(x, c) come from the k-NN table and its distance table (PACKED: one
// 16-byte load of four c | d << 16 words), pos, the successor and eout from shared memory,
// and d(y, e) is the only gather per entry. The move rewrites only the positions between the
// segment and the insertion point.
#include "common.cuh"
#include "two_opt.cuh"

namespace tspb {

struct OrMove {
  long long delta;
  unsigned long long key;
};

__device__ __forceinline__ bool or_less(const OrMove& a, const OrMove& b) {
  return a.delta < b.delta || (a.delta == b.delta && a.key < b.key);
}

__device__ __forceinline__ OrMove warp_min_or(OrMove m) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    OrMove w;
    w.delta = __shfl_xor_sync(FULL, m.delta, o);
    w.key = __shfl_xor_sync(FULL, m.key, o);
    if (or_less(w, m)) m = w;
  }
  return m;
}

// Block-wide lexicographic minimum; sh holds 33 entries. Every thread gets the result.
__device__ __forceinline__ OrMove block_min_or(OrMove m, OrMove* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  m = warp_min_or(m);
  if (lane == 0) sh[wid] = m;
  __syncthreads();
  if (wid == 0) {
    OrMove v{0, NO_KEY};
    if (lane < nw) v = sh[lane];
    v = warp_min_or(v);
    if (lane == 0) sh[32] = v;
  }
  __syncthreads();
  const OrMove r = sh[32];
  __syncthreads();  // sh is reused by the next call
  return r;
}

template <int THREADS, bool PACKED>
__global__ void __launch_bounds__(THREADS) or_opt_kernel(int32_t* __restrict__ tours, int num, int n, DistSrc ds,
                                                         const int32_t* __restrict__ cand,
                                                         const int32_t* __restrict__ cdist,
                                                         const uint32_t* __restrict__ packed, int k, int S,
                                                         long long max_iter, int32_t* __restrict__ status,
                                                         long long* __restrict__ stats, long long budget) {
  extern __shared__ __align__(16) int sm[];
  __shared__ OrMove red[33];
  __shared__ long long redll[32];
  __shared__ int s_flag;
  int* tour = sm;
  int* pos = tour + n;
  int* eout = pos + n;
  int* tmp = eout + n;
  const int tid = threadIdx.x;
  const int chunks = (k + 3) >> 2;
  const int items = (n - 1) * S * 2 * chunks;  // (i-1, L-1, o) groups x four-candidate chunks
  for (int t = blockIdx.x; t < num; t += gridDim.x) {
    int32_t* g = tours + (long long)t * n;
    if (tid == 0) s_flag = 0;
    for (int p = tid; p < n; p += THREADS) {
      tour[p] = g[p];
      pos[p] = -1;
    }
    __syncthreads();
    for (int p = tid; p < n; p += THREADS) {
      const int v = tour[p];
      if ((unsigned)v >= (unsigned)n || atomicExch(&pos[v], p) != -1) s_flag = 1;
    }
    __syncthreads();
    if (s_flag) {
      if (tid == 0) {
        status[t] = TSPB_ERR_NOT_PERMUTATION;
        if (stats)
          for (int q = 0; q < 3; ++q) stats[(long long)t * 3 + q] = 0;
      }
      __syncthreads();  // every thread has read s_flag before it is reset
      continue;
    }
    for (int p = tid; p < n; p += THREADS) {
      const int a = tour[p];
      eout[a] = ds(a, tour[p + 1 == n ? 0 : p + 1]);
    }
    long long passes = 0, moves = 0, my_eval = 0;
    int err = TSPB_OK;
    const long long t0 = clock64();
    while (passes < max_iter) {
      __syncthreads();  // the state of the last move (or the setup) is visible
      if (tid == 0) s_flag = clock64() - t0 > budget;
      __syncthreads();
      if (s_flag) {
        err = TSPB_ERR_BUDGET;
        break;
      }
      OrMove m{0, NO_KEY};
      for (int it = tid; it < items; it += THREADS) {
        const int grp = it / chunks, ch = it - grp * chunks;
        const int o = grp & 1, il = grp >> 1;
        const int L = il % S + 1, i = il / S + 1;
        if (i + L - 1 > n - 1 || (o == 1 && L < 2)) continue;
        const int s0 = tour[i], sl = tour[i + L - 1], p = tour[i - 1], q = tour[i + L == n ? 0 : i + L];
        const int x = o ? sl : s0, y = o ? s0 : sl;
        const long long base = (long long)ds(p, q) - eout[p] - eout[sl];
        const int r0 = ch * 4;
        int c[4], dxc[4], e[4], dye[4];
        bool ok[4];
        if constexpr (PACKED) {  // k % 4 == 0: the four entries exist and are 16-byte aligned
          const uint4 w = __ldg(reinterpret_cast<const uint4*>(packed + (long long)x * k + r0));
          const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            ok[u] = true;
            c[u] = (int)(ws[u] & 0xffffu);
            dxc[u] = (int)(ws[u] >> 16);
          }
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            ok[u] = r0 + u < k;
            if (ok[u]) {
              const long long at = (long long)x * k + r0 + u;
              c[u] = __ldg(cand + at);
              dxc[u] = __ldg(cdist + at);
            }
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (!ok[u]) continue;
          if ((unsigned)c[u] >= (unsigned)n) {
            ok[u] = false;
            continue;
          }
          const int j = pos[c[u]];
          ok[u] = j < i - 1 || j > i + L - 1;
          if (ok[u]) e[u] = tour[j + 1 == n ? 0 : j + 1];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (ok[u]) dye[u] = ds(y, e[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (!ok[u]) continue;
          ++my_eval;
          const long long d = base + dxc[u] + dye[u] - eout[c[u]];
          if (d < 0) {
            const OrMove v{d, ((((unsigned long long)(i - 1) * S + (L - 1)) * k + (r0 + u)) << 1) | (unsigned)o};
            if (or_less(v, m)) m = v;
          }
        }
      }
      ++passes;
      const OrMove b = block_min_or(m, red);
      if (b.key == NO_KEY) break;  // a local optimum
      const int bo = (int)(b.key & 1);
      const unsigned long long rest = b.key >> 1;
      const int br = (int)(rest % (unsigned long long)k);
      const unsigned long long bil = rest / (unsigned long long)k;
      const int bL = (int)(bil % (unsigned long long)S) + 1, bi = (int)(bil / (unsigned long long)S) + 1;
      const int bx = bo ? tour[bi + bL - 1] : tour[bi];
      const int bc = __ldg(cand + (long long)bx * k + br);
      if ((unsigned)bc >= (unsigned)n) {  // cannot happen for a scanned move; uniform across the CTA
        err = TSPB_ERR_RANGE;
        break;
      }
      const int bj = pos[bc];
      if (bj >= bi - 1 && bj <= bi + bL - 1) {
        err = TSPB_ERR_RANGE;
        break;
      }
      const bool case_a = bj > bi + bL - 1;
      const int lo = case_a ? bi : bj + 1, hi = case_a ? bj : bi + bL - 1;
      for (int np = lo + tid; np <= hi; np += THREADS) {
        int v;
        if (case_a) {
          if (np <= bj - bL) {
            v = tour[np + bL];
          } else {
            const int mm = np - (bj - bL + 1);
            v = bo ? tour[bi + bL - 1 - mm] : tour[bi + mm];
          }
        } else {
          if (np <= bj + bL) {
            const int mm = np - (bj + 1);
            v = bo ? tour[bi + bL - 1 - mm] : tour[bi + mm];
          } else {
            v = tour[np - bL];
          }
        }
        tmp[np] = v;
      }
      __syncthreads();
      for (int np = lo + tid; np <= hi; np += THREADS) {
        const int v = tmp[np];
        tour[np] = v;
        pos[v] = np;
      }
      __syncthreads();
      for (int np = lo - 1 + tid; np <= hi; np += THREADS) {
        const int a = tour[np];
        eout[a] = ds(a, tour[np + 1 == n ? 0 : np + 1]);
      }
      ++moves;
    }
    __syncthreads();
    for (int p = tid; p < n; p += THREADS) g[p] = tour[p];
    const long long ev = block_sum(my_eval, redll);
    if (tid == 0) {
      status[t] = err;
      if (stats) {
        stats[(long long)t * 3 + 0] = passes;
        stats[(long long)t * 3 + 1] = moves;
        stats[(long long)t * 3 + 2] = ev;
      }
    }
    __syncthreads();  // tour, s_flag and redll are reused by the next tour
  }
}

template <int THREADS>
static int launch_or_opt(int32_t* tours, int num, int n, const DistSrc& ds, const int32_t* cand,
                         const int32_t* cdist, const uint32_t* packed, int k, int S, long long max_iter,
                         int32_t* status, long long* stats, size_t smem, cudaStream_t st) {
  auto kern = packed ? or_opt_kernel<THREADS, true> : or_opt_kernel<THREADS, false>;
  if (smem > 48 * 1024) TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0, dev = 0, sms = 0;
  TSPB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem));
  if (per_sm <= 0) return TSPB_ERR_UNSUPPORTED;
  TSPB_CUDA_CHECK(cudaGetDevice(&dev));
  TSPB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long grid = (long long)per_sm * sms < num ? (long long)per_sm * sms : num;
  kern<<<(int)grid, THREADS, smem, st>>>(tours, num, n, ds, cand, cdist, packed, k, S, max_iter, status, stats,
                                         watchdog_cycles());
  return tspb_launch_status();
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_or_opt_max_n(void) {
  const long long avail = (long long)smem_optin() - 2048;
  return avail > 0 ? (int)(avail / 16) : 0;
}

extern "C" int tspb_or_opt(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                           const double* coords, const int32_t* cand, const int32_t* cand_dist,
                           const uint32_t* cand_packed, int32_t k, int32_t max_segment, int64_t max_iterations,
                           int32_t threads, int32_t* status, int64_t* stats, void* stream) {
  if (num_tours < 0 || n < 0 || max_iterations < 0 || max_segment < 1 || max_segment > 8) return TSPB_ERR_ARG;
  if (threads != 128 && threads != 256 && threads != 512) return TSPB_ERR_ARG;
  if (num_tours == 0 || n < 3) return TSPB_OK;
  if (!tours || !status || (!dist && !coords) || (dist && dist_stride < n)) return TSPB_ERR_ARG;
  if (k < 1 || k > n - 1 || !cand || !cand_dist) return TSPB_ERR_ARG;
  if (n > tspb_or_opt_max_n()) return TSPB_ERR_UNSUPPORTED;
  // scan items and keys stay in 32 / 64 bits
  if ((long long)(n - 1) * max_segment * 2 * ((k + 3) / 4) > 0x7fffffffLL) return TSPB_ERR_UNSUPPORTED;
  DistSrc ds;
  ds.dist = dist;
  ds.stride = dist_stride;
  ds.coords = reinterpret_cast<const double2*>(coords);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const size_t smem = (size_t)16 * n;
  long long* s = reinterpret_cast<long long*>(stats);
  // the packed words serve only whole, aligned groups of four
  const uint32_t* pk =
      cand_packed && k % 4 == 0 && reinterpret_cast<uintptr_t>(cand_packed) % 16 == 0 ? cand_packed : nullptr;
  switch (threads) {
    case 128:
      return launch_or_opt<128>(tours, num_tours, n, ds, cand, cand_dist, pk, k, max_segment, max_iterations, status, s,
                                smem, st);
    case 512:
      return launch_or_opt<512>(tours, num_tours, n, ds, cand, cand_dist, pk, k, max_segment, max_iterations, status, s,
                                smem, st);
    default:
      return launch_or_opt<256>(tours, num_tours, n, ds, cand, cand_dist, pk, k, max_segment, max_iterations, status, s,
                                smem, st);
  }
}
