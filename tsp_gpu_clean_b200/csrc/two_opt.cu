// Batched 2-opt local search for sm_100a: one CTA per tour, every pass on device.
//
// Semantics follow the reference CPU strategy LocalSearchCPUTourTwoOpt
// (src/algorithms/strategies/local_search/two_opt.py):
//   - scan order: exhaustive pairs (i, j) row-major with j >= i + 2 and (0, n-1)
//     excluded (:188-196); candidate mode rows i in [0, n-3] and candidate rank r in
//     [0, k), j = pos[N_k[tour[i], r]], kept when i + 1 < j < n and j < n - 1 for
//     i == 0, duplicates kept (:347-367);
//   - gain d(a,c) + d(b,d) - d(a,b) - d(c,d) (:237-245) in exact integer arithmetic;
//   - best: the smallest (gain, scan index) over improving pairs (:386-440);
//   - first: the smallest scan index with a negative gain (:442-489);
//   - multi_move: improving pairs sorted by (gain, scan index), accepted greedily when
//     the window [i, j] touches no accepted window (:491-563);
//   - at most max_iterations passes, stopping at the first pass without a move (:565-595).
//
// Device layout per tour: tour, pos (inverse permutation) and edge (d(tour[p],
// tour[p+1])) as int32 arrays in shared memory when 12n bytes fit, else in the
// caller's global workspace. The k-NN table and d(a, N_k[a][r]) are read through L1;
// the one remaining random gather per pair, d(b, d), hits the L2-resident matrix (or
// is rebuilt from FP64 coordinates). multi_move sorts its improving moves in a global
// workspace slice per tour.
#include <algorithm>
#include <atomic>

#include "two_opt.cuh"

namespace tspb {

constexpr long long EXH_BLOCK = 1LL << 18;  // exhaustive pairs per CPU block (two_opt.py:155)

// Pairs of the exhaustive cyclic scan before row i (two_opt.py:188-196).
__device__ __forceinline__ long long exh_row_offset(long long n, long long i) {
  if (i == 0) return 0;
  return (n - 3) + (i - 1) * (n - 2) - (i - 1) * i / 2;
}

struct Smem {
  unsigned long long red64[32];
  long long redll[32];
  unsigned m;       // multi: improving moves found this pass
  unsigned acc;     // multi: moves accepted this pass
  int bad;          // input validation failure
  int stop;         // pass loop must end with an error status
};


// SMEM: tour arrays in shared memory (addressed with shared-memory instructions), else in
// the tour's global workspace slice.
template <int MODE, bool CAND, bool SMEM>
__global__ void __launch_bounds__(1024) two_opt_kernel(const TwoOptArgs A) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ Smem S;

  const int n = A.n;
  const int tid = threadIdx.x;
  const int T = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, nwarps = T >> 5;
  const int t = blockIdx.x;
  if (t >= A.num_tours) return;
  if (A.skip != nullptr && *A.skip != 0) return;

  int32_t* g_tour = A.tours + (long long)t * n;
  unsigned char* ws = A.ws ? A.ws + (size_t)t * A.ws_tour_bytes : nullptr;
  unsigned char* arr = SMEM ? dsm : ws;
  int* s_tour = reinterpret_cast<int*>(arr);
  int* s_pos = s_tour + n;
  int* s_edge = s_pos + n;
  unsigned* occ = reinterpret_cast<unsigned*>(dsm + (SMEM ? (size_t)12 * n : 0));
  unsigned long long* keys = MODE == TSPB_MODE_MULTI_MOVE ? reinterpret_cast<unsigned long long*>(ws + A.ws_keys_off) : nullptr;
  const DistSrc ds = A.ds;
  const int k = A.k;

  // ---- load the tour, build pos, validate --------------------------------------------
  if (tid == 0) S.bad = 0;
  for (int p = tid; p < n; p += T) {
    s_tour[p] = g_tour[p];
    s_pos[p] = -1;
  }
  __syncthreads();
  for (int p = tid; p < n; p += T) {
    const int v = s_tour[p];
    if ((unsigned)v >= (unsigned)n) {
      S.bad = 1;
    } else if (CAND) {
      if (atomicExch(&s_pos[v], p) != -1) S.bad = 1;
    }
  }
  __syncthreads();
  if (S.bad) {
    if (tid == 0) {
      if (A.status) A.status[t] = CAND ? TSPB_ERR_NOT_PERMUTATION : TSPB_ERR_ARG;
      if (A.stats) {
        for (int q = 0; q < 4; ++q) A.stats[(long long)t * 4 + q] = 0;
      }
    }
    return;
  }
  for (int p = tid; p < n; p += T) s_edge[p] = ds(s_tour[p], s_tour[p + 1 == n ? 0 : p + 1]);
  __syncthreads();

  const int rows = n - 2;  // rows i in [0, n - 3]
  const long long exh_total = (long long)(n - 3) + (long long)(n - 3) * (n - 2) / 2;
  long long passes = 0, moves = 0, pairs_closed = 0;
  long long my_pairs = 0, my_eval = 0;
  int err = TSPB_OK;
  const long long t_start = clock64();
  if (tid == 0) S.stop = 0;

  while (passes < A.max_iter) {
    if (tid == 0 && clock64() - t_start > A.budget) S.stop = TSPB_ERR_BUDGET;
    __syncthreads();
    if (S.stop) {
      err = S.stop;
      break;
    }
    ++passes;
    unsigned long long best = NO_KEY;  // BEST / MULTI use gain keys, FIRST uses the index
    unsigned first_idx = NO_IDX;
    if (MODE == TSPB_MODE_MULTI_MOVE) {
      if (tid == 0) S.m = 0;
      __syncthreads();
    }

    if (CAND) {
      const int E = rows * k;
      if (MODE == TSPB_MODE_FIRST) {
        // Chunks in scan order; stop evaluating gains once a chunk holds an improving
        // pair, but keep counting the pairs the CPU scan evaluates (the whole block).
        const int U = 4;
        const int CH = T * U;
        for (int base = 0; base < E; base += CH) {
          unsigned mine = NO_IDX;
          for (int u = 0; u < U; ++u) {
            const int e = base + u * T + tid;
            if (e >= E) break;
            const int i = e / k;
            const int r = e - i * k;
            const int a = s_tour[i];
            const int c = __ldg(A.cand + (long long)a * k + r);
            if ((unsigned)c >= (unsigned)n) continue;
            const int j = s_pos[c];
            const int lim = i == 0 ? n - 1 : n;
            if (j <= i + 1 || j >= lim) continue;
            ++my_pairs;
            if (first_idx != NO_IDX || mine != NO_IDX) continue;
            const int b = s_tour[i + 1];
            const int d = s_tour[j + 1 == n ? 0 : j + 1];
            const int dac = A.cand_dist ? __ldg(A.cand_dist + (long long)a * k + r) : ds(a, c);
            const int gain = (dac - s_edge[i]) + (ds(b, d) - s_edge[j]);
            ++my_eval;
            if (gain < 0) mine = (unsigned)e;
          }
          if (first_idx == NO_IDX) first_idx = block_min(mine, reinterpret_cast<unsigned*>(S.red64));
        }
      } else {
        const int Tq = T / k, Tr = T - (T / k) * k;
        int i = tid / k, r = tid - (tid / k) * k;
        for (int e = tid; e < E; e += T) {
          const int a = s_tour[i];
          const int c = __ldg(A.cand + (long long)a * k + r);
          const int ci = i, cr = r;
          r += Tr;
          i += Tq;
          if (r >= k) {
            r -= k;
            ++i;
          }
          if ((unsigned)c >= (unsigned)n) continue;
          const int j = s_pos[c];
          const int lim = ci == 0 ? n - 1 : n;
          if (j <= ci + 1 || j >= lim) continue;
          ++my_pairs;
          const int b = s_tour[ci + 1];
          const int d = s_tour[j + 1 == n ? 0 : j + 1];
          const int dac = A.cand_dist ? __ldg(A.cand_dist + (long long)a * k + cr) : ds(a, c);
          const int gain = (dac - s_edge[ci]) + (ds(b, d) - s_edge[j]);
          ++my_eval;
          if (gain < 0) {
            const unsigned long long key = gain_key(gain, (unsigned)e);
            if (MODE == TSPB_MODE_BEST) {
              best = key < best ? key : best;
            } else {
              const unsigned slot = atomicAdd(&S.m, 1u);
              keys[slot] = key;
            }
          }
        }
      }
    } else {
      // Exhaustive scan: warp per row, lanes over j; scan index i * n + j.
      if (MODE == TSPB_MODE_FIRST) {
        for (int base = 0; base < rows; base += nwarps) {
          unsigned mine = NO_IDX;
          const int i = base + wid;
          if (i < rows && first_idx == NO_IDX) {
            const int a = s_tour[i], b = s_tour[i + 1], eab = s_edge[i];
            const int lim = i == 0 ? n - 1 : n;
            for (int j = i + 2 + lane; j < lim; j += 32) {
              const int c = s_tour[j], d = s_tour[j + 1 == n ? 0 : j + 1];
              const int gain = (ds(a, c) - eab) + (ds(b, d) - s_edge[j]);
              ++my_eval;
              if (gain < 0) {
                mine = (unsigned)i * (unsigned)n + (unsigned)j;
                break;
              }
            }
          }
          first_idx = block_min(mine, reinterpret_cast<unsigned*>(S.red64));
          if (first_idx != NO_IDX) break;
        }
      } else {
        for (int i = wid; i < rows; i += nwarps) {
          const int a = s_tour[i], b = s_tour[i + 1], eab = s_edge[i];
          const int lim = i == 0 ? n - 1 : n;
          for (int j = i + 2 + lane; j < lim; j += 32) {
            const int c = s_tour[j], d = s_tour[j + 1 == n ? 0 : j + 1];
            const int gain = (ds(a, c) - eab) + (ds(b, d) - s_edge[j]);
            ++my_eval;
            if (gain < 0) {
              const unsigned long long key = gain_key(gain, (unsigned)i * (unsigned)n + (unsigned)j);
              if (MODE == TSPB_MODE_BEST) {
                best = key < best ? key : best;
              } else {
                const unsigned slot = atomicAdd(&S.m, 1u);
                keys[slot] = key;
              }
            }
          }
        }
      }
    }

    // ---- decide ------------------------------------------------------------------------
    int bi = -1, bj = -1;
    if (MODE == TSPB_MODE_BEST) {
      best = block_min(best, S.red64);
      if (!CAND && tid == 0) pairs_closed += exh_total;
      if (best == NO_KEY) break;
      const unsigned idx = (unsigned)best;
      if (CAND) {
        bi = (int)(idx / (unsigned)k);
        const int r = (int)(idx - (unsigned)bi * (unsigned)k);
        bj = s_pos[__ldg(A.cand + (long long)s_tour[bi] * k + r)];
      } else {
        bi = (int)(idx / (unsigned)n);
        bj = (int)(idx - (unsigned)bi * (unsigned)n);
      }
    } else if (MODE == TSPB_MODE_FIRST) {
      if (!CAND && tid == 0) {
        if (first_idx == NO_IDX) {
          pairs_closed += exh_total;
        } else {
          const long long fi = first_idx / (unsigned)n, fj = first_idx - fi * n;
          const long long lin = exh_row_offset(n, fi) + (fj - fi - 2);
          const long long upto = (lin / EXH_BLOCK + 1) * EXH_BLOCK;
          pairs_closed += upto < exh_total ? upto : exh_total;
        }
      }
      if (first_idx == NO_IDX) break;
      if (CAND) {
        bi = (int)(first_idx / (unsigned)k);
        const int r = (int)(first_idx - (unsigned)bi * (unsigned)k);
        bj = s_pos[__ldg(A.cand + (long long)s_tour[bi] * k + r)];
      } else {
        bi = (int)(first_idx / (unsigned)n);
        bj = (int)(first_idx - (unsigned)bi * (unsigned)n);
      }
    }

    if (MODE != TSPB_MODE_MULTI_MOVE) {
      if (bi < 0 || bj <= bi + 1 || bj >= n) {  // cannot happen for a valid scan; never index with it
        err = TSPB_ERR_RANGE;
        break;
      }
      __syncthreads();  // every thread decoded (bi, bj) before the tour changes
      const int lo = bi + 1, hi = bj;
      const int half = (hi - lo + 1) >> 1;
      for (int q = tid; q < half; q += T) {
        const int x = s_tour[lo + q], y = s_tour[hi - q];
        s_tour[lo + q] = y;
        s_tour[hi - q] = x;
        s_pos[y] = lo + q;
        s_pos[x] = hi - q;
      }
      __syncthreads();
      for (int p = bi + tid; p <= bj; p += T) s_edge[p] = ds(s_tour[p], s_tour[p + 1 == n ? 0 : p + 1]);
      __syncthreads();
      ++moves;
      continue;
    }

    // ---- multi_move: sort improving moves, greedy disjoint selection, apply -------------
    __syncthreads();
    if (!CAND && tid == 0) pairs_closed += exh_total;
    const unsigned m = S.m;
    if (m == 0) break;
    unsigned M = 1;
    while (M < m) M <<= 1;
    for (unsigned q = m + tid; q < M; q += T) keys[q] = NO_KEY;
    const int words = (n + 31) >> 5;
    for (int w = tid; w < words; w += T) occ[w] = 0u;
    __syncthreads();
    for (unsigned size = 2; size <= M; size <<= 1) {
      for (unsigned stride = size >> 1; stride > 0; stride >>= 1) {
        for (unsigned q = tid; q < (M >> 1); q += T) {
          const unsigned lo = 2 * q - (q & (stride - 1));
          const unsigned hi = lo + stride;
          const bool asc = (lo & size) == 0;
          const unsigned long long x = keys[lo], y = keys[hi];
          if ((x > y) == asc) {
            keys[lo] = y;
            keys[hi] = x;
          }
        }
        __syncthreads();
      }
    }
    if (wid == 0) {
      unsigned acc = 0;
      for (unsigned q = 0; q < m; ++q) {
        const unsigned long long key = keys[q];
        const unsigned idx = (unsigned)key;
        int i, j;
        if (CAND) {
          i = (int)(idx / (unsigned)k);
          const int r = (int)(idx - (unsigned)i * (unsigned)k);
          j = s_pos[__ldg(A.cand + (long long)s_tour[i] * k + r)];
        } else {
          i = (int)(idx / (unsigned)n);
          j = (int)(idx - (unsigned)i * (unsigned)n);
        }
        if (i < 0 || j <= i + 1 || j >= n) continue;  // cannot happen for a valid scan
        const int lo = i, hi = j;  // occupancy window [max(0, i), j]
        const int w0 = lo >> 5, w1 = hi >> 5;
        bool hit = false;
        for (int w = w0 + lane; w <= w1; w += 32) {
          unsigned mask = ~0u;
          if (w == w0) mask &= ~0u << (lo & 31);
          if (w == w1) mask &= ~0u >> (31 - (hi & 31));
          hit |= (occ[w] & mask) != 0u;
        }
        hit = __any_sync(FULL, hit);
        if (!hit) {
          for (int w = w0 + lane; w <= w1; w += 32) {
            unsigned mask = ~0u;
            if (w == w0) mask &= ~0u << (lo & 31);
            if (w == w1) mask &= ~0u >> (31 - (hi & 31));
            occ[w] |= mask;
          }
          if (lane == 0) keys[acc] = ((unsigned long long)(unsigned)i << 32) | (unsigned)j;
          ++acc;
        }
        __syncwarp();
      }
      if (lane == 0) S.acc = acc;
    }
    __syncthreads();
    const unsigned acc = S.acc;
    for (unsigned mi = wid; mi < acc; mi += nwarps) {
      const unsigned long long ij = keys[mi];
      const int lo = (int)(ij >> 32) + 1, hi = (int)(unsigned)ij;
      const int half = (hi - lo + 1) >> 1;
      for (int q = lane; q < half; q += 32) {
        const int x = s_tour[lo + q], y = s_tour[hi - q];
        s_tour[lo + q] = y;
        s_tour[hi - q] = x;
        s_pos[y] = lo + q;
        s_pos[x] = hi - q;
      }
    }
    __syncthreads();
    for (int p = tid; p < n; p += T) s_edge[p] = ds(s_tour[p], s_tour[p + 1 == n ? 0 : p + 1]);
    __syncthreads();
    moves += 1;
  }

  // ---- write back ---------------------------------------------------------------------
  __syncthreads();
  for (int p = tid; p < n; p += T) g_tour[p] = s_tour[p];
  const long long tp = block_sum(my_pairs, S.redll);
  const long long te = block_sum(my_eval, S.redll);
  if (tid == 0) {
    if (A.status) A.status[t] = err;
    if (A.stats) {
      long long* st = A.stats + (long long)t * 4;
      st[0] = passes;
      st[1] = CAND ? tp : pairs_closed;
      st[2] = moves;
      st[3] = te;
    }
  }
}

static std::atomic<long long> g_watchdog_cycles{BUDGET_CYCLES};

long long watchdog_cycles() { return g_watchdog_cycles.load(std::memory_order_relaxed); }

// Opt-in shared memory per block of the current device, cached per device index (a
// process may drive GPUs of different models).
int smem_optin() {
  constexpr int MAX_DEV = 64;
  static std::atomic<int> cached[MAX_DEV];  // 0: not yet queried
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 0;
  if (dev >= MAX_DEV) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
  }
  int v = cached[dev].load(std::memory_order_relaxed);
  if (v == 0) {
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cached[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

struct Layout {
  bool arrays_in_smem;
  size_t smem_bytes;
  size_t ws_tour_bytes;
  size_t ws_keys_off;
};

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

static unsigned long long next_pow2(unsigned long long v) {
  unsigned long long p = 1;
  while (p < v) p <<= 1;
  return p;
}

static Layout two_opt_layout(int n, int k, int mode, bool cand) {
  Layout L{};
  const size_t arrays = (size_t)12 * n;
  const size_t occ = mode == TSPB_MODE_MULTI_MOVE ? (size_t)((n + 31) / 32) * 4 : 0;
  const size_t budget = (size_t)smem_optin() - sizeof(Smem) - 1024;
  L.arrays_in_smem = arrays + occ <= budget;
  L.smem_bytes = (L.arrays_in_smem ? arrays : 0) + occ;
  size_t off = L.arrays_in_smem ? 0 : align256(arrays);
  L.ws_keys_off = off;
  if (mode == TSPB_MODE_MULTI_MOVE) {
    const unsigned long long rows = n > 2 ? (unsigned long long)(n - 2) : 0ull;
    const unsigned long long cap = cand ? rows * (unsigned long long)k : (unsigned long long)n * (unsigned long long)n / 2;
    off += align256((size_t)next_pow2(cap > 0 ? cap : 1) * 8);
  }
  L.ws_tour_bytes = off;
  return L;
}

template <int MODE, bool CAND>
static int launch(const TwoOptArgs& a, int threads, size_t smem, cudaStream_t st) {
  auto kern = a.arrays_in_smem ? two_opt_kernel<MODE, CAND, true> : two_opt_kernel<MODE, CAND, false>;
  if (smem > 48 * 1024) TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<a.num_tours, threads, smem, st>>>(a);
  return tspb_launch_status();
}

}  // namespace tspb

using namespace tspb;

// Per-tour global bytes of the cached kernel when its arrays do not fit in shared memory.
static size_t cached_ws_tour_bytes(int n, int mode) {
  const size_t need = two_opt_cached_tour_bytes(n, mode);
  const size_t budget = (size_t)smem_optin() - 2048;
  return need <= budget ? 0 : align256(need);
}

extern "C" size_t tspb_two_opt_workspace_bytes(int32_t num_tours, int32_t n, int32_t k, int32_t mode, int32_t block_threads) {
  if (mode >= 0) mode &= ~TSPB_MODE_SYMMETRIC;
  (void)block_threads;
  if (num_tours <= 0 || n < 4) return 0;
  const Layout L = two_opt_layout(n, k, mode, k > 0);
  size_t per = L.ws_tour_bytes;
  if (k > 0 && mode != TSPB_MODE_MULTI_MOVE) {
    const size_t c = cached_ws_tour_bytes(n, mode);
    per = per > c ? per : c;
    const size_t need = two_opt_scan_tour_bytes(n, mode);
    const size_t sc = need <= (size_t)smem_optin() - 2048 ? 0 : align256(need);
    per = per > sc ? per : sc;
  }
  return per * (size_t)num_tours;
}

static int two_opt_impl(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                        const double* coords, const int32_t* cand, const int32_t* cand_dist, const int32_t* rev_off,
                        const int32_t* rev_idx, const uint32_t* cand_packed, int32_t k, int32_t mode,
                        int64_t max_iterations, int32_t block_threads, int64_t* stats, int32_t* status,
                        const int32_t* skip, void* workspace, size_t workspace_bytes, void* stream) {
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // coordinates rebuild EUC_2D distances, which are symmetric
  const int symmetric = (mode & TSPB_MODE_SYMMETRIC) != 0 || dist == nullptr ? 1 : 0;
  if (mode >= 0) mode &= ~TSPB_MODE_SYMMETRIC;
  if (num_tours < 0 || n < 0 || mode < 0 || mode > 2) return TSPB_ERR_ARG;
  if (num_tours == 0) return TSPB_OK;
  if (tours == nullptr || (dist == nullptr && coords == nullptr)) return TSPB_ERR_ARG;
  if (n > 65535) return TSPB_ERR_UNSUPPORTED;  // scan indices are 32-bit (i * n + j)
  if (n < 4 || max_iterations <= 0) {
    if (stats) TSPB_CUDA_CHECK(cudaMemsetAsync(stats, 0, sizeof(int64_t) * 4 * (size_t)num_tours, st));
    if (status) TSPB_CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * (size_t)num_tours, st));
    return TSPB_OK;
  }
  const bool use_cand = cand != nullptr && k > 0;
  if (use_cand && (long long)(n - 2) * k > 0x7fffffffLL) return TSPB_ERR_UNSUPPORTED;
  if (dist != nullptr && dist_stride < n) return TSPB_ERR_ARG;
  int threads = block_threads > 0 ? block_threads : 256;
  if (threads % 32 != 0 || threads > 1024) return TSPB_ERR_ARG;
  const bool has_rev = rev_off != nullptr && rev_idx != nullptr;
  if (use_cand && mode != TSPB_MODE_MULTI_MOVE && (!has_rev || cand_packed != nullptr)) {
    if (threads != 64 && threads != 128 && threads != 256 && threads != 512) return TSPB_ERR_ARG;
    const size_t need = two_opt_scan_tour_bytes(n, mode);
    const size_t per = need <= (size_t)smem_optin() - 2048 ? 0 : align256(need);
    if (per > 0 && (workspace == nullptr || workspace_bytes < per * (size_t)num_tours)) return TSPB_ERR_WORKSPACE;
    if (cand_packed != nullptr && n > 65535) return TSPB_ERR_ARG;
    TwoOptArgs c{};
    c.tours = tours;
    c.num_tours = num_tours;
    c.n = n;
    c.ds.dist = dist;
    c.ds.stride = dist_stride;
    c.ds.coords = reinterpret_cast<const double2*>(coords);
    c.cand = cand;
    c.cand_dist = cand_dist;
    c.cand_packed = cand_packed;
    c.k = k;
    c.max_iter = max_iterations;
    c.stats = reinterpret_cast<long long*>(stats);
    c.status = status;
    c.ws = reinterpret_cast<unsigned char*>(workspace);
    c.ws_tour_bytes = per;
    c.arrays_in_smem = per == 0 ? 1 : 0;
    c.skip = skip;
    c.budget = watchdog_cycles();
    c.symmetric = symmetric;
    if (has_rev && mode == TSPB_MODE_FIRST) {  // incremental restart of first mode
      c.rev_off = rev_off;
      c.rev_idx = rev_idx;
    }
    return launch_two_opt_scan(c, mode, threads, st);
  }
  if (use_cand && rev_off != nullptr && rev_idx != nullptr && mode != TSPB_MODE_MULTI_MOVE) {
    if (threads != 64 && threads != 128 && threads != 256 && threads != 512) return TSPB_ERR_ARG;
    if (k > 255) return TSPB_ERR_UNSUPPORTED;  // per-row counts are packed bytes
    const size_t per = cached_ws_tour_bytes(n, mode);
    if (per > 0 && (workspace == nullptr || workspace_bytes < per * (size_t)num_tours)) return TSPB_ERR_WORKSPACE;
    TwoOptArgs c{};
    c.tours = tours;
    c.num_tours = num_tours;
    c.n = n;
    c.ds.dist = dist;
    c.ds.stride = dist_stride;
    c.ds.coords = reinterpret_cast<const double2*>(coords);
    c.cand = cand;
    c.cand_dist = cand_dist;
    c.k = k;
    c.max_iter = max_iterations;
    c.stats = reinterpret_cast<long long*>(stats);
    c.status = status;
    c.ws = reinterpret_cast<unsigned char*>(workspace);
    c.ws_tour_bytes = per;
    c.arrays_in_smem = per == 0 ? 1 : 0;
    c.rev_off = rev_off;
    c.rev_idx = rev_idx;
    c.skip = skip;
    c.budget = watchdog_cycles();
    return launch_two_opt_cached(c, mode, threads, st);
  }
  const Layout L = two_opt_layout(n, use_cand ? k : 0, mode, use_cand);
  if (L.ws_tour_bytes > 0) {
    if (workspace == nullptr || workspace_bytes < L.ws_tour_bytes * (size_t)num_tours) return TSPB_ERR_WORKSPACE;
  }
  TwoOptArgs a{};
  a.tours = tours;
  a.num_tours = num_tours;
  a.n = n;
  a.ds.dist = dist;
  a.ds.stride = dist_stride;
  a.ds.coords = reinterpret_cast<const double2*>(coords);
  a.cand = use_cand ? cand : nullptr;
  a.cand_dist = use_cand ? cand_dist : nullptr;
  a.k = use_cand ? k : 0;
  a.max_iter = max_iterations;
  a.stats = reinterpret_cast<long long*>(stats);
  a.status = status;
  a.ws = reinterpret_cast<unsigned char*>(workspace);
  a.ws_tour_bytes = L.ws_tour_bytes;
  a.ws_keys_off = L.ws_keys_off;
  a.arrays_in_smem = L.arrays_in_smem ? 1 : 0;
  a.skip = skip;
  a.budget = watchdog_cycles();
  if (use_cand) {
    switch (mode) {
      case TSPB_MODE_BEST: return launch<TSPB_MODE_BEST, true>(a, threads, L.smem_bytes, st);
      case TSPB_MODE_FIRST: return launch<TSPB_MODE_FIRST, true>(a, threads, L.smem_bytes, st);
      default: return launch<TSPB_MODE_MULTI_MOVE, true>(a, threads, L.smem_bytes, st);
    }
  }
  switch (mode) {
    case TSPB_MODE_BEST: return launch<TSPB_MODE_BEST, false>(a, threads, L.smem_bytes, st);
    case TSPB_MODE_FIRST: return launch<TSPB_MODE_FIRST, false>(a, threads, L.smem_bytes, st);
    default: return launch<TSPB_MODE_MULTI_MOVE, false>(a, threads, L.smem_bytes, st);
  }
}

extern "C" int64_t tspb_set_watchdog_cycles(int64_t cycles) {
  return g_watchdog_cycles.exchange(cycles > 0 ? (long long)cycles : BUDGET_CYCLES);
}

extern "C" int tspb_two_opt(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist, int64_t dist_stride,
                            const double* coords, const int32_t* cand, const int32_t* cand_dist, const int32_t* rev_off,
                            const int32_t* rev_idx, const uint32_t* cand_packed, int32_t k, int32_t mode,
                            int64_t max_iterations, int32_t block_threads, int64_t* stats, int32_t* status,
                            void* workspace, size_t workspace_bytes, void* stream) {
  return two_opt_impl(tours, num_tours, n, dist, dist_stride, coords, cand, cand_dist, rev_off, rev_idx, cand_packed, k,
                      mode, max_iterations, block_threads, stats, status, nullptr, workspace, workspace_bytes, stream);
}

extern "C" int tspb_two_opt_gated(const int32_t* skip, int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist,
                                  int64_t dist_stride, const double* coords, const int32_t* cand, const int32_t* cand_dist,
                                  const int32_t* rev_off, const int32_t* rev_idx, const uint32_t* cand_packed, int32_t k,
                                  int32_t mode, int64_t max_iterations, int32_t block_threads, int64_t* stats,
                                  int32_t* status, void* workspace, size_t workspace_bytes, void* stream) {
  if (skip == nullptr) return TSPB_ERR_ARG;
  return two_opt_impl(tours, num_tours, n, dist, dist_stride, coords, cand, cand_dist, rev_off, rev_idx, cand_packed, k,
                      mode, max_iterations, block_threads, stats, status, skip, workspace, workspace_bytes, stream);
}
