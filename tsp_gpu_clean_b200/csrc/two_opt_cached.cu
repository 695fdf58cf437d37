// Candidate-mode 2-opt (best / first) with exact incremental state, one CTA per tour.
//
// The reference rescans every (i, r) entry of the k-NN neighbourhood on every pass
// (src/algorithms/strategies/local_search/two_opt.py:303-367, 386-489). Here the tour is
// held node-indexed as well as position-indexed:
//   tour[p] node at position p      pos[a]  position of node a
//   succ[a] node after a            eout[a] d(a, succ[a])
// so the gain of entry (a, r), c = N_k[a][r], is
//   (d(a, c) - eout[a]) + (d(succ[a], succ[c]) - eout[c])
// with validity pos[c] > pos[a] + 1 (and pos[c] < n - 1 when pos[a] == 0): three
// dependent loads (k-NN entry, then pos/succ/eout of c, then one L2 gather).
//
// Per node a (its "row"), kept exact across passes:
//   ncnt[a]  entries of the row the reference scan evaluates (valid j);
//   best:    nkey[a] = smallest improving (gain, r) of the row;
//   first:   a clean bit = the row is known to hold no improving entry.
// A pass reports sum(ncnt) as the reference's pair count and picks
//   best:  the smallest (gain, pos[a]*k + r) over nkey   (the reference's argmin);
//   first: the smallest pos[a]*k + r with a negative gain (rows scanned in position
//          order, clean rows skipped, rows found clean get their bit set).
//
// After reversing positions [bi+1, bj], entries can change only in
//   1. window rows: nodes at positions [bi, bj], plus the node at position 0 when
//      bj == n-1 (its j == n-1 entry is excluded, :362-365) - recounted, and for best
//      re-keyed, whole;
//   2. entries whose candidate c sits in [bi, bj] (found through the reverse k-NN
//      index): their validity cannot change (positions outside the window keep their
//      order relative to it), only the gain. best re-evaluates them: a better key lowers
//      the row key atomically, and the row's own best entry getting worse marks the row
//      dirty for a whole-row recompute. first only clears the row's clean bit.
// Results (tour sequence, pass and pair counts) are those of the full rescan, bit for
// bit; the work per pass is O(k * window) instead of O(k * n).
#include "two_opt.cuh"

namespace tspb {

constexpr int ILP = 4;  // entries whose loads a thread keeps in flight together

struct CachedSmem {
  unsigned long long red64[32];
  long long redll[32];
  long long total;  // valid entries of the current tour (the reference's pair count)
  int bad;
  int stop;
  int nwin;         // window rows this pass
  int e2;           // reverse-index entries of the window this pass
};

struct NodeTour {
  const int32_t* cand;
  const int32_t* cand_dist;
  const int32_t* rev_off;
  const int32_t* rev_idx;
  DistSrc ds;
  int n, k, rows;
  int* tour;
  int* pos;
  int* succ;
  int* eout;
  unsigned long long* nkey;  // best only
  unsigned* ncnt;            // packed byte counts, node a in byte a & 3 of word a >> 2
  unsigned* bits;            // best: dirty rows; first: clean rows
  int* off2;                 // per-pass prefix of reverse-list lengths over the window

  __device__ __forceinline__ int count(int a) const { return (ncnt[a >> 2] >> ((a & 3) * 8)) & 0xff; }
  __device__ __forceinline__ void set_count(int a, int v) const {
    atomicAnd(&ncnt[a >> 2], ~(0xffu << ((a & 3) * 8)));
    atomicOr(&ncnt[a >> 2], (unsigned)v << ((a & 3) * 8));
  }
  __device__ __forceinline__ void add_count(int a, int v) const { atomicAdd(&ncnt[a >> 2], (unsigned)v << ((a & 3) * 8)); }
  __device__ __forceinline__ bool valid_ij(int i, int j) const { return j > i + 1 && j < (i == 0 ? n - 1 : n); }
};

// Evaluates U entries (a[u], r[u]) with their loads batched; gain[u] valid when ok[u].
template <int U>
__device__ __forceinline__ void eval_batch(const NodeTour& T, const int (&a)[U], const int (&r)[U], bool (&ok)[U],
                                           int (&gain)[U], long long& evals) {
  int c[U], cd[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const long long ar = (long long)a[u] * T.k + r[u];
    c[u] = a[u] >= 0 ? __ldg(T.cand + ar) : -1;
    cd[u] = (a[u] >= 0 && T.cand_dist) ? __ldg(T.cand_dist + ar) : 0;
  }
  int sa[U], sc[U], ea[U], ec[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    ok[u] = false;
    if (a[u] < 0 || (unsigned)c[u] >= (unsigned)T.n) continue;
    const int i = T.pos[a[u]], j = T.pos[c[u]];
    ok[u] = T.valid_ij(i, j);
    sa[u] = T.succ[a[u]];
    sc[u] = T.succ[c[u]];
    ea[u] = T.eout[a[u]];
    ec[u] = T.eout[c[u]];
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (!ok[u]) continue;
    const int dac = T.cand_dist ? cd[u] : T.ds(a[u], c[u]);
    gain[u] = (dac - ea[u]) + (T.ds(sa[u], sc[u]) - ec[u]);
    ++evals;
  }
}

// Validity only (no distances): how many entries of the reference scan a row holds.
template <int U>
__device__ __forceinline__ void valid_batch(const NodeTour& T, const int (&a)[U], const int (&r)[U], bool (&ok)[U]) {
  int c[U];
#pragma unroll
  for (int u = 0; u < U; ++u) c[u] = a[u] >= 0 ? __ldg(T.cand + (long long)a[u] * T.k + r[u]) : -1;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    ok[u] = false;
    if (a[u] < 0 || (unsigned)c[u] >= (unsigned)T.n) continue;
    ok[u] = T.valid_ij(T.pos[a[u]], T.pos[c[u]]);
  }
}

__device__ __forceinline__ unsigned long long best_key(int gain, int r) { return gain_key(gain, (unsigned)r); }

// Whole row of node a for best: (smallest improving key, valid count).
__device__ __forceinline__ void row_best(const NodeTour& T, int a, unsigned long long& key, int& cnt, long long& evals) {
  key = NO_KEY;
  cnt = 0;
  for (int r0 = 0; r0 < T.k; r0 += ILP) {
    int aa[ILP], rr[ILP], g[ILP];
    bool ok[ILP];
#pragma unroll
    for (int u = 0; u < ILP; ++u) {
      rr[u] = r0 + u;
      aa[u] = rr[u] < T.k ? a : -1;
    }
    eval_batch<ILP>(T, aa, rr, ok, g, evals);
#pragma unroll
    for (int u = 0; u < ILP; ++u) {
      if (!ok[u]) continue;
      ++cnt;
      if (g[u] < 0) {
        const unsigned long long kk = best_key(g[u], rr[u]);
        key = kk < key ? kk : key;
      }
    }
  }
}

// First improving r of node a's row in scan order, or -1.
__device__ __forceinline__ int row_first(const NodeTour& T, int a, long long& evals) {
  for (int r0 = 0; r0 < T.k; r0 += ILP) {
    int aa[ILP], rr[ILP], g[ILP];
    bool ok[ILP];
#pragma unroll
    for (int u = 0; u < ILP; ++u) {
      rr[u] = r0 + u;
      aa[u] = rr[u] < T.k ? a : -1;
    }
    eval_batch<ILP>(T, aa, rr, ok, g, evals);
#pragma unroll
    for (int u = 0; u < ILP; ++u)
      if (ok[u] && g[u] < 0) return rr[u];
  }
  return -1;
}

// Resident CTAs per SM the register budget must allow (1024-tour batches fill one wave).
template <int THREADS>
struct MinBlocks {
  static constexpr int value = THREADS == 64 ? 16 : THREADS == 128 ? 8 : THREADS == 256 ? 4 : 2;
};

// SMEM: per-tour arrays in shared memory (shared-memory instructions), else in the tour's
// global workspace slice.
template <int MODE, int THREADS, bool SMEM>
__global__ void __launch_bounds__(THREADS, MinBlocks<THREADS>::value) two_opt_cached_kernel(const TwoOptArgs A) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ CachedSmem S;
  const int n = A.n, k = A.k, rows = n - 2;
  const int tid = threadIdx.x;
  const int t = blockIdx.x;
  if (t >= A.num_tours) return;
  if (A.skip != nullptr && *A.skip != 0) return;

  int32_t* g_tour = A.tours + (long long)t * n;
  unsigned char* base = SMEM ? dsm : A.ws + (size_t)t * A.ws_tour_bytes;
  NodeTour T{A.cand, A.cand_dist, A.rev_off, A.rev_idx, A.ds, n, k, rows};
  T.nkey = reinterpret_cast<unsigned long long*>(base);
  T.tour = reinterpret_cast<int*>(T.nkey + (MODE == TSPB_MODE_BEST ? n : 0));
  T.pos = T.tour + n;
  T.succ = T.pos + n;
  T.eout = T.succ + n;
  T.off2 = T.eout + n;             // n + 1 entries
  T.ncnt = reinterpret_cast<unsigned*>(T.off2 + n + 1);
  const int cwords = (n + 3) >> 2;
  T.bits = T.ncnt + cwords;
  const int bwords = (n + 31) >> 5;

  // ---- load, validate, successor and edge arrays ------------------------------------------
  if (tid == 0) {
    S.bad = 0;
    S.stop = 0;
    S.total = 0;
  }
  for (int p = tid; p < n; p += THREADS) {
    T.tour[p] = g_tour[p];
    T.pos[p] = -1;
  }
  for (int w = tid; w < cwords; w += THREADS) T.ncnt[w] = 0u;
  for (int w = tid; w < bwords; w += THREADS) T.bits[w] = 0u;
  __syncthreads();
  for (int p = tid; p < n; p += THREADS) {
    const int v = T.tour[p];
    if ((unsigned)v >= (unsigned)n || atomicExch(&T.pos[v], p) != -1) S.bad = 1;
  }
  __syncthreads();
  if (S.bad) {
    if (tid == 0) {
      if (A.status) A.status[t] = TSPB_ERR_NOT_PERMUTATION;
      if (A.stats)
        for (int q = 0; q < 4; ++q) A.stats[(long long)t * 4 + q] = 0;
    }
    return;
  }
  for (int p = tid; p < n; p += THREADS) {
    const int x = T.tour[p], y = T.tour[p + 1 == n ? 0 : p + 1];
    T.succ[x] = y;
    T.eout[x] = T.ds(x, y);
  }
  __syncthreads();

  long long evals = 0;
  // ---- initial rows --------------------------------------------------------------------------
  {
    long long csum = 0;
    for (int a = tid; a < n; a += THREADS) {
      if (MODE == TSPB_MODE_BEST) {
        unsigned long long key;
        int cnt;
        row_best(T, a, key, cnt, evals);
        T.nkey[a] = key;
        T.add_count(a, cnt);
        csum += cnt;
      } else {
        int cnt = 0;
        for (int r0 = 0; r0 < k; r0 += ILP) {
          int aa[ILP], rr[ILP];
          bool ok[ILP];
#pragma unroll
          for (int u = 0; u < ILP; ++u) {
            rr[u] = r0 + u;
            aa[u] = rr[u] < k ? a : -1;
          }
          valid_batch<ILP>(T, aa, rr, ok);
#pragma unroll
          for (int u = 0; u < ILP; ++u) cnt += ok[u];
        }
        T.add_count(a, cnt);
        csum += cnt;
      }
    }
    csum = warp_sum(csum);
    if ((tid & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&S.total), (unsigned long long)csum);
  }
  __syncthreads();

  long long passes = 0, moves = 0, pairs = 0;
  int err = TSPB_OK;
  const long long t_start = clock64();
  while (passes < A.max_iter) {
    if (tid == 0 && clock64() - t_start > A.budget) S.stop = TSPB_ERR_BUDGET;
    __syncthreads();
    if (S.stop) {
      err = S.stop;
      break;
    }
    ++passes;
    if (tid == 0) pairs += S.total;

    // ---- pick ---------------------------------------------------------------------------------
    unsigned long long pick = NO_KEY;
    if (MODE == TSPB_MODE_BEST) {
      for (int a = tid; a < n; a += THREADS) {
        const unsigned long long rk = T.nkey[a];
        if (rk != NO_KEY) {
          const unsigned long long g = (rk & 0xffffffff00000000ull) | ((unsigned)T.pos[a] * (unsigned)k + (unsigned)rk);
          pick = g < pick ? g : pick;
        }
      }
      pick = block_min(pick, S.red64);
    } else {
      // rows in position order, four positions per thread per chunk; clean rows skipped
      constexpr int PER = 4;
      for (int base_p = 0; base_p < rows; base_p += THREADS * PER) {
        unsigned long long mine = NO_KEY;
        for (int u = 0; u < PER && mine == NO_KEY; ++u) {
          const int i = base_p + u * THREADS + tid;
          if (i >= rows) break;
          const int a = T.tour[i];
          if (T.bits[a >> 5] & (1u << (a & 31))) continue;
          const int fr = row_first(T, a, evals);
          if (fr < 0) {
            atomicOr(&T.bits[a >> 5], 1u << (a & 31));
          } else {
            mine = (unsigned long long)((unsigned)i * (unsigned)k + (unsigned)fr);
          }
        }
        pick = block_min(mine, S.red64);
        if (pick != NO_KEY) break;
      }
    }
    if (pick == NO_KEY) break;
    const unsigned idx = (unsigned)pick;
    const int bi = (int)(idx / (unsigned)k);
    const int br = (int)(idx - (unsigned)bi * (unsigned)k);
    const int bj = T.pos[__ldg(A.cand + (long long)T.tour[bi] * k + br)];
    if (bi < 0 || bj <= bi + 1 || bj >= n) {
      err = TSPB_ERR_RANGE;
      break;
    }
    __syncthreads();

    // ---- reversal of positions [bi+1, bj] -----------------------------------------------------
    {
      const int lo = bi + 1, hi = bj, half = (hi - lo + 1) >> 1;
      for (int q = tid; q < half; q += THREADS) {
        const int x = T.tour[lo + q], y = T.tour[hi - q];
        T.tour[lo + q] = y;
        T.tour[hi - q] = x;
        T.pos[y] = lo + q;
        T.pos[x] = hi - q;
      }
    }
    __syncthreads();
    ++moves;
    const int nw = bj - bi + 1;                       // window positions [bi, bj]
    const bool row0 = (bj == n - 1) && (bi > 0);      // node at position 0 also re-counted
    const int nrow = nw + (row0 ? 1 : 0);
    long long dcnt = 0;
    for (int q = tid; q < nw; q += THREADS) {
      const int p = bi + q;
      const int x = T.tour[p], y = T.tour[p + 1 == n ? 0 : p + 1];
      T.succ[x] = y;
      T.eout[x] = T.ds(x, y);
      const int c = x;
      const int len = __ldg(T.rev_off + c + 1) - __ldg(T.rev_off + c);
      T.off2[q + 1] = len;
    }
    for (int q = tid; q < nrow; q += THREADS) {
      const int a = T.tour[q < nw ? bi + q : 0];
      dcnt -= T.count(a);
      T.set_count(a, 0);
      if (MODE == TSPB_MODE_BEST) T.nkey[a] = NO_KEY;
      else atomicAnd(&T.bits[a >> 5], ~(1u << (a & 31)));
    }
    __syncthreads();
    // exclusive prefix of the window's reverse-list lengths (single pass, one warp per 32)
    {
      const int lane = tid & 31, wid = tid >> 5;
      if (wid == 0) {
        int carry = 0;
        for (int b0 = 0; b0 < nw; b0 += 32) {
          const int q = b0 + lane;
          int v = q < nw ? T.off2[q + 1] : 0;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, v, o);
            if (lane >= o) v += y;
          }
          if (q < nw) T.off2[q + 1] = carry + v;
          carry += __shfl_sync(FULL, v, 31);
        }
        if (lane == 0) {
          T.off2[0] = 0;
          S.e2 = carry;
        }
      }
    }
    __syncthreads();

    // ---- window rows (counts; best also keys) and candidate-side entries ----------------------
    const int e1 = nrow * k;
    const int e2 = S.e2;
    for (int q0 = tid; q0 < e1 + e2; q0 += THREADS * ILP) {
      int aa[ILP], rr[ILP], g[ILP];
      bool ok[ILP];
      bool side2[ILP];
#pragma unroll
      for (int u = 0; u < ILP; ++u) {
        const int q = q0 + u * THREADS;
        aa[u] = -1;
        rr[u] = 0;
        side2[u] = false;
        if (q < e1) {
          const int row = q / k;
          rr[u] = q - row * k;
          aa[u] = T.tour[row < nw ? bi + row : 0];
        } else if (q < e1 + e2) {
          const int q2 = q - e1;
          int lo = 0, hi = nw;  // largest w with off2[w] <= q2
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (T.off2[mid] <= q2) lo = mid; else hi = mid;
          }
          const int c = T.tour[bi + lo];
          const int e = __ldg(T.rev_idx + __ldg(T.rev_off + c) + (q2 - T.off2[lo]));
          const int a = e / k;
          const int ia = T.pos[a];
          if (!((ia >= bi && ia <= bj) || (row0 && ia == 0))) {
            aa[u] = a;
            rr[u] = e - a * k;
            side2[u] = true;
          }
        }
      }
      if (MODE == TSPB_MODE_BEST) {
        eval_batch<ILP>(T, aa, rr, ok, g, evals);
#pragma unroll
        for (int u = 0; u < ILP; ++u) {
          if (aa[u] < 0) continue;
          const int a = aa[u];
          const unsigned long long key = (ok[u] && g[u] < 0) ? best_key(g[u], rr[u]) : NO_KEY;
          if (!side2[u]) {
            if (ok[u]) {
              T.add_count(a, 1);
              ++dcnt;
            }
            if (key != NO_KEY) atomicMin(&T.nkey[a], key);
          } else {
            const unsigned long long old = T.nkey[a];
            if (key < old) {
              atomicMin(&T.nkey[a], key);
            } else if ((unsigned)old == (unsigned)rr[u] && key != old) {
              atomicOr(&T.bits[a >> 5], 1u << (a & 31));
            }
          }
        }
      } else {
        bool v[ILP];
        valid_batch<ILP>(T, aa, rr, v);
#pragma unroll
        for (int u = 0; u < ILP; ++u) {
          if (aa[u] < 0) continue;
          const int a = aa[u];
          if (!side2[u]) {
            if (v[u]) {
              T.add_count(a, 1);
              ++dcnt;
            }
          } else {
            atomicAnd(&T.bits[a >> 5], ~(1u << (a & 31)));
          }
        }
      }
    }
    dcnt = warp_sum(dcnt);
    if ((tid & 31) == 0 && dcnt != 0) atomicAdd(reinterpret_cast<unsigned long long*>(&S.total), (unsigned long long)dcnt);
    __syncthreads();
    if (MODE == TSPB_MODE_BEST) {
      // dirty rows: their best entry got worse; recompute the key of the whole row
      for (int w = tid; w < bwords; w += THREADS) {
        unsigned m = T.bits[w];
        if (m == 0u) continue;
        T.bits[w] = 0u;
        while (m) {
          const int b = __ffs(m) - 1;
          m &= m - 1;
          const int a = (w << 5) + b;
          unsigned long long key;
          int cnt;
          row_best(T, a, key, cnt, evals);
          T.nkey[a] = key;
        }
      }
      __syncthreads();
    }
  }

  __syncthreads();
  for (int p = tid; p < n; p += THREADS) g_tour[p] = T.tour[p];
  const long long te = block_sum(evals, S.redll);
  if (tid == 0) {
    if (A.status) A.status[t] = err;
    if (A.stats) {
      long long* st = A.stats + (long long)t * 4;
      st[0] = passes;
      st[1] = pairs;
      st[2] = moves;
      st[3] = te;
    }
  }
}

size_t two_opt_cached_tour_bytes(int n, int mode) {
  const size_t key = mode == TSPB_MODE_BEST ? (size_t)8 * n : 0;
  return key + (size_t)16 * n + (size_t)4 * (n + 1) + (size_t)4 * ((n + 3) / 4) + (size_t)4 * ((n + 31) / 32);
}

template <int MODE, int THREADS>
static int launch_cached(const TwoOptArgs& a, size_t smem, cudaStream_t st) {
  auto kern = a.arrays_in_smem ? two_opt_cached_kernel<MODE, THREADS, true> : two_opt_cached_kernel<MODE, THREADS, false>;
  if (smem > 48 * 1024) TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<a.num_tours, THREADS, smem, st>>>(a);
  return tspb_launch_status();
}

int launch_two_opt_cached(const TwoOptArgs& a, int mode, int threads, cudaStream_t st) {
  const size_t smem = a.arrays_in_smem ? two_opt_cached_tour_bytes(a.n, mode) : 0;
  if (mode == TSPB_MODE_BEST) {
    switch (threads) {
      case 64: return launch_cached<TSPB_MODE_BEST, 64>(a, smem, st);
      case 128: return launch_cached<TSPB_MODE_BEST, 128>(a, smem, st);
      case 512: return launch_cached<TSPB_MODE_BEST, 512>(a, smem, st);
      default: return launch_cached<TSPB_MODE_BEST, 256>(a, smem, st);
    }
  }
  switch (threads) {
    case 64: return launch_cached<TSPB_MODE_FIRST, 64>(a, smem, st);
    case 128: return launch_cached<TSPB_MODE_FIRST, 128>(a, smem, st);
    case 512: return launch_cached<TSPB_MODE_FIRST, 512>(a, smem, st);
    default: return launch_cached<TSPB_MODE_FIRST, 256>(a, smem, st);
  }
}

// ---- reverse k-NN index: for every node c, the flat entries a*k + r with cand[a][r] == c --
__global__ void rev_count_kernel(const int32_t* __restrict__ cand, long long total, int n, int32_t* __restrict__ cnt) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int c = __ldg(cand + e);
  if ((unsigned)c < (unsigned)n) atomicAdd(&cnt[c], 1);
}

// Single-block exclusive scan of n counts into off[0..n]; cnt is reset to zero for the fill.
__global__ void rev_scan_kernel(int32_t* __restrict__ cnt, int n, int32_t* __restrict__ off) {
  __shared__ int carry;
  __shared__ int warp_tot[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    const int i = base + tid;
    const int v = i < n ? cnt[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    int pre = 0;
    for (int w = 0; w < wid; ++w) pre += warp_tot[w];
    if (i < n) {
      off[i] = carry + pre + x - v;
      cnt[i] = 0;
    }
    __syncthreads();
    if (tid == blockDim.x - 1) carry += pre + x;
    __syncthreads();
  }
  if (tid == 0) off[n] = carry;
}

__global__ void rev_fill_kernel(const int32_t* __restrict__ cand, long long total, int n, const int32_t* __restrict__ off,
                                int32_t* __restrict__ cursor, int32_t* __restrict__ idx) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int c = __ldg(cand + e);
  if ((unsigned)c < (unsigned)n) idx[off[c] + atomicAdd(&cursor[c], 1)] = (int32_t)e;
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_candidate_reverse_index(const int32_t* cand, int32_t n, int32_t k, int32_t* rev_off, int32_t* rev_idx,
                                            int32_t* scratch, void* stream) {
  if (n < 0 || k < 0) return TSPB_ERR_ARG;
  if (!rev_off || !scratch || (n > 0 && k > 0 && (!cand || !rev_idx))) return TSPB_ERR_ARG;
  if ((long long)n * k > 0x7fffffffLL) return TSPB_ERR_UNSUPPORTED;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  TSPB_CUDA_CHECK(cudaMemsetAsync(scratch, 0, sizeof(int32_t) * (size_t)(n > 0 ? n : 1), st));
  const long long total = (long long)n * k;
  if (total > 0) rev_count_kernel<<<(int)((total + 255) / 256), 256, 0, st>>>(cand, total, n, scratch);
  rev_scan_kernel<<<1, 1024, 0, st>>>(scratch, n, rev_off);
  if (total > 0) rev_fill_kernel<<<(int)((total + 255) / 256), 256, 0, st>>>(cand, total, n, rev_off, scratch, rev_idx);
  return tspb_launch_status();
}
