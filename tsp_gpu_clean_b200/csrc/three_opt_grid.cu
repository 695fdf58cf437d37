// 3-opt with the rules of the reference's grid kernels: the candidate-pruned scan (one move
// per pass or multi_move) and the exhaustive multi_move.
//
// The reference defines these two parts of its experimental 3-opt only through its CUDA
// kernels (benchmark_scripts/experiments-and-examples/experiment-comparing-3opt-and-2opt/
// kernels/three_opt_common.cuh:155-447, three_opt_batch.cu, three_opt_multi_move.cu), so
// their results follow that kernel's thread layout: B = prev_power_of_2(min(threads, n))
// (at most 256) threads per tour, thread t scanning the anchors i = t, t + B, ... and keeping
// its first strictly smallest move, then a block reduction (batch) or a greedy selection of
// disjoint moves (multi_move). This file computes the same moves with another layout:
//
// - a warp per anchor row: its lanes split the row's candidate work (2-opt seeds, the
//   pass-A and pass-B pairs of k-NN entries, or for the exhaustive scan the k of each
//   (i, j)), and the row's best is the minimum of (delta, position in the row's scan
//   order), packed into one u64 per row: (delta + 2^32) << 27 | order;
// - "thread" t's best is then the first row, in increasing i over i = t (mod B), holding the
//   smallest delta (one pass over n / B row keys), and its move is re-derived from (i, order);
// - the reduction and the multi_move selection run on those B bests exactly as the
//   reference orders them (pairwise t vs t + s for s = B/2 .. 64, then t = 1 .. 63 in
//   order, strictly smaller wins; multi_move: lowest t among the smallest, disjoint spans).
//
// A move (i0 < j0 < k0, case) is applied as the reversals [i0+1, j0] (cases 1, 4, 5, 7),
// [j0+1, k0] (2, 4, 5, 6), then [i0+1, k0] (3, 5, 6, 7). Distances are below 2^30, so a
// delta of three edges fits the 32-bit field of the row key.
#include "common.cuh"
#include "two_opt.cuh"

namespace tspb {

constexpr int kGridThreads = 256;      // CTA size; also the largest reference block
constexpr int kGridExhaustiveMaxN = 4096;
constexpr unsigned long long kGridNoKey = ~0ull;
constexpr int kOrderBits = 27;

__device__ __forceinline__ unsigned long long row_key(long long delta, unsigned order) {
  return ((unsigned long long)(delta + (1LL << 32)) << kOrderBits) | order;
}
__device__ __forceinline__ long long row_key_delta(unsigned long long key) {
  return (long long)(key >> kOrderBits) - (1LL << 32);
}

struct Move {
  int i, j, k, c;
};

// Cyclic cuts (i -> jc -> kc) as sorted linear cuts (the reference's C3 rotation).
__device__ __forceinline__ Move rotate_cuts(int i, int jc, int kc, int c) {
  if (i < jc && jc < kc) return {i, jc, kc, c};
  if (kc < i && i < jc) return {kc, i, jc, c == 4 ? 6 : c == 6 ? 7 : c == 7 ? 4 : 5};
  return {jc, kc, i, c == 4 ? 7 : c == 7 ? 6 : c == 6 ? 4 : 5};
}

struct GridTour {
  const int* t;
  const int* pos;
  const int* edge;
  int n;
  DistSrc ds;
  __device__ __forceinline__ int at(int p) const { return t[p >= n ? p - n : p]; }
};

// The candidate move of pair (p1, p2) with sub-case `sub` (0..2), or {-1} when that
// sub-case is not one the reference evaluates for these relative positions.
__device__ __forceinline__ bool pair_case(const GridTour& G, int i, int p1, int p2, int sub, int& jc, int& kc,
                                          int& c) {
  const int n = G.n;
  int rel1 = p1 - i, rel2 = p2 - i;
  if (rel1 < 0) rel1 += n;
  if (rel2 < 0) rel2 += n;
  if (rel1 >= 2 && rel1 < rel2) {
    if (sub == 0) { jc = p1; kc = p2; c = 4; }
    else if (sub == 1) { jc = p1 > 0 ? p1 - 1 : n - 1; kc = p2; c = 5; }
    else { jc = p1 > 0 ? p1 - 1 : n - 1; kc = p2 > 0 ? p2 - 1 : n - 1; c = 6; }
    return true;
  }
  if (sub != 0) return false;
  if (rel1 >= 2 && rel1 == rel2) { jc = p1 > 0 ? p1 - 1 : n - 1; kc = p1; c = 5; return true; }
  if (rel2 >= 2 && rel2 < rel1) { jc = p2 > 0 ? p2 - 1 : n - 1; kc = p1; c = 7; return true; }
  return false;
}

// Delta of a pair case: d(a,v1) + d(b,v2) - d(a,b) - edge[jc] - edge[kc] + the third new edge.
__device__ __forceinline__ long long pair_delta(const GridTour& G, int base, int jc, int kc, int c) {
  int x, y;
  if (c == 4) { x = G.at(jc + 1); y = G.at(kc + 1); }       // (d, f)
  else if (c == 6) { x = G.t[jc]; y = G.t[kc]; }             // (c, e)
  else { x = G.t[jc]; y = G.at(kc + 1); }                     // cases 5, 7: (c, f)
  return (long long)base - G.edge[jc] - G.edge[kc] + G.ds(x, y);
}

struct CandRow {
  const int32_t* cand;
  const int32_t* cdist;
  int k, inner;
};

// Re-derive the move of anchor i at scan position `order` (candidate scan).
__device__ Move cand_move(const GridTour& G, const CandRow& C, int i, unsigned order) {
  const int k = C.k, inner = C.inner;
  const int a = G.t[i], b = G.at(i + 1);
  if (order < (unsigned)k) {
    const int p1 = G.pos[__ldg(C.cand + (size_t)a * k + order)];
    return {i, p1, p1, 1};
  }
  unsigned o = order - (unsigned)k;
  const unsigned span = (unsigned)k * (unsigned)inner * 3u;
  int r1, r2;
  const bool passB = o >= span;
  if (passB) o -= span;
  const int q = (int)(o / 3u), sub = (int)(o % 3u);
  if (!passB) { r1 = q / inner; r2 = q % inner; }
  else { r2 = q / inner; r1 = q % inner; }
  const int p1 = G.pos[__ldg(C.cand + (size_t)a * k + r1)];
  const int p2 = G.pos[__ldg(C.cand + (size_t)b * k + r2)];
  int jc = 0, kc = 0, c = 0;
  pair_case(G, i, p1, p2, sub, jc, kc, c);
  return rotate_cuts(i, jc, kc, c);
}

// Best (delta, order) of anchor row i of the candidate scan, by one warp.
__device__ unsigned long long cand_row(const GridTour& G, const CandRow& C, int i, long long& evals) {
  const int n = G.n, k = C.k, inner = C.inner, lane = threadIdx.x & 31;
  const int a = G.t[i], b = G.at(i + 1);
  const int d_ab = G.edge[i];
  const int32_t* ca = C.cand + (size_t)a * k;
  const int32_t* cb = C.cand + (size_t)b * k;
  const int32_t* da = C.cdist + (size_t)a * k;
  const int32_t* db = C.cdist + (size_t)b * k;
  long long bd = 0;
  unsigned bo = 0xffffffffu;
  auto take = [&](long long d, unsigned o) {
    if (d < bd || (d == bd && d < 0 && o < bo)) { bd = d; bo = o; }
  };
  // 2-opt seeds
  for (int r1 = lane; r1 < k; r1 += 32) {
    const int v1 = __ldg(ca + r1), p1 = G.pos[v1];
    if (p1 > i + 1 && !(i == 0 && p1 == n - 1)) {
      ++evals;
      const long long d = (long long)__ldg(da + r1) - d_ab - G.edge[p1] + G.ds(b, G.at(p1 + 1));
      take(d, (unsigned)r1);
    }
  }
  // leading entries closer than d(a, b) (pass A) and d(b, a') (pass B): the reference stops
  // each outer loop at the first entry that is not
  int R1 = k, R2 = k;
  for (int r0 = 0; r0 < k; r0 += 32) {
    const int r = r0 + lane;
    const unsigned m1 = __ballot_sync(FULL, r < k && __ldg(da + (r < k ? r : 0)) >= d_ab);
    const unsigned m2 = __ballot_sync(FULL, r < k && __ldg(db + (r < k ? r : 0)) >= d_ab);
    if (R1 == k && m1) R1 = r0 + __ffs(m1) - 1;
    if (R2 == k && m2) R2 = r0 + __ffs(m2) - 1;
  }
  const int base_a = k, base_b = k + k * inner * 3;
  // pass A: (r1 < R1, r2 < inner)
  for (int q = lane; q < R1 * inner; q += 32) {
    const int r1 = q / inner, r2 = q - r1 * inner;
    const int v1 = __ldg(ca + r1), v2 = __ldg(cb + r2);
    const int p1 = G.pos[v1], p2 = G.pos[v2];
    const int base = __ldg(da + r1) + __ldg(db + r2) - d_ab;
    for (int sub = 0; sub < 3; ++sub) {
      int jc, kc, c;
      if (!pair_case(G, i, p1, p2, sub, jc, kc, c)) break;
      ++evals;
      take(pair_delta(G, base, jc, kc, c), (unsigned)(base_a + q * 3 + sub));
    }
  }
  // pass B: (r2 < R2, r1 < inner with d(a, v1) >= d(a, b))
  for (int q = lane; q < R2 * inner; q += 32) {
    const int r2 = q / inner, r1 = q - r2 * inner;
    const int dav1 = __ldg(da + r1);
    if (dav1 < d_ab) continue;
    const int v1 = __ldg(ca + r1), v2 = __ldg(cb + r2);
    const int p1 = G.pos[v1], p2 = G.pos[v2];
    const int base = dav1 + __ldg(db + r2) - d_ab;
    for (int sub = 0; sub < 3; ++sub) {
      int jc, kc, c;
      if (!pair_case(G, i, p1, p2, sub, jc, kc, c)) break;
      ++evals;
      take(pair_delta(G, base, jc, kc, c), (unsigned)(base_b + q * 3 + sub));
    }
  }
  // warp minimum of (delta, order)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long od = __shfl_xor_sync(FULL, bd, o);
    const unsigned oo = __shfl_xor_sync(FULL, bo, o);
    if (od < bd || (od == bd && oo < bo)) { bd = od; bo = oo; }
  }
  return bd < 0 ? row_key(bd, bo) : kGridNoKey;
}

// Best (delta, key) of the exhaustive (i, j) row, key = (j n + k) 8 + case, by one warp.
__device__ unsigned long long exhaustive_row(const GridTour& G, int i, int j, long long& evals) {
  const int n = G.n, lane = threadIdx.x & 31;
  const int a = G.t[i], b = G.t[i + 1], c = G.t[j], d = G.t[j + 1];
  const int d_ab = G.edge[i], d_cd = G.edge[j];
  const int d_ac = G.ds(a, c), d_ad = G.ds(a, d), d_bd = G.ds(b, d);
  long long bd = 0;
  unsigned bo = 0xffffffffu;
  auto take = [&](long long dl, unsigned o) {
    if (dl < bd || (dl == bd && dl < 0 && o < bo)) { bd = dl; bo = o; }
  };
  const unsigned jn = (unsigned)j * (unsigned)n;
  if (lane == 0 && j > i + 1) {
    ++evals;
    take((long long)d_ac + d_bd - d_ab - d_cd, (jn + (unsigned)j) * 8u + 1u);
  }
  const long long old_ab_cd = (long long)d_ab + d_cd;
  for (int k = j + 1 + lane; k <= n - 1; k += 32) {
    const int e = G.t[k], f = G.at(k + 1);
    const int d_ef = G.edge[k];
    const long long old3 = old_ab_cd + d_ef;
    const int d_ae = G.ds(a, e), d_be = G.ds(b, e), d_ce = G.ds(c, e);
    const int d_bf = G.ds(b, f), d_cf = G.ds(c, f), d_df = G.ds(d, f);
    const unsigned base = (jn + (unsigned)k) * 8u;
    if (k > j + 1) take((long long)d_ce + d_df - d_cd - d_ef, base + 2u);
    if (!(i == 0 && k == n - 1)) take((long long)d_ae + d_bf - d_ab - d_ef, base + 3u);
    take((long long)d_ac + d_be + d_df - old3, base + 4u);
    take((long long)d_ad + d_be + d_cf - old3, base + 5u);
    take((long long)d_ad + d_ce + d_bf - old3, base + 6u);
    take((long long)d_ae + d_bd + d_cf - old3, base + 7u);
    evals += 4 + (k > j + 1) + !(i == 0 && k == n - 1);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long od = __shfl_xor_sync(FULL, bd, o);
    const unsigned oo = __shfl_xor_sync(FULL, bo, o);
    if (od < bd || (od == bd && oo < bo)) { bd = od; bo = oo; }
  }
  return bd < 0 ? row_key(bd, bo) : kGridNoKey;
}

__device__ __forceinline__ void grid_reverse(int* tour, int lo, int hi) {
  const int half = (hi - lo + 1) >> 1;
  for (int q = threadIdx.x; q < half; q += blockDim.x) {
    const int x = tour[lo + q], y = tour[hi - q];
    tour[lo + q] = y;
    tour[hi - q] = x;
  }
}

// Applies a move with the whole CTA (ends with a barrier).
__device__ __forceinline__ void grid_apply(int* tour, const Move m) {
  if (m.c == 1 || m.c == 4 || m.c == 5 || m.c == 7) grid_reverse(tour, m.i + 1, m.j);
  if (m.c == 2 || m.c == 4 || m.c == 5 || m.c == 6) grid_reverse(tour, m.j + 1, m.k);
  __syncthreads();
  if (m.c == 3 || m.c == 5 || m.c == 6 || m.c == 7) {
    grid_reverse(tour, m.i + 1, m.k);
    __syncthreads();
  }
}

struct GridArgs {
  int32_t* tours;
  int num;
  int n;
  DistSrc ds;
  const int32_t* cand;
  const int32_t* cdist;
  int k, inner;
  int B;  // the reference's threads per tour
  long long max_iter;
  int32_t* status;
  long long* stats;
  long long budget;
};

template <bool CAND, bool MULTI>
__global__ void __launch_bounds__(kGridThreads) three_opt_grid_kernel(const GridArgs A) {
  extern __shared__ __align__(16) unsigned char gsm[];
  const int n = A.n, B = A.B, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = kGridThreads / 32;
  unsigned long long* rkey = reinterpret_cast<unsigned long long*>(gsm);  // n
  long long* vd = reinterpret_cast<long long*>(rkey + n);                  // B
  Move* vm = reinterpret_cast<Move*>(vd + kGridThreads);                   // B
  int* tour = reinterpret_cast<int*>(vm + kGridThreads);                   // n
  int* pos = tour + n;
  int* edge = pos + n;
  __shared__ int s_flag, s_sel;
  __shared__ unsigned long long s_evals;
  const int rows = CAND ? n : n - 2;  // anchors the reference scans
  GridTour G{tour, pos, edge, n, A.ds};
  const CandRow C{A.cand, A.cdist, A.k, A.inner};
  for (int r = blockIdx.x; r < A.num; r += gridDim.x) {
    int32_t* g = A.tours + (long long)r * n;
    if (tid == 0) { s_flag = 0; s_evals = 0; }
    for (int p = tid; p < n; p += kGridThreads) {
      tour[p] = g[p];
      pos[p] = -1;
    }
    __syncthreads();
    for (int p = tid; p < n; p += kGridThreads) {
      const int v = tour[p];
      if ((unsigned)v >= (unsigned)n || atomicExch(&pos[v], p) != -1) s_flag = 1;
    }
    __syncthreads();
    const bool bad = s_flag != 0;
    __syncthreads();
    if (bad) {
      if (tid == 0) {
        if (A.status) A.status[r] = TSPB_ERR_NOT_PERMUTATION;
        if (A.stats)
          for (int q = 0; q < 3; ++q) A.stats[(long long)r * 3 + q] = 0;
      }
      continue;
    }
    long long passes = 0, moves = 0, evals = 0;
    int err = TSPB_OK;
    const long long t0 = clock64();
    while (passes < A.max_iter) {
      if (tid == 0) s_flag = clock64() - t0 > A.budget;
      for (int p = tid; p < n; p += kGridThreads) {
        const int x = tour[p];
        pos[x] = p;
        edge[p] = A.ds(x, tour[p + 1 == n ? 0 : p + 1]);
      }
      for (int i = tid; i < n; i += kGridThreads) rkey[i] = kGridNoKey;
      __syncthreads();
      if (s_flag) {
        err = TSPB_ERR_BUDGET;
        break;
      }
      ++passes;
      // row bests
      if constexpr (CAND) {
        for (int i = wid; i < rows; i += NW) {
          const unsigned long long key = cand_row(G, C, i, evals);
          if (lane == 0) rkey[i] = key;
        }
      } else {
        for (int i = 0; i < rows; ++i)
          for (int j = i + 1 + wid; j <= n - 2; j += NW) {
            const unsigned long long key = exhaustive_row(G, i, j, evals);
            if (lane == 0 && key != kGridNoKey) atomicMin(&rkey[i], key);
          }
      }
      __syncthreads();
      // the B reference threads' bests: first row (in i order) holding the smallest delta
      if (tid < B) {
        long long bd = 0;
        int bi = -1;
        unsigned long long bk = kGridNoKey;
        for (int i = tid; i < rows; i += B) {
          const unsigned long long key = rkey[i];
          if (key == kGridNoKey) continue;
          const long long d = row_key_delta(key);
          if (d < bd) { bd = d; bi = i; bk = key; }
        }
        Move m{-1, -1, -1, 0};
        if (bi >= 0) {
          const unsigned order = (unsigned)(bk & ((1ull << kOrderBits) - 1));
          if constexpr (CAND) {
            m = cand_move(G, C, bi, order);
          } else {
            const unsigned jk = order >> 3;
            m = {bi, (int)(jk / (unsigned)n), (int)(jk % (unsigned)n), (int)(order & 7u)};
          }
        }
        vd[tid] = bd;
        vm[tid] = m;
      }
      __syncthreads();
      int applied = 0;
      if constexpr (!MULTI) {
        // pairwise halving down to 64, then slots 1..63 in order: strictly smaller wins
        for (int s = B / 2; s > 32; s >>= 1) {
          if (tid < s && vd[tid + s] < vd[tid]) {
            vd[tid] = vd[tid + s];
            vm[tid] = vm[tid + s];
          }
          __syncthreads();
        }
        if (tid == 0) {
          const int rem = B < 64 ? B : 64;
          for (int q = 1; q < rem; ++q)
            if (vd[q] < vd[0]) {
              vd[0] = vd[q];
              vm[0] = vm[q];
            }
        }
        __syncthreads();
        if (vd[0] < 0) {
          grid_apply(tour, vm[0]);
          applied = 1;
        }
      } else {
        const int max_moves = B < n / 2 ? B : n / 2;
        for (; applied < max_moves;) {
          if (tid == 0) {
            int bt = -1;
            long long bd = 0;
            for (int q = 0; q < B; ++q)
              if (vd[q] < bd) { bd = vd[q]; bt = q; }
            s_sel = bt;
            if (bt >= 0) vd[bt] = 0;
          }
          __syncthreads();
          const int sel = s_sel;
          if (sel < 0) break;
          const Move m = vm[sel];
          grid_apply(tour, m);
          ++applied;
          if (tid < B && vd[tid] < 0 && !(vm[tid].k < m.i || m.k < vm[tid].i)) vd[tid] = 0;
          __syncthreads();
        }
      }
      moves += applied;
      if (applied == 0) break;  // nothing improves: every further pass changes nothing
      __syncthreads();
    }
    __syncthreads();
    for (int p = tid; p < n; p += kGridThreads) g[p] = tour[p];
    const long long warp_evals = warp_sum(evals);
    if (lane == 0 && warp_evals) atomicAdd(&s_evals, (unsigned long long)warp_evals);
    __syncthreads();
    if (tid == 0) {
      if (A.status) A.status[r] = err;
      if (A.stats) {
        A.stats[(long long)r * 3 + 0] = passes;
        A.stats[(long long)r * 3 + 1] = moves;
        A.stats[(long long)r * 3 + 2] = (long long)s_evals;
      }
    }
    __syncthreads();
  }
}

static size_t grid_smem(int n) {
  return (size_t)8 * n + (size_t)kGridThreads * (sizeof(long long) + sizeof(Move)) + (size_t)12 * n;
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_three_opt_grid_threads(int32_t threads_per_block, int32_t n) {
  int v = threads_per_block < n ? threads_per_block : n;
  if (v < 1) v = 1;
  int p = 1;
  while (p * 2 <= v) p *= 2;
  return p > 256 ? 256 : p;
}

extern "C" int tspb_three_opt_grid(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist,
                                   int64_t dist_stride, const double* coords, const int32_t* cand,
                                   const int32_t* cand_dist, int32_t k, int32_t inner_k, int32_t multi_move,
                                   int32_t threads_per_block, int64_t max_iterations, int32_t* status, int64_t* stats,
                                   void* stream) {
  if (num_tours < 0 || n < 0 || max_iterations < 0 || threads_per_block <= 0 || k < 0 || inner_k < 0)
    return TSPB_ERR_ARG;
  if (num_tours == 0 || n < 4 || max_iterations == 0) {
    cudaStream_t st0 = reinterpret_cast<cudaStream_t>(stream);
    if (stats && num_tours > 0) TSPB_CUDA_CHECK(cudaMemsetAsync(stats, 0, sizeof(int64_t) * 3 * (size_t)num_tours, st0));
    if (status && num_tours > 0) TSPB_CUDA_CHECK(cudaMemsetAsync(status, 0, sizeof(int32_t) * (size_t)num_tours, st0));
    return TSPB_OK;
  }
  if (!tours || (!dist && !coords) || (dist && dist_stride < n)) return TSPB_ERR_ARG;
  const bool use_cand = k > 0;
  if (use_cand && (!cand || !cand_dist)) return TSPB_ERR_ARG;
  if (!use_cand && !multi_move) return TSPB_ERR_ARG;  // exhaustive one-move passes: tspb_three_opt
  if (!use_cand && n > kGridExhaustiveMaxN) return TSPB_ERR_UNSUPPORTED;
  if (use_cand && (k > 1024 || n > 65535)) return TSPB_ERR_UNSUPPORTED;
  if (!use_cand && (long long)n * n * 8 >= (1LL << kOrderBits)) return TSPB_ERR_UNSUPPORTED;
  const int inner = use_cand ? (inner_k > 0 && inner_k < k ? inner_k : k) : 0;
  const size_t smem = grid_smem(n);
  if (smem > (size_t)smem_optin() - 2048) return TSPB_ERR_UNSUPPORTED;
  GridArgs a{};
  a.tours = tours;
  a.num = num_tours;
  a.n = n;
  a.ds.dist = dist;
  a.ds.stride = dist_stride;
  a.ds.coords = reinterpret_cast<const double2*>(coords);
  a.cand = cand;
  a.cdist = cand_dist;
  a.k = k;
  a.inner = inner;
  a.B = tspb_three_opt_grid_threads(threads_per_block, n);
  a.max_iter = max_iterations;
  a.status = status;
  a.stats = reinterpret_cast<long long*>(stats);
  a.budget = watchdog_cycles();
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  auto kern = use_cand ? (multi_move ? three_opt_grid_kernel<true, true> : three_opt_grid_kernel<true, false>)
                       : three_opt_grid_kernel<false, true>;
  TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0, dev = 0, sms = 0;
  TSPB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGridThreads, smem));
  if (per_sm <= 0) return TSPB_ERR_UNSUPPORTED;
  TSPB_CUDA_CHECK(cudaGetDevice(&dev));
  TSPB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long grid = (long long)per_sm * sms < num_tours ? (long long)per_sm * sms : num_tours;
  kern<<<(int)grid, kGridThreads, smem, st>>>(a);
  return tspb_launch_status();
}
