// Per-tour body of the candidate-mode 2-opt rescan (best / first), shared by the
// one-CTA-per-tour kernel and the persistent multi-instance batch kernel.
//
// Same semantics as the reference scan (src/algorithms/strategies/local_search/two_opt.py:
// pair order :347-367, gains :237-245, best :386-440, first :442-489, passes :565-595),
// arranged so that one pass keeps as many independent loads in flight as possible:
//
// - the tour is held position- and node-indexed: tour[p], pos[a], succ[a] and
//   eout[a] = d(a, succ[a]); the gain of entry (i, r) with a = tour[i], c = N_k[a][r] is
//   (d(a,c) - eout[a]) + (d(succ[a], succ[c]) - eout[c]);
// - the k-NN table and d(a, c) come packed as one u32 per entry (c | d(a,c) << 16) when
//   both fit 16 bits, so the whole per-instance table (80 KB at n=1000, k=20) stays in L1;
// - each thread evaluates U entries per round with their loads issued back to back
//   (k-NN word -> shared-memory lookups -> one L2 gather of d(succ[a], succ[c]), or an
//   FP64 rebuild from coordinates when the instance has no matrix).
//
// best keeps a per-thread (gain, i*k + r) minimum and reduces once per pass. first
// publishes improving indices with a shared atomicMin; each thread stops scanning as soon
// as the published minimum lies below all of its remaining entries (no barrier per round),
// and one barrier at the end of the scan makes the minimum the pass's first improving entry.
//
// best with incremental row keys (INC, grouped layout, reverse k-NN index): every row keeps
// the minimum key of its improving entries. After a move with window [bi, bj] only the rows
// in the window and the earlier rows with a candidate in the window can change (rows after
// bj see the window's candidates at invalid positions), so a pass recomputes those rows
// and reduces the row keys; long windows take a full recomputation. It computes fewer
// gains but adds barriers and a row-key reduction to every pass, so the batch engine's
// tuner selects it only where it measures faster.
//
// first with the reverse k-NN index (incremental restart): the reference restarts every
// pass at entry 0. After a move with window [bi, bj] (the first improving entry was in row
// bi, so every entry before it was non-improving), an entry (i, r) of a row i < bi keeps
// a = t[i], succ[a] and eout[a]; it changes only when its candidate c lies in positions
// [bi, bj], where pos/succ/eout of c may have changed. The next pass therefore evaluates
// just those affected entries (found through the reverse index) and, when none improves,
// scans from row bi on: the first improving entry it finds is the reference's.
//
// best over a CTA pair (CL = 2, a thread-block cluster of two CTAs; grouped layout): both
// CTAs hold the whole tour state and apply every move; CTA r scans the rounds r, r + 2, ...
// of each pass, and the two per-CTA minima meet through distributed shared memory (one
// cluster barrier per pass), so both take the same move. The watchdog flags of both CTAs
// travel with the minima, so both stop together.
#pragma once

#include <cooperative_groups.h>

// First mode's incremental restart checks the entries that point into the last move's
// window (about 30 warp instructions per window position) instead of rescanning the rows
// before it (about 9 per row); it is taken when RATIO x window length <= the move's row.
#ifndef TSPB_RESTART_RATIO
#define TSPB_RESTART_RATIO 3
#endif

#include "two_opt.cuh"

namespace tspb {

struct ScanSmem {
  unsigned long long red64[32];
  long long redll[32];
  long long total;  // first (and incremental best): valid entries of the current tour, kept exact
  unsigned first;
  int nlist;        // incremental best: rows to recompute in this pass
  int bad;
  int stop;
  unsigned long long xkey[2];  // CTA pair: this CTA's pass minimum (by pass parity)
  int xstop[2];                // CTA pair: this CTA's watchdog flag of that pass
  long long xcnt[2];           // CTA pair: this CTA's pair and gain counts at exit
};

template <int THREADS>
struct ScanMinBlocks {
  static constexpr int value = THREADS == 64 ? 16 : THREADS == 128 ? 8 : THREADS == 256 ? 4 : THREADS == 512 ? 2 : 1;
};

// Bytes of tour state per tour: tour, pos, succ, eout (+ per-row valid counts for first
// when it counts pairs; best with incremental row keys adds the keys, valid counts and a
// row list).
__host__ __device__ inline size_t scan_tour_state_bytes(int n, int mode, bool incremental = false, bool count = true) {
  if (mode == TSPB_MODE_FIRST) return (size_t)(count ? 20 : 16) * (size_t)n;
  return (size_t)(incremental ? 30 : 16) * (size_t)n;
}

struct ScanTour {
  int32_t* g_tour;        // the tour in global memory: read at entry, written back at exit
  unsigned char* arrays;  // scan_tour_state_bytes(n, mode) bytes (shared memory or workspace)
  int n, k;
  DistSrc ds;
  const uint32_t* packed;  // c | d(a, c) << 16 per entry, or nullptr
  const int32_t* cand;
  const int32_t* cand_dist;
  long long max_iter;
  int32_t* status;   // optional: TSPB status of this tour
  long long* stats;  // optional: passes, pairs, moves, evaluated gains
  int accumulate;    // 1: stats are added to the slot and only an error is stored in status
                     // (sticky across launches); 0: both are overwritten
  int32_t* moved;    // optional: 1 when at least one move was applied, else 0
  uint8_t* converged;  // optional: 1 when the refinement ended on a pass without an improving
                       // move (the tour is then a fixed point of any further refinement)
  const int32_t* rev_off = nullptr;  // optional (first mode): CSR reverse k-NN index, n + 1 offsets
  const int32_t* rev_idx = nullptr;  // flat entries a * k + r grouped by candidate node
  double* cost = nullptr;  // optional: the refined tour's length (exact int64 sum of eout, as float64)
  long long budget = BUDGET_CYCLES;  // watchdog: SM cycles before the tour ends with TSPB_ERR_BUDGET
  int symmetric = 0;  // 1: d(a, b) == d(b, a); a move's out-edges come from the old ones (below)
};

// k-NN table layouts of scan_tour: plain int32 candidates (+ optional distances), packed
// words with round-robin entries, and packed words with each thread's U entries taken
// contiguously from one row (needs k % U == 0): the row's a, succ[a], eout[a] are read
// once per U entries and the U words arrive in one vector load.
enum ScanLayout { SCAN_PLAIN = 0, SCAN_PACKED = 1, SCAN_GROUPED = 2 };

template <int U>
__device__ __forceinline__ void load_words(const uint32_t* p, uint32_t (&w)[U]) {
  if constexpr (U == 4) {
    const uint4 v = __ldg(reinterpret_cast<const uint4*>(p));
    w[0] = v.x;
    w[1] = v.y;
    w[2] = v.z;
    w[3] = v.w;
  } else if constexpr (U == 2) {
    const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
    w[0] = v.x;
    w[1] = v.y;
  } else {
#pragma unroll
    for (int u = 0; u < U; ++u) w[u] = __ldg(p + u);
  }
}

// Refines one tour with the whole CTA. Every thread of the CTA must call it.
//
// COUNT: first mode (and incremental best) keeps every row's valid-pair count so that
// stats[1] holds the reference's pair count. No decision of the scan reads these counts,
// and refreshing them after a move visits every candidate of every row in the reversed
// window, so a caller that passes no stats runs the COUNT = false instance (or, with
// COUNT = true, skips the refresh at run time): same moves, same tours.
//
// SYM: the symmetric-distance refresh after a move is compiled in (used when T.symmetric
// is set). The batch engine compiles it out: its large CTAs cover most windows in one round
// of distance reads, and the extra code measured slower there.
template <int MODE, int THREADS, int U, int LAYOUT, bool INC = false, bool COUNT = true, int CL = 1, bool SYM = true>
__device__ __forceinline__ void scan_tour(const ScanTour T, ScanSmem& S) {
  constexpr bool PACKED = LAYOUT != SCAN_PLAIN;
  constexpr bool GROUPED = LAYOUT == SCAN_GROUPED;
  static_assert(CL == 1 || (CL == 2 && MODE == TSPB_MODE_BEST && GROUPED && !INC),
                "a CTA pair runs best mode on the grouped layout only");
  const unsigned rank = CL > 1 ? cooperative_groups::this_cluster().block_rank() : 0u;
  const int n = T.n, k = T.k, rows = n - 2;
  const int tid = threadIdx.x;
  int32_t* g_tour = T.g_tour;
  int* tour = reinterpret_cast<int*>(T.arrays);
  int* pos = tour + n;
  int* succ = pos + n;
  int* eout = succ + n;
  // INC: the caller gives the reverse index; per-row minimum keys (8-byte aligned at 16n),
  // valid counts and the row list follow the tour state
  constexpr bool inc_best = MODE == TSPB_MODE_BEST && GROUPED && INC;
  unsigned long long* rkey = reinterpret_cast<unsigned long long*>(eout + n);
  int* rcnt = inc_best ? reinterpret_cast<int*>(rkey + n) : eout + n;  // valid entries per row (position)
  uint16_t* rlist = reinterpret_cast<uint16_t*>(rcnt + n);
  constexpr bool track_rows_ct = COUNT && (MODE == TSPB_MODE_FIRST || inc_best);
  const bool track_rows = track_rows_ct && T.stats != nullptr;
  const DistSrc ds = T.ds;
  const uint32_t* __restrict__ packed = T.packed;
  const int32_t* __restrict__ cand = T.cand;
  const int32_t* __restrict__ cdist = T.cand_dist;
  const int32_t* __restrict__ dist = T.ds.dist;
  const unsigned stride = (unsigned)T.ds.stride;

  if (tid == 0) {
    S.bad = 0;
    S.stop = 0;
    S.total = 0;
  }
  for (int p = tid; p < n; p += THREADS) {
    tour[p] = g_tour[p];
    pos[p] = -1;
  }
  __syncthreads();
  for (int p = tid; p < n; p += THREADS) {
    const int v = tour[p];
    if ((unsigned)v >= (unsigned)n || atomicExch(&pos[v], p) != -1) S.bad = 1;
  }
  __syncthreads();
  if (S.bad) {
    if (tid == 0) {
      if (T.moved) *T.moved = 0;
      if (T.converged) *T.converged = 0;
      if (T.status) *T.status = TSPB_ERR_NOT_PERMUTATION;
      if (T.stats && !T.accumulate)
        for (int q = 0; q < 4; ++q) T.stats[q] = 0;
    }
    __syncthreads();  // every thread has read S.bad before the caller reuses S
    return;
  }
  for (int p = tid; p < n; p += THREADS) {
    const int x = tour[p], y = tour[p + 1 == n ? 0 : p + 1];
    succ[x] = y;
    eout[x] = ds(x, y);
  }
  __syncthreads();

  // Valid entries of row i (the pairs the reference scan evaluates for that row).
  auto row_count = [&](int i) -> int {
    const int a = tour[i];
    const int lo = i + 2, span = n - (i == 0) - lo;
    int c = 0;
    for (int r0 = 0; r0 < k; r0 += 4) {
      int cc[4];
      if constexpr (GROUPED && U % 4 == 0) {  // k % 4 == 0 and a 16-byte aligned table
        uint32_t w[4];
        load_words<4>(packed + ((unsigned)a * (unsigned)k + (unsigned)r0), w);
#pragma unroll
        for (int u = 0; u < 4; ++u) cc[u] = (int)(w[u] & 0xffffu);
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const unsigned ar = (unsigned)a * (unsigned)k + (unsigned)(r0 + u);
          cc[u] = r0 + u < k ? (PACKED ? (int)(__ldg(packed + ar) & 0xffffu) : __ldg(cand + ar)) : -1;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if ((unsigned)cc[u] < (unsigned)n) c += (unsigned)(pos[cc[u]] - lo) < (unsigned)span;
    }
    return c;
  };
  if (track_rows) {
    long long sum = 0;
    for (int i = tid; i < n; i += THREADS) {
      const int v = i < rows ? row_count(i) : 0;
      rcnt[i] = v;
      sum += v;
    }
    sum = warp_sum(sum);
    if ((tid & 31) == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&S.total), (unsigned long long)sum);
    __syncthreads();
  }

  const int E = rows * k;
  constexpr int STEP = THREADS * U;
  const int sq = STEP / k, sr = STEP - (STEP / k) * k;
  const int g_row0 = (tid * U) / k, g_col0 = tid * U - g_row0 * k;  // grouped layout: first entry
  long long passes = 0, moves = 0, my_pairs = 0, my_eval = 0;
  int err = TSPB_OK;
  bool converged = false;  // the last pass found no improving move: a local optimum
  const long long t_start = clock64();
  const bool incremental = MODE == TSPB_MODE_FIRST && T.rev_off != nullptr && T.rev_idx != nullptr;
  // entry e = a * k + r of the reverse index -> a, as a multiply-high by ceil(2^32 / k):
  // exact for every e < n k when n k k < 2^32 (else a plain division)
  const unsigned kmag = (unsigned)(((1ull << 32) + (unsigned)k - 1) / (unsigned)k);
  const bool kmag_exact = (unsigned long long)n * (unsigned)k * (unsigned)k < (1ull << 32);
  auto entry_node = [&](int e) -> int {
    return kmag_exact ? (int)__umulhi((unsigned)e, kmag) : e / k;
  };
  int win_lo = -1, win_hi = -1;  // window [bi, bj] of the last move (incremental first mode)

  while (passes < T.max_iter) {
    if (tid == 0) {
      if (clock64() - t_start > T.budget) S.stop = TSPB_ERR_BUDGET;
      S.first = NO_IDX;
    }
    __syncthreads();
    if (CL == 1 && S.stop) {  // a CTA pair stops only after exchanging its flags (below)
      err = S.stop;
      break;
    }
    ++passes;
    if (track_rows && tid == 0) my_pairs += S.total;
    int bgain = 0;            // best: smallest gain of this thread (strictly below 0 to count)
    unsigned bidx = NO_IDX;   // and its scan index (first in thread order wins ties)
    int cnt = 0, evals = 0;
    int start_row = 0;        // first row of this pass's scan
    bool found = false;       // the affected entries already hold the first improving one
    if (incremental && win_lo >= 0 && TSPB_RESTART_RATIO * (win_hi - win_lo + 1) <= win_lo) {
      // affected entries of rows < win_lo: candidate c at a position of the window
      const int lane = tid & 31, wid = tid >> 5;
      constexpr int NW = THREADS / 32;
      for (int q = win_lo + wid; q <= win_hi; q += NW) {
        const int c = tour[q];
        const int s0 = __ldg(T.rev_off + c), s1 = __ldg(T.rev_off + c + 1);
        const int sc = succ[c], ec = eout[c];
        for (int sx = s0 + lane; sx < s1; sx += 32) {
          const int e = __ldg(T.rev_idx + sx);
          const int a = entry_node(e);
          const int i = pos[a];
          if (i >= win_lo) continue;  // rows from win_lo on are scanned below
          if ((unsigned)(q - (i + 2)) >= (unsigned)(n - (i == 0) - (i + 2))) continue;
          const int dac = PACKED ? (int)(__ldg(packed + e) >> 16) : (cdist ? __ldg(cdist + e) : ds(a, c));
          const int lbe = (dac - eout[a]) - ec;
          if (lbe >= 0) continue;  // cannot improve whatever d(succ a, succ c) is
          ++evals;
          const int sa = succ[a];
          const int dbd = dist ? __ldcg(dist + ((unsigned)sa * stride + (unsigned)sc)) : ds(sa, sc);
          if (lbe + dbd < 0) atomicMin(&S.first, (unsigned)(i * k + (e - a * k)));
        }
      }
      __syncthreads();
      found = S.first != NO_IDX;
      start_row = win_lo;
    }
    if constexpr (inc_best) {
      // minimum improving key of the U entries of row gi starting at column gr
      auto group_key = [&](int gi, int gr) -> unsigned long long {
        const int a = tour[gi];
        uint32_t w[U];
        load_words<U>(packed + ((unsigned)a * (unsigned)k + (unsigned)gr), w);
        const int sa = succ[a], ea = eout[a];
        const int lo = gi + 2;
        const unsigned span = (unsigned)(n - (gi == 0) - lo);
        bool ok[U];
        int c[U], sc[U], dbd[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          c[u] = (int)(w[u] & 0xffffu);
          ok[u] = (unsigned)c[u] < (unsigned)n && (unsigned)(pos[c[u]] - lo) < span;
          if (ok[u]) {
            sc[u] = succ[c[u]];
            ok[u] = ((int)(w[u] >> 16) - ea) - eout[c[u]] < 0;  // only improving entries hold keys
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) dbd[u] = dist ? __ldcg(dist + ((unsigned)sa * stride + (unsigned)sc[u])) : ds(sa, sc[u]);
        unsigned long long key = NO_KEY;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (!ok[u]) continue;
          ++evals;
          const int gain = ((int)(w[u] >> 16) - ea) + (dbd[u] - eout[c[u]]);
          if (gain < 0) {
            const unsigned long long kk = gain_key(gain, (unsigned)(gi * k + gr + u));
            key = kk < key ? kk : key;
          }
        }
        return key;
      };
      constexpr unsigned long long DIRTY = NO_KEY - 1;  // never a key: keys hold negative gains
      const int G = k / U;
      const bool full = win_lo < 0 || 2LL * (win_hi - win_lo + 1) * (k + 1) > (long long)rows;
      if (full) {
        for (int i = tid; i < rows; i += THREADS) rkey[i] = NO_KEY;
        __syncthreads();
        for (int it = tid; it < rows * G; it += THREADS) {
          const int gi = it / G, gr = (it - gi * G) * U;
          const unsigned long long key = group_key(gi, gr);
          if (key != NO_KEY) atomicMin(&rkey[gi], key);
        }
      } else {
        if (tid == 0) S.nlist = 0;
        const int r_hi = win_hi < rows - 1 ? win_hi : rows - 1;
        for (int i = win_lo + tid; i <= r_hi; i += THREADS) rkey[i] = DIRTY;
        const int lane = tid & 31, wid = tid >> 5;
        constexpr int NW = THREADS / 32;
        for (int q = win_lo + wid; q <= win_hi; q += NW) {
          const int c = tour[q];
          const int s0 = __ldg(T.rev_off + c), s1 = __ldg(T.rev_off + c + 1);
          for (int sx = s0 + lane; sx < s1; sx += 32) {
            const int i = pos[entry_node(__ldg(T.rev_idx + sx))];
            if (i < win_lo) rkey[i] = DIRTY;
          }
        }
        __syncthreads();
        // compaction with one shared atomic per warp (every lane takes every round)
        for (int i0 = 0; i0 < rows; i0 += THREADS) {
          const int i = i0 + tid;
          const bool d = i < rows && rkey[i] == DIRTY;
          const unsigned m = __ballot_sync(0xffffffffu, d);
          int base = 0;
          if (lane == 0 && m) base = atomicAdd(&S.nlist, __popc(m));
          base = __shfl_sync(0xffffffffu, base, 0);
          if (d) {
            rkey[i] = NO_KEY;
            rlist[base + __popc(m & ((1u << lane) - 1u))] = (uint16_t)i;
          }
        }
        __syncthreads();
        const int items = S.nlist * G;
        for (int it = tid; it < items; it += THREADS) {
          const int q = it / G;
          const int gi = rlist[q], gr = (it - q * G) * U;
          const unsigned long long key = group_key(gi, gr);
          if (key != NO_KEY) atomicMin(&rkey[gi], key);
        }
      }
      __syncthreads();
      unsigned long long key = NO_KEY;
      for (int i = tid; i < rows; i += THREADS) {
        const unsigned long long v = rkey[i];
        key = v < key ? v : key;
      }
      if (key != NO_KEY) {
        bgain = key_gain(key);
        bidx = (unsigned)key;
      }
      found = true;  // skip the per-pass scan below
    }
    if (found) {
      // nothing to scan: first mode's smallest improving affected entry is the first of the
      // pass; incremental best already holds this thread's share of the row keys
    } else if constexpr (GROUPED) {
      // entries [e0 + tid*U, e0 + tid*U + U) of round e0 lie in row gi, columns gr..gr+U-1;
      // a CTA pair takes alternate rounds
      int gi = g_row0 + start_row, gr = g_col0;
      int e_first = start_row * k;
      if constexpr (CL > 1) {
        e_first += (int)rank * STEP;
        const int eb0 = e_first + tid * U;
        gi = eb0 / k;
        gr = eb0 - gi * k;
      }
      for (int e0 = e_first; e0 < E; e0 += CL * STEP) {
        const int eb = e0 + tid * U;
        if (eb < E) {
          const int a = tour[gi];
          uint32_t w[U];
          load_words<U>(packed + ((unsigned)a * (unsigned)k + (unsigned)gr), w);
          const int sa = succ[a], ea = eout[a];
          const int lo = gi + 2;
          const unsigned span = (unsigned)(n - (gi == 0) - lo);
          bool ok[U];
          int c[U], sc[U], lb[U];
          const int bound = MODE == TSPB_MODE_BEST ? bgain : 0;
#pragma unroll
          for (int u = 0; u < U; ++u) {
            c[u] = (int)(w[u] & 0xffffu);
            ok[u] = (unsigned)c[u] < (unsigned)n && (unsigned)(pos[c[u]] - lo) < span;
            if (MODE == TSPB_MODE_BEST) cnt += ok[u];
            if (ok[u]) {
              sc[u] = succ[c[u]];
              // gain >= lb (the gathered distance is >= 0): an entry whose lb cannot beat
              // this thread's bound is settled without its L2 gather
              lb[u] = ((int)(w[u] >> 16) - ea) - eout[c[u]];
              ok[u] = lb[u] < bound;
            }
          }
          int dbd[U];
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (ok[u]) dbd[u] = dist ? __ldcg(dist + ((unsigned)sa * stride + (unsigned)sc[u])) : ds(sa, sc[u]);
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            ++evals;
            const int gain = lb[u] + dbd[u];
            if (MODE == TSPB_MODE_BEST) {
              if (gain < bgain) {
                bgain = gain;
                bidx = (unsigned)(eb + u);
              }
            } else if (gain < 0) {
              atomicMin(&S.first, (unsigned)(eb + u));
            }
          }
        }
        if constexpr (CL > 1) {
          gr += (CL * STEP) % k;
          gi += (CL * STEP) / k;
        } else {
          gr += sr;
          gi += sq;
        }
        if (gr >= k) {
          gr -= k;
          ++gi;
        }
        // first: no barrier per round; a thread stops once an improving index below all of
        // its remaining entries (>= e0 + STEP) is known. S.first only decreases, so every
        // entry below the pass's final minimum is still evaluated by its thread.
        if (MODE == TSPB_MODE_FIRST && *reinterpret_cast<volatile unsigned*>(&S.first) < (unsigned)(e0 + STEP)) break;
      }
    } else {
    int ri[U], rr[U], ee[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      ee[u] = start_row * k + u * THREADS + tid;
      ri[u] = ee[u] / k;
      rr[u] = ee[u] - ri[u] * k;
    }
    for (int e0 = start_row * k; e0 < E; e0 += STEP) {
      int a[U], c[U], cd[U];
#pragma unroll
      for (int u = 0; u < U; ++u) a[u] = ee[u] < E ? tour[ri[u]] : -1;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        c[u] = -1;
        if (a[u] < 0) continue;
        const unsigned ar = (unsigned)a[u] * (unsigned)k + (unsigned)rr[u];
        if (PACKED) {
          const uint32_t w = __ldg(packed + ar);
          c[u] = (int)(w & 0xffffu);
          cd[u] = (int)(w >> 16);
        } else {
          c[u] = __ldg(cand + ar);
          cd[u] = cdist ? __ldg(cdist + ar) : -1;
        }
      }
      bool ok[U];
      int sa[U], sc[U], lb[U];
      const int bound = MODE == TSPB_MODE_BEST ? bgain : 0;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        ok[u] = false;
        if ((unsigned)c[u] >= (unsigned)n) continue;
        const int i = ri[u];
        // j in (i + 1, lim): one unsigned range test
        ok[u] = (unsigned)(pos[c[u]] - (i + 2)) < (unsigned)(n - (i == 0) - (i + 2));
        if (MODE == TSPB_MODE_BEST) cnt += ok[u];
        if (ok[u]) {
          sa[u] = succ[a[u]];
          sc[u] = succ[c[u]];
          const int dac = (PACKED || cd[u] >= 0) ? cd[u] : ds(a[u], c[u]);
          lb[u] = (dac - eout[a[u]]) - eout[c[u]];  // gain >= lb: skip the gather when lb cannot win
          ok[u] = lb[u] < bound;
        }
      }
      int dbd[U];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (ok[u]) dbd[u] = dist ? __ldcg(dist + ((unsigned)sa[u] * stride + (unsigned)sc[u])) : ds(sa[u], sc[u]);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
        ++evals;
        const int gain = lb[u] + dbd[u];
        if (MODE == TSPB_MODE_BEST) {
          if (gain < bgain) {
            bgain = gain;
            bidx = (unsigned)ee[u];
          }
        } else if (gain < 0) {
          atomicMin(&S.first, (unsigned)ee[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        ee[u] += STEP;
        rr[u] += sr;
        ri[u] += sq;
        if (rr[u] >= k) {
          rr[u] -= k;
          ++ri[u];
        }
      }
      if (MODE == TSPB_MODE_FIRST && *reinterpret_cast<volatile unsigned*>(&S.first) < (unsigned)(e0 + STEP)) break;
    }
    }
    my_pairs += cnt;
    my_eval += evals;
    unsigned idx;
    if (MODE == TSPB_MODE_BEST) {
      const unsigned long long key = bidx == NO_IDX ? NO_KEY : gain_key(bgain, bidx);
      unsigned long long best = block_min(key, S.red64);
      if constexpr (CL > 1) {
        // the two CTAs' minima and watchdog flags meet through distributed shared memory;
        // slots alternate by pass, so one cluster barrier per pass suffices
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        const int slot = (int)(passes & 1);
        if (tid == 0) {
          S.xkey[slot] = best;
          S.xstop[slot] = S.stop;
        }
        cl.sync();
        const unsigned long long peer = *cl.map_shared_rank(&S.xkey[slot], rank ^ 1u);
        const int peer_stop = *cl.map_shared_rank(&S.xstop[slot], rank ^ 1u);
        best = peer < best ? peer : best;
        if (S.stop || peer_stop) {
          err = TSPB_ERR_BUDGET;
          break;
        }
      }
      if (best == NO_KEY) {
        converged = true;
        break;
      }
      idx = (unsigned)best;
    } else {
      __syncthreads();
      idx = S.first;
      if (idx == NO_IDX) {
        converged = true;
        break;
      }
    }
    const int bi = (int)(idx / (unsigned)k);
    const int br = (int)(idx - (unsigned)bi * (unsigned)k);
    const unsigned bar = (unsigned)tour[bi] * (unsigned)k + (unsigned)br;
    const int ca = PACKED ? (int)(__ldg(packed + bar) & 0xffffu) : __ldg(cand + bar);
    const int bj = pos[ca];
    if (bi < 0 || bj <= bi + 1 || bj >= n) {
      err = TSPB_ERR_RANGE;
      break;
    }
    __syncthreads();
    {
      const int lo = bi + 1, hi = bj, half = (hi - lo + 1) >> 1;
      for (int q = tid; q < half; q += THREADS) {
        const int x = tour[lo + q], y = tour[hi - q];
        tour[lo + q] = y;
        tour[hi - q] = x;
        pos[y] = lo + q;
        pos[x] = hi - q;
      }
    }
    __syncthreads();
    if (SYM && T.symmetric && bj - bi >= THREADS) {
      // Inside the reversed window [lo, hi] a node's new successor is its old predecessor,
      // so its new out-edge is that predecessor's old one (the same edge, read the other
      // way). Only the two edges the move creates come from the distance source. Chunks
      // run by increasing position: a chunk reads the old out-edges of positions p + 1
      // before its barrier and writes those of positions p after it, and later chunks read
      // only higher positions than any earlier chunk wrote. A window that one round of
      // distance reads covers (bj - bi < THREADS) keeps that round: a chunk's barrier
      // would cost more than the reads it saves.
      const int lo = bi + 1, hi = bj;
      for (int base = lo; base < hi; base += THREADS) {
        const int p = base + tid;
        int x = -1, y = 0, e = 0;
        if (p < hi) {
          x = tour[p];
          y = tour[p + 1];
          e = eout[y];
        }
        __syncthreads();
        if (x >= 0) {
          succ[x] = y;
          eout[x] = e;
        }
      }
      if (tid == 0) {  // the edge (tour[bi], tour[lo]) the move creates
        const int x = tour[bi], y = tour[lo];
        succ[x] = y;
        eout[x] = ds(x, y);
      }
      if (tid == THREADS - 1) {  // and (tour[hi], tour[hi + 1]), from another warp
        const int x = tour[hi], y = tour[hi + 1 == n ? 0 : hi + 1];
        succ[x] = y;
        eout[x] = ds(x, y);
      }
    } else {
      for (int p = bi + tid; p <= bj; p += THREADS) {
        const int x = tour[p], y = tour[p + 1 == n ? 0 : p + 1];
        succ[x] = y;
        eout[x] = ds(x, y);
      }
    }
    __syncthreads();
    ++moves;
    win_lo = bi;
    win_hi = bj;
    if (track_rows) {
      // Only rows [bi, bj] (and row 0 when bj == n-1) can change their valid count.
      const int r_hi = bj < rows - 1 ? bj : rows - 1;
      const bool row0 = bj == n - 1 && bi > 0;
      const int nr = r_hi - bi + 1 + (row0 ? 1 : 0);
      long long d = 0;
      for (int q = tid; q < nr; q += THREADS) {
        const int i = q < r_hi - bi + 1 ? bi + q : 0;
        const int v = row_count(i);
        d += v - rcnt[i];
        rcnt[i] = v;
      }
      d = warp_sum(d);
      if ((tid & 31) == 0 && d != 0) atomicAdd(reinterpret_cast<unsigned long long*>(&S.total), (unsigned long long)d);
    }
  }

  __syncthreads();
  if (rank == 0)
    for (int p = tid; p < n; p += THREADS) g_tour[p] = tour[p];
  long long tp = block_sum(my_pairs, S.redll);
  long long te = block_sum(my_eval, S.redll);
  if constexpr (CL > 1) {  // the pair's counts add up in CTA 0, which alone writes the results
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    if (tid == 0) {
      S.xcnt[0] = tp;
      S.xcnt[1] = te;
    }
    cl.sync();
    if (rank == 0) {
      tp += *cl.map_shared_rank(&S.xcnt[0], 1u);
      te += *cl.map_shared_rank(&S.xcnt[1], 1u);
    }
    cl.sync();  // CTA 1's shared memory stays valid until CTA 0 has read it
    if (rank != 0) return;
  }
  if (T.cost != nullptr) {  // eout[x] = d(x, succ[x]) of the final tour: its edges, each once
    long long len = 0;
    for (int p = tid; p < n; p += THREADS) len += eout[p];
    len = block_sum(len, S.redll);
    if (tid == 0) *T.cost = (double)len;
  }
  if (tid == 0) {
    if (T.moved) *T.moved = moves > 0 ? 1 : 0;
    if (T.converged) *T.converged = converged && err == TSPB_OK ? 1 : 0;
    if (T.status && (!T.accumulate || err != TSPB_OK)) *T.status = err;
    if (T.stats) {
      long long* st = T.stats;
      const long long v[4] = {passes, tp, moves, te};
      for (int q = 0; q < 4; ++q) st[q] = T.accumulate ? st[q] + v[q] : v[q];
    }
  }
  __syncthreads();  // S.redll is read by every thread before the caller reuses S
}

}  // namespace tspb
