// Device bodies of one GA generation shared by the single-run kernels (generation.cu)
// and the multi-instance batch kernels (batch.cu).
//
// Reference semantics reproduced bit for bit:
//   SelectionCPUTournament.select_batch    (tournament_selection.py:98-128)
//   CrossoverCPUPermPartiallyMapped         (pmx_crossover.py:49-171, open permutations)
//   MutationCPUPermInversion.mutate_batch   (inversion_mutation.py:65-99)
//   evaluate_tour_cpu                       (tour_cost.py:17-29)
#pragma once

#include "common.cuh"

namespace tspb {

// One generation's slice of the pre-drawn tape.
struct GenTapeSlice {
  const int32_t* tourn;  // [P][kt]
  const int32_t* cut_a;  // [P/2]
  const int32_t* cut_b;  // [P/2]
  const double* u;       // [P]
  const int32_t* inv_a;  // [P]
  const int32_t* inv_b;  // [P]
};

__device__ __forceinline__ int tournament_winner(const double* fit, const int32_t* c, int kt, int pop) {
  int best = c[0];
  if ((unsigned)best >= (unsigned)pop) best = 0;
  double bf = fit[best];
  for (int q = 1; q < kt; ++q) {
    const int v = c[q];
    if ((unsigned)v >= (unsigned)pop) continue;
    const double f = fit[v];
    if (f < bf) {
      bf = f;
      best = v;
    }
  }
  return best;
}

// Shared memory of offspring_row: inv_p2[n], child[n] ints and the in-segment bitmap.
__host__ __device__ inline size_t offspring_smem_bytes(int n) {
  return (size_t)8 * n + (size_t)((n + 31) / 32) * 4;
}

// Exclusive prefix sum of v over the CTA (blockDim a multiple of 32); `red` holds 32 ints.
__device__ __forceinline__ int block_exclusive_scan(int v, int* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();  // red may still be read by a previous scan
  if (lane == 31) red[wid] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int w = 0; w < nw; ++w) {
      const int t = red[w];
      red[w] = acc;
      acc += t;
    }
  }
  __syncthreads();
  return red[wid] + x - v;
}

// Order Crossover fill (order_crossover.py:52-83, open permutations): child[c1..c2]
// already holds p1's segment, whose genes are marked in `in_seg`. The free positions
// c2+1, ..., n-1, 0, ..., c1-1 form one run in that rotated order; they take, in order,
// the genes of p2 read from index c2+1 onward (wrapping) that are not in the segment.
// Each thread scans a contiguous stretch of the rotated p2; a CTA prefix count of kept
// genes gives every kept gene its free position. `red` holds 32 ints.
__device__ __forceinline__ void ox_fill(const int32_t* __restrict__ p2, int n, int c2, int* child,
                                        const unsigned* in_seg, int* red) {
  const int T = blockDim.x, tid = threadIdx.x;
  const int chunk = (n + T - 1) / T;
  const int t0 = min(tid * chunk, n), t1 = min(t0 + chunk, n);
  const int base = c2 + 1;  // <= n
  int cnt = 0;
  for (int t = t0; t < t1; ++t) {
    int idx = base + t;
    if (idx >= n) idx -= n;
    const int g = __ldg(p2 + idx);
    cnt += (in_seg[g >> 5] & (1u << (g & 31))) ? 0 : 1;
  }
  int m = block_exclusive_scan(cnt, red);
  for (int t = t0; t < t1; ++t) {
    int idx = base + t;
    if (idx >= n) idx -= n;
    const int g = __ldg(p2 + idx);
    if (in_seg[g >> 5] & (1u << (g & 31))) continue;
    int dst = base + m;
    if (dst >= n) dst -= n;
    child[dst] = g;
    ++m;
  }
}

// Parents of a child and whether the child equals each of them (filled when requested).
struct ChildOrigin {
  int parent[2];
  int same[2];
};

// Child `row` of one generation with the whole CTA: tournament winners (row pairs 2q, 2q+1
// share the cuts q; an odd last row copies its winner), crossover (PMX or OX), mutation
// when u < rate (inversion or swap), then the row and its closed-tour length are written to
// off_row / off_fit_row. `sm` holds offspring_smem_bytes(n) bytes. With `origin`, every
// thread also learns the parents and whether the child is identical to each. OX and swap
// draw exactly the numbers PMX and inversion draw (order_crossover.py:148-150,
// swap_mutation.py:86-93), so the tape is the same for every operator choice.
__device__ __forceinline__ void offspring_row(const int32_t* __restrict__ pop, const double* __restrict__ fit, int P,
                                              int n, int kt, const GenTapeSlice& tape, double rate, const DistSrc& ds,
                                              int row, int* sm, int32_t* __restrict__ off_row,
                                              double* __restrict__ off_fit_row, ChildOrigin* origin = nullptr,
                                              int crossover = TSPB_XOVER_PMX, int mutation = TSPB_MUT_INVERSION) {
  int* inv_p2 = sm;
  int* child = sm + n;
  unsigned* in_seg = reinterpret_cast<unsigned*>(sm + 2 * n);
  __shared__ int w[2];
  __shared__ long long red[32];
  __shared__ int scan_red[32];
  const int tid = threadIdx.x, T = blockDim.x;
  const int pairs = P >> 1;
  const int q = row >> 1, h = row & 1;
  const bool paired = row < 2 * pairs;
  if (tid < 2) {
    const int sel = paired ? 2 * q + (tid == 0 ? h : 1 - h) : row;
    w[tid] = tournament_winner(fit, tape.tourn + (long long)sel * kt, kt, P);
  }
  __syncthreads();
  const int32_t* p1 = pop + (long long)w[0] * n;
  const int32_t* p2 = pop + (long long)w[1] * n;
  if (!paired || n < 2) {
    for (int p = tid; p < n; p += T) child[p] = __ldg(p1 + p);
  } else if (crossover == TSPB_XOVER_OX) {
    int c1 = tape.cut_a[q], c2 = tape.cut_b[q];
    if (c1 > c2) {
      const int tmp = c1;
      c1 = c2;
      c2 = tmp;
    }
    const int words = (n + 31) >> 5;
    for (int wd = tid; wd < words; wd += T) in_seg[wd] = 0u;
    __syncthreads();
    for (int p = c1 + tid; p <= c2; p += T) {
      const int v1 = __ldg(p1 + p);
      child[p] = v1;
      atomicOr(&in_seg[v1 >> 5], 1u << (v1 & 31));
    }
    __syncthreads();
    ox_fill(p2, n, c2, child, in_seg, scan_red);
  } else {
    int c1 = tape.cut_a[q], c2 = tape.cut_b[q];
    if (c1 > c2) {
      const int tmp = c1;
      c1 = c2;
      c2 = tmp;
    }
    const int words = (n + 31) >> 5;
    for (int p = tid; p < n; p += T) child[p] = -1;
    for (int wd = tid; wd < words; wd += T) in_seg[wd] = 0u;
    __syncthreads();
    for (int p = tid; p < n; p += T) {
      inv_p2[__ldg(p2 + p)] = p;
      if (p >= c1 && p <= c2) {
        const int v1 = __ldg(p1 + p);
        child[p] = v1;
        atomicOr(&in_seg[v1 >> 5], 1u << (v1 & 31));
      }
    }
    __syncthreads();
    const int seg_len = c2 - c1 + 1;
    for (int idx = c1 + tid; idx <= c2; idx += T) {
      const int val = __ldg(p2 + idx);
      if (in_seg[val >> 5] & (1u << (val & 31))) continue;
      int pos = idx, steps = 0;
      while (pos >= c1 && pos <= c2 && steps <= seg_len) {
        pos = inv_p2[__ldg(p1 + pos)];
        ++steps;
      }
      if (pos < c1 || pos > c2) child[pos] = val;
    }
    __syncthreads();
    for (int p = tid; p < n; p += T)
      if (child[p] == -1) child[p] = __ldg(p2 + p);
  }
  __syncthreads();
  // mutation of this child
  if (tape.u[row] < rate) {
    const int a = tape.inv_a[row], b = tape.inv_b[row];
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    if (mutation == TSPB_MUT_SWAP) {
      if (tid == 0 && lo >= 0 && hi < n) {
        const int x = child[a];
        child[a] = child[b];
        child[b] = x;
      }
    } else if (lo >= 0 && hi < n) {
      const int half = (hi - lo + 1) >> 1;
      for (int t = tid; t < half; t += T) {
        const int x = child[lo + t], y = child[hi - t];
        child[lo + t] = y;
        child[hi - t] = x;
      }
    }
  }
  __syncthreads();
  // write out and reduce the closed-tour length (exact int64, one float64 at the end)
  long long acc = 0;
  int diff1 = 0, diff2 = 0;
  for (int p = tid; p < n; p += T) {
    const int v = child[p];
    off_row[p] = v;
    acc += ds(v, child[p + 1 == n ? 0 : p + 1]);
    if (origin) {
      diff1 |= v != __ldg(p1 + p);
      diff2 |= v != __ldg(p2 + p);
    }
  }
  acc = block_sum(acc, red);
  if (tid == 0) *off_fit_row = n <= 1 ? 0.0 : (double)acc;
  if (origin) {
    origin->parent[0] = w[0];
    origin->parent[1] = w[1];
    origin->same[0] = !__syncthreads_or(diff1);
    origin->same[1] = !__syncthreads_or(diff2);
  }
}

// Closed-tour length of one row by one warp (exact int64 sum, one float64 at the end).
__device__ __forceinline__ double warp_tour_length(const int32_t* __restrict__ t, int n, const DistSrc& ds) {
  const int lane = threadIdx.x & 31;
  long long acc = 0;
  for (int p = lane; p < n; p += 32) acc += ds(t[p], t[p + 1 == n ? 0 : p + 1]);
  acc = warp_sum(acc);
  return n <= 1 ? 0.0 : (double)acc;
}

}  // namespace tspb
