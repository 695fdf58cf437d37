// Uneven multi-instance batch: many independent memetic-GA runs, one per instance, with
// instances of different sizes, advanced by one captured launch sequence per generation.
//
// Every run computes what the single-run kernels (generation.cu) compute for it alone:
// the same tape slices, survival order, elite rule, best tracking and patience
// (genetic_algorithm.py:618-706, 789-965; pipeline_steps.py:153-195). What is new is the
// data layout and the scheduling:
//
// - populations of all instances live in two flat buffers (pop[0], pop[1]) at
//   per-instance offsets; a run at generation g reads pop[g & 1] and writes pop[(g+1) & 1],
//   so the same launch sequence serves runs that are at different generations;
// - a per-instance control block {generation, state, stall, done} gates every kernel;
// - every row carries a "converged" bit: its last 2-opt refinement ended on a pass with no
//   improving move, so refining it again changes nothing and is skipped. The bit follows
//   the row through survival; a child identical to a converged parent inherits it;
// - an elite-edge fitness tie lets NumPy's unstable argsort choose which tied rows are
//   elites. When every tied row is converged, each choice refines only rows that do not
//   change, so the run goes on. Otherwise the run pauses: the host takes the argsort and
//   the run finishes that generation in the RESUME phase of a later launch sequence while
//   the other runs continue;
// - with local_search_stage="post_mutation" every child is refined before it is evaluated
//   (genetic_algorithm.py:333-343): the OFFSPRING phase of the same 2-opt kernel;
// - the elite 2-opt is one persistent launch per size bucket whose CTAs take
//   (instance, row) units from an atomic counter, largest instances first, with the
//   bucket's CTA size chosen by the host's autotuner.
//
// Instances with no distance matrix rebuild every distance from FP64 coordinates with the
// reference's EUC_2D rounding (DistSrc).
#include "generation.cuh"
#include "two_opt_scan.cuh"

namespace tspb {

__device__ __forceinline__ DistSrc inst_ds(const tspb_batch_instance& I) {
  DistSrc d;
  d.dist = I.dist;
  d.stride = I.dist_stride;
  d.coords = reinterpret_cast<const double2*>(I.coords);
  return d;
}

__device__ __forceinline__ int32_t* pop_buf(const tspb_batch& B, int parity) { return parity ? B.pop[1] : B.pop[0]; }
__device__ __forceinline__ double* fit_buf(const tspb_batch& B, int parity) { return parity ? B.fit[1] : B.fit[0]; }
__device__ __forceinline__ uint8_t* clean_buf(const tspb_batch& B, int parity) {
  return parity ? B.clean[1] : B.clean[0];
}

// State that a phase's steps run in.
__device__ __forceinline__ int phase_state(int phase) {
  return phase == TSPB_BATCH_PHASE_RESUME ? TSPB_BATCH_RESUME : TSPB_BATCH_RUN;
}

// Warp per row of pop[parity], INIT_ROWS rows per CTA, blockIdx.x the instance: every
// row's fitness. One CTA per instance would walk P tours with 8 warps, which for one run
// of 512 tours of 2000 cities took milliseconds on a single SM.
constexpr int INIT_ROWS = 8;
__global__ void __launch_bounds__(32 * INIT_ROWS) batch_fitness_kernel(const tspb_batch B, int parity) {
  const int i = blockIdx.x, P = B.P;
  const int r = blockIdx.y * INIT_ROWS + (threadIdx.x >> 5);
  if (r >= P) return;  // warp-uniform
  const tspb_batch_instance I = B.inst[i];
  const double f = warp_tour_length(pop_buf(B, parity) + I.pop_offset + (long long)r * I.n, I.n, inst_ds(I));
  if ((threadIdx.x & 31) == 0) fit_buf(B, parity)[(long long)i * P + r] = f;
}

// CTA per instance, after batch_fitness_kernel: the initial best (first minimum), the
// history's first entry and the control block.
__global__ void __launch_bounds__(256) batch_init_kernel(const tspb_batch B, int parity) {
  const int i = blockIdx.x;
  const tspb_batch_instance I = B.inst[i];
  const int P = B.P, n = I.n;
  const int32_t* pop = pop_buf(B, parity) + I.pop_offset;
  double* fit = fit_buf(B, parity) + (long long)i * P;
  __shared__ int best_row;
  if (threadIdx.x == 0) {
    int b = 0;
    for (int r = 1; r < P; ++r)
      if (fit[r] < fit[b]) b = r;  // first minimum (np.argmin)
    best_row = b;
    B.best_cost[i] = fit[b];
    B.history[(long long)i * (B.G + 1)] = fit[b];
    int* c = B.ctl + 4 * i;
    c[0] = 0;
    c[1] = B.G > 0 ? TSPB_BATCH_RUN : TSPB_BATCH_DONE;
    c[2] = 0;
    c[3] = 0;
  }
  __syncthreads();
  const int32_t* src = pop + (long long)best_row * n;
  for (int t = threadIdx.x; t < n; t += blockDim.x) B.best_tour[I.node_offset + t] = src[t];
}

// CTA per (item, child row).
__global__ void __launch_bounds__(256) batch_offspring_kernel(const tspb_batch B, const int32_t* __restrict__ items,
                                                              int max_n) {
  extern __shared__ int sm[];
  const int P = B.P;
  const int it = blockIdx.x / P, row = blockIdx.x - it * P;
  const int i = items[it];
  const int* c = B.ctl + 4 * i;
  if (c[1] != TSPB_BATCH_RUN) return;
  const long long g = c[0];
  const tspb_batch_instance I = B.inst[i];
  if (I.n > max_n) return;  // the host sizes shared memory for the bucket's largest n
  const int n = I.n, kt = B.kt, pairs = P >> 1;
  const long long slot = (long long)i * B.G + g;
  GenTapeSlice sl;
  sl.tourn = B.tape_tourn + slot * P * kt;
  sl.cut_a = B.tape_cut_a + slot * pairs;
  sl.cut_b = B.tape_cut_b + slot * pairs;
  sl.u = B.tape_u + slot * P;
  sl.inv_a = B.tape_inv_a + slot * P;
  sl.inv_b = B.tape_inv_b + slot * P;
  const int parity = (int)(g & 1);
  const DistSrc ds = inst_ds(I);
  const uint8_t* clean = B.clean[0] ? clean_buf(B, parity) + (long long)i * P : nullptr;
  ChildOrigin origin;
  offspring_row(pop_buf(B, parity) + I.pop_offset, fit_buf(B, parity) + (long long)i * P, P, n, kt, sl,
                B.mutation_rate, ds, row, sm, B.off + I.pop_offset + (long long)row * n,
                B.off_fit + (long long)i * P + row, clean ? &origin : nullptr, B.crossover, B.mutation);
  if (clean && threadIdx.x == 0)  // a child identical to a converged parent is converged
    B.off_clean[(long long)i * P + row] =
        (origin.same[0] && clean[origin.parent[0]]) || (origin.same[1] && clean[origin.parent[1]]) ? 1 : 0;
}

// The elite-edge tie of generation g, settled by the whole CTA right after the survival
// sort: key[r], idx[r] (shared memory, r < P) are the survivors' fitness and source index
// (< P: the population, else the offspring). Positions elite-1 and elite with equal fitness
// let NumPy's unstable argsort choose the elites. The run goes on when every survivor of
// that fitness is converged (any choice refines only rows that do not change), else it
// pauses for the host's argsort. The survivors are gathered in the same generation whether
// the run pauses or not (the gather serves RUN and PAUSED runs).
__device__ void survival_tie(const tspb_batch& B, int i, int g, int parity, const double* key, const int* idx) {
  const int P = B.P, e = B.elite;
  if (e <= 0 || e >= P) return;  // uniform: no edge
  const double fe = key[e - 1];
  const bool tie = key[e] == fe;
  bool ok = true;
  if (tie) {
    if (!B.clean[0]) {
      ok = false;
    } else {
      const uint8_t* ca = clean_buf(B, parity) + (long long)i * P;
      const uint8_t* cb = B.off_clean + (long long)i * P;
      for (int r = threadIdx.x; r < P; r += blockDim.x)
        if (key[r] == fe) ok = ok && (idx[r] < P ? ca[idx[r]] : cb[idx[r] - P]) != 0;
    }
  }
  const int settled = __syncthreads_and(ok ? 1 : 0);
  if (threadIdx.x == 0) {
    B.ties[(long long)i * B.G + g] = tie ? 1 : 0;
    if (tie && !settled) B.ctl[4 * i + 1] = TSPB_BATCH_PAUSED;
  }
}

// CTA per instance: the stable order of the 2P combined fitness values (old population
// first), i.e. (fitness, index) ascending, as the reference's lexsort keeps it; the first P
// indices go to order[], then the elite-edge tie. A bitonic sort of (fitness, index) pairs
// in shared memory, padded with +inf to the next power of two n2.
__global__ void batch_survival_rank_kernel(const tspb_batch B, int n2) {
  extern __shared__ __align__(16) unsigned char rank_sm[];
  double* key = reinterpret_cast<double*>(rank_sm);
  int* idx = reinterpret_cast<int*>(key + n2);
  const int i = blockIdx.x, P = B.P;
  const int* c = B.ctl + 4 * i;
  if (c[1] != TSPB_BATCH_RUN) return;
  const int parity = c[0] & 1;
  const double* fa = fit_buf(B, parity) + (long long)i * P;
  const double* fb = B.off_fit + (long long)i * P;
  const int count = 2 * P;
  for (int j = threadIdx.x; j < n2; j += blockDim.x) {
    key[j] = j < P ? fa[j] : (j < count ? fb[j - P] : __longlong_as_double(0x7ff0000000000000LL));
    idx[j] = j;
  }
  __syncthreads();
  for (int kk = 2; kk <= n2; kk <<= 1) {
    for (int jj = kk >> 1; jj > 0; jj >>= 1) {
      for (int t = threadIdx.x; t < n2; t += blockDim.x) {
        const int u = t ^ jj;
        if (u > t) {
          const double kt = key[t], ku = key[u];
          const int it = idx[t], iu = idx[u];
          const bool t_after_u = kt > ku || (kt == ku && it > iu);
          if (t_after_u == ((t & kk) == 0)) {
            key[t] = ku;
            key[u] = kt;
            idx[t] = iu;
            idx[u] = it;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int r = threadIdx.x; r < P; r += blockDim.x) B.order[(long long)i * P + r] = idx[r];
  survival_tie(B, i, c[0], parity, key, idx);
}

// The same order with n2 / 2 threads (64 <= n2 <= 2048): thread t holds positions t and
// t + n2/2 in registers. A compare-exchange at distance j pairs positions e and e ^ j: for
// j < 32 the partner sits in the same warp (lane ^ j, same slot), for j = n2/2 it is the
// thread's other slot, otherwise the pair meets in shared memory. Each position keeps the
// smaller (fitness, index) when it is the lower one of an ascending pair ((e & k) == 0) or
// the higher one of a descending pair, as in the shared-memory sort above.
__device__ __forceinline__ bool rank_after(double ka, int ia, double kb, int ib) {
  return ka > kb || (ka == kb && ia > ib);
}

__device__ __forceinline__ void rank_keep(double& k, int& id, double pk, int pid, int e, int p, int kk) {
  const bool asc = (e & kk) == 0;
  const bool want_small = (e < p) == asc;
  if (rank_after(k, id, pk, pid) == want_small) {  // the partner is the one this position keeps
    k = pk;
    id = pid;
  }
}

__global__ void batch_survival_rank_reg_kernel(const tspb_batch B, int n2) {
  extern __shared__ __align__(16) unsigned char rank_sm[];
  double* skey = reinterpret_cast<double*>(rank_sm);
  int* sidx = reinterpret_cast<int*>(skey + n2);
  const int i = blockIdx.x, P = B.P;
  const int* c = B.ctl + 4 * i;
  if (c[1] != TSPB_BATCH_RUN) return;  // uniform per CTA
  const int parity = c[0] & 1;
  const double* fa = fit_buf(B, parity) + (long long)i * P;
  const double* fb = B.off_fit + (long long)i * P;
  const int half = n2 >> 1, t = threadIdx.x, count = 2 * P;
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  auto load = [&](int e) { return e < P ? fa[e] : (e < count ? fb[e - P] : inf); };
  const int e0 = t, e1 = t + half;
  double k0 = load(e0), k1 = load(e1);
  int i0 = e0, i1 = e1;
  for (int kk = 2; kk <= n2; kk <<= 1) {
    for (int jj = kk >> 1; jj > 0; jj >>= 1) {
      if (jj == half) {  // e1 = e0 ^ half: both in this thread (kk == n2, ascending)
        if (rank_after(k0, i0, k1, i1)) {
          const double tk = k0;
          const int ti = i0;
          k0 = k1;
          i0 = i1;
          k1 = tk;
          i1 = ti;
        }
      } else if (jj < 32) {
        const double p0 = __shfl_xor_sync(FULL, k0, jj), p1 = __shfl_xor_sync(FULL, k1, jj);
        const int q0 = __shfl_xor_sync(FULL, i0, jj), q1 = __shfl_xor_sync(FULL, i1, jj);
        rank_keep(k0, i0, p0, q0, e0, e0 ^ jj, kk);
        rank_keep(k1, i1, p1, q1, e1, e1 ^ jj, kk);
      } else {
        skey[e0] = k0;
        sidx[e0] = i0;
        skey[e1] = k1;
        sidx[e1] = i1;
        __syncthreads();
        const double p0 = skey[e0 ^ jj], p1 = skey[e1 ^ jj];
        const int q0 = sidx[e0 ^ jj], q1 = sidx[e1 ^ jj];
        __syncthreads();  // every partner read before the next stage writes
        rank_keep(k0, i0, p0, q0, e0, e0 ^ jj, kk);
        rank_keep(k1, i1, p1, q1, e1, e1 ^ jj, kk);
      }
    }
  }
  if (e0 < P) {  // half >= P: slot 1 is never a survivor
    B.order[(long long)i * P + e0] = i0;
    skey[e0] = k0;  // the sorted survivors for the tie check (every earlier read is behind a barrier)
    sidx[e0] = i0;
  }
  __syncthreads();
  survival_tie(B, i, c[0], parity, skey, sidx);
}

// CTA per (instance, survivor): new_pop[r] = combined[order[r]] with its fitness and
// converged bit. A run the rank kernel just paused is gathered too (the host's argsort
// reads the survivors); a run still waiting for the host is gathered again in later
// replays from the same unchanged order, population and offspring, which rewrites the
// same rows.
__global__ void __launch_bounds__(128) batch_survival_gather_kernel(const tspb_batch B) {
  const int P = B.P;
  const int i = blockIdx.x / P, r = blockIdx.x - i * P;
  const int* c = B.ctl + 4 * i;
  if (c[1] != TSPB_BATCH_RUN && c[1] != TSPB_BATCH_PAUSED) return;
  const int g = c[0], parity = g & 1;
  const tspb_batch_instance I = B.inst[i];
  const int n = I.n;
  const int32_t* order = B.order + (long long)i * P;
  const double* fit = fit_buf(B, parity) + (long long)i * P;
  const double* off_fit = B.off_fit + (long long)i * P;
  const int o = order[r];
  const int32_t* src = o < P ? pop_buf(B, parity) + I.pop_offset + (long long)o * n
                             : B.off + I.pop_offset + (long long)(o - P) * n;
  int32_t* dst = pop_buf(B, parity ^ 1) + I.pop_offset + (long long)r * n;
  if ((n & 3) == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int t = threadIdx.x; t < (n >> 2); t += blockDim.x) d4[t] = s4[t];
  } else {
    for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
  }
  if (threadIdx.x == 0) {
    const double f = o < P ? fit[o] : off_fit[o - P];
    fit_buf(B, parity ^ 1)[(long long)i * P + r] = f;
    if (B.clean[0]) {
      const uint8_t* cs = clean_buf(B, parity) + (long long)i * P;
      clean_buf(B, parity ^ 1)[(long long)i * P + r] = o < P ? cs[o] : B.off_clean[(long long)i * P + o - P];
    }
  }
}

// Persistent 2-opt over the (item, row) units of one phase. COORDS: the bucket's
// instances rebuild distances from coordinates (no matrix); otherwise they all have one.
// LAYOUT: SCAN_GROUPED when every item's k is a multiple of U and its packed table is
// U*4-byte aligned, else SCAN_PACKED. REV (TSPB_BATCH_INCREMENTAL): the items carry their
// reverse k-NN index; best mode then keeps incremental row keys (INC, grouped layout only)
// and first mode restarts incrementally. CL = 2 (TSPB_BATCH_PAIR, best mode, grouped, no
// REV): the grid is made of two-CTA clusters, CTA 0 of a cluster takes each unit from the
// queue and hands it to CTA 1 through distributed shared memory, and the pair refines the
// row together (scan_tour's CTA pair).
template <int MODE, int THREADS, int U, bool COORDS, int LAYOUT, bool REV = false, int CL = 1>
__global__ void __launch_bounds__(THREADS, ScanMinBlocks<THREADS>::value)
    batch_two_opt_kernel(const tspb_batch B, const int32_t* __restrict__ items, int num_items, int rows, int phase,
                         long long max_iter, int max_n, unsigned* __restrict__ queue, long long budget) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ ScanSmem S;
  __shared__ unsigned s_unit;
  const unsigned units = (unsigned)num_items * (unsigned)rows;
  for (;;) {
    unsigned u;
    if constexpr (CL == 1) {
      if (threadIdx.x == 0) s_unit = atomicAdd(queue, 1u);
      __syncthreads();
      u = s_unit;
      __syncthreads();  // every thread has read s_unit before thread 0 takes the next unit
    } else {
      cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
      if (cl.block_rank() == 0 && threadIdx.x == 0) s_unit = atomicAdd(queue, 1u);
      cl.sync();
      u = *cl.map_shared_rank(&s_unit, 0u);
      cl.sync();  // both CTAs hold the unit before CTA 0 takes the next one
    }
    if (u >= units) return;
    const int it = (int)(u / (unsigned)rows), e = (int)(u - (unsigned)it * (unsigned)rows);
    const int i = items[it];
    const bool offspring = phase == TSPB_BATCH_PHASE_OFFSPRING;
    int parity = 0, row = e;
    if (phase != TSPB_BATCH_PHASE_POSTINIT) {
      const int* c = B.ctl + 4 * i;
      if (c[1] != phase_state(phase)) continue;
      parity = (c[0] + 1) & 1;
      if (phase == TSPB_BATCH_PHASE_RESUME) {
        row = B.host_elites[(long long)i * B.elite + e];
        if ((unsigned)row >= (unsigned)B.P) {
          if (threadIdx.x == 0) B.ls_status[(long long)i * B.rows_max + e] = TSPB_ERR_RANGE;
          continue;
        }
      }
    }
    uint8_t* clean = !B.clean[0] ? nullptr
                     : (offspring ? B.off_clean : clean_buf(B, parity)) + (long long)i * B.P + row;
    if (clean && *clean) continue;  // a converged local optimum: refining it changes nothing
    const tspb_batch_instance I = B.inst[i];
    const bool layout_ok = LAYOUT != SCAN_GROUPED ||
                           (I.k % U == 0 && (reinterpret_cast<uintptr_t>(I.cand_packed) % (U * sizeof(uint32_t))) == 0);
    const bool rev_ok = !REV || (I.rev_off != nullptr && I.rev_idx != nullptr);
    if ((I.dist == nullptr) != COORDS || I.n > max_n || I.n < 4 || I.k < 1 || !layout_ok || !rev_ok) {
      if (threadIdx.x == 0) B.ls_status[(long long)i * B.rows_max + e] = TSPB_ERR_UNSUPPORTED;
      continue;
    }
    ScanTour T;
    T.g_tour = (offspring ? B.off : pop_buf(B, parity)) + I.pop_offset + (long long)row * I.n;
    T.arrays = dsm;
    T.n = I.n;
    T.k = I.k;
    T.ds.dist = COORDS ? nullptr : I.dist;
    T.ds.stride = COORDS ? 0 : I.dist_stride;
    T.ds.coords = COORDS ? reinterpret_cast<const double2*>(I.coords) : nullptr;
    T.packed = I.cand_packed;
    T.cand = nullptr;
    T.cand_dist = nullptr;
    T.max_iter = max_iter;
    T.status = B.ls_status + (long long)i * B.rows_max + e;
    T.stats = B.ls_stats ? reinterpret_cast<long long*>(B.ls_stats) + ((long long)i * B.rows_max + e) * 4 : nullptr;
    T.accumulate = 1;
    T.moved = nullptr;
    T.converged = clean;
    T.rev_off = REV ? I.rev_off : nullptr;
    T.rev_idx = REV ? I.rev_idx : nullptr;
    T.budget = budget;
    // the refined row's fitness (fit, or off_fit for children); POSTINIT leaves fitness
    // to tspb_batch_init (the tuner's probes refine scratch rows there)
    T.cost = phase == TSPB_BATCH_PHASE_POSTINIT
                 ? nullptr
                 : (offspring ? B.off_fit : fit_buf(B, parity)) + (long long)i * B.P + row;
    scan_tour<MODE, THREADS, U, LAYOUT, REV && MODE == TSPB_MODE_BEST, true, CL, false>(T, S);
  }
}

// CTA per instance of a phase: argmin of fitness (first minimum), strict improvement by
// more than 1e-6 copies the tour, history[g + 1] = best so far, patience, generation + 1.
__global__ void __launch_bounds__(128) batch_track_kernel(const tspb_batch B, int phase) {
  const int i = blockIdx.x;
  int* c = B.ctl + 4 * i;
  if (c[1] != phase_state(phase)) return;
  __shared__ double sv[32];
  __shared__ int si[32];
  __shared__ int improve;
  const int P = B.P, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int g = c[0], parity = (g + 1) & 1;
  const tspb_batch_instance I = B.inst[i];
  const double* fit = fit_buf(B, parity) + (long long)i * P;
  double bv = __longlong_as_double(0x7ff0000000000000LL);
  int bi = P;
  for (int r = tid; r < P; r += blockDim.x) {
    const double f = fit[r];
    if (f < bv || (f == bv && r < bi)) {
      bv = f;
      bi = r;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(FULL, bv, o);
    const int oi = __shfl_xor_sync(FULL, bi, o);
    if (ov < bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
    }
  }
  if (lane == 0) {
    sv[wid] = bv;
    si[wid] = bi;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (sv[w] < bv || (sv[w] == bv && si[w] < bi)) {
        bv = sv[w];
        bi = si[w];
      }
    si[0] = bi;
    double best = B.best_cost[i];
    improve = bv < best - 1e-6;
    int stall = c[2];
    if (improve) {
      best = bv;
      B.best_cost[i] = bv;
      stall = 0;
    } else {
      stall += 1;
    }
    B.history[(long long)i * (B.G + 1) + g + 1] = best;
    c[2] = stall;
    c[3] = g + 1;
    c[0] = g + 1;
    // early stops in the reference's order: a known optimum reached or within 1 %, then
    // patience (the arithmetic spelled out so that no step is contracted)
    const double opt = I.optimal;
    int next = g + 1 >= B.G ? TSPB_BATCH_DONE : TSPB_BATCH_RUN;
    if (stall >= I.patience) next = TSPB_BATCH_STOPPED;
    if (opt > 0.0) {
      if (best <= __dadd_rn(opt, 1e-6))
        next = TSPB_BATCH_HIT_OPTIMAL;
      else if (__dmul_rn(__ddiv_rn(__dsub_rn(best, opt), opt), 100.0) < 1.0)
        next = TSPB_BATCH_NEAR_OPTIMAL;
    }
    c[1] = next;
  }
  __syncthreads();
  if (improve) {
    const int32_t* src = pop_buf(B, parity) + I.pop_offset + (long long)si[0] * I.n;
    for (int t = tid; t < I.n; t += blockDim.x) B.best_tour[I.node_offset + t] = src[t];
  }
}

template <int MODE, int THREADS, int U>
static int batch_two_opt_launch(const tspb_batch& b, const int32_t* items, int num_items, int rows, int phase,
                                long long max_iter, int max_n, size_t smem, int ctas, int flags, unsigned* queue,
                                cudaStream_t st) {
  const bool coords = flags & TSPB_BATCH_COORDS, grouped = flags & TSPB_BATCH_GROUPED;
  const bool rev = flags & TSPB_BATCH_INCREMENTAL;
  using Kern = void (*)(const tspb_batch, const int32_t*, int, int, int, long long, int, unsigned*, long long);
  Kern kern = coords ? (grouped ? batch_two_opt_kernel<MODE, THREADS, U, true, SCAN_GROUPED>
                                : batch_two_opt_kernel<MODE, THREADS, U, true, SCAN_PACKED>)
                     : (grouped ? batch_two_opt_kernel<MODE, THREADS, U, false, SCAN_GROUPED>
                                : batch_two_opt_kernel<MODE, THREADS, U, false, SCAN_PACKED>);
  if (rev) {
    // the reverse-index variants exist for the grouped layout (the caller checked GROUPED),
    // which every CTA size launches with four words per thread
    if constexpr (U == 4)
      kern = coords ? batch_two_opt_kernel<MODE, THREADS, U, true, SCAN_GROUPED, true>
                    : batch_two_opt_kernel<MODE, THREADS, U, false, SCAN_GROUPED, true>;
    else
      return TSPB_ERR_ARG;
  }
  if (flags & TSPB_BATCH_PAIR) {
    // two-CTA clusters, one per unit at a time (best mode, grouped layout; checked by the caller)
    if constexpr (MODE == TSPB_MODE_BEST && U == 4) {
      Kern pk = coords ? batch_two_opt_kernel<MODE, THREADS, U, true, SCAN_GROUPED, false, 2>
                       : batch_two_opt_kernel<MODE, THREADS, U, false, SCAN_GROUPED, false, 2>;
      TSPB_CUDA_CHECK(cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = 2;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.blockDim = dim3(THREADS);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = st;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      cfg.gridDim = dim3(2);
      TSPB_CUDA_CHECK(cudaOccupancyMaxActiveClusters(&clusters, pk, &cfg));
      if (clusters <= 0) return TSPB_ERR_UNSUPPORTED;
      const long long units = (long long)num_items * rows;
      long long pairs = clusters;
      if (ctas > 0 && ctas / 2 < pairs) pairs = ctas / 2 > 0 ? ctas / 2 : 1;
      if (pairs > units) pairs = units;
      int sms = 0, dev = 0;
      TSPB_CUDA_CHECK(cudaGetDevice(&dev));
      TSPB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      const int pct = carveout_for((int)((2 * pairs + sms - 1) / sms), smem);
      if (pct > 0) TSPB_CUDA_CHECK(cudaFuncSetAttribute(pk, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
      TSPB_CUDA_CHECK(cudaMemsetAsync(queue, 0, sizeof(unsigned), st));
      cfg.gridDim = dim3((unsigned)(2 * pairs));
      TSPB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, pk, b, items, num_items, rows, phase, max_iter, max_n, queue,
                                         watchdog_cycles()));
      return tspb_launch_status();
    } else {
      return TSPB_ERR_ARG;
    }
  }
  TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  TSPB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem));
  if (per_sm <= 0) return TSPB_ERR_UNSUPPORTED;
  int dev = 0, sms = 0;
  TSPB_CUDA_CHECK(cudaGetDevice(&dev));
  TSPB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long units = (long long)num_items * rows;
  long long grid = (long long)per_sm * sms;
  if (ctas > 0 && ctas < grid) grid = ctas;
  if (grid > units) grid = units;
  const int per_sm_used = (int)((grid + sms - 1) / sms);
  const int pct = carveout_for(per_sm_used < per_sm ? per_sm_used : per_sm, smem);
  if (pct > 0) TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  TSPB_CUDA_CHECK(cudaMemsetAsync(queue, 0, sizeof(unsigned), st));
  kern<<<(int)grid, THREADS, smem, st>>>(b, items, num_items, rows, phase, max_iter, max_n, queue, watchdog_cycles());
  return tspb_launch_status();
}

template <int MODE, int THREADS, int U>
static int batch_two_opt_occ(size_t smem, bool rev, bool pair) {
  if (pair) {  // co-resident two-CTA clusters, in CTAs
    if constexpr (MODE == TSPB_MODE_BEST && U == 4) {
      auto pk = batch_two_opt_kernel<MODE, THREADS, U, false, SCAN_GROUPED, false, 2>;
      if (cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = 2;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(2);
      cfg.blockDim = dim3(THREADS);
      cfg.dynamicSmemBytes = smem;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, pk, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
      }
      return 2 * clusters;
    } else {
      return 0;
    }
  }
  auto kern = rev ? batch_two_opt_kernel<MODE, THREADS, U, false, SCAN_GROUPED, true>
                  : batch_two_opt_kernel<MODE, THREADS, U, false, SCAN_GROUPED>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem) != cudaSuccess) return 0;
  return per_sm;
}

template <int MODE>
static int batch_two_opt_mode(const tspb_batch& b, const int32_t* items, int num_items, int rows, int phase,
                              long long max_iter, int max_n, int threads, size_t smem, int ctas, int flags,
                              unsigned* queue, cudaStream_t st) {
  switch (threads) {
    case 64:
      return batch_two_opt_launch<MODE, 64, 4>(b, items, num_items, rows, phase, max_iter, max_n, smem, ctas, flags,
                                               queue, st);
    case 128:
      return batch_two_opt_launch<MODE, 128, 4>(b, items, num_items, rows, phase, max_iter, max_n, smem, ctas, flags,
                                                queue, st);
    case 256:
      return batch_two_opt_launch<MODE, 256, 4>(b, items, num_items, rows, phase, max_iter, max_n, smem, ctas, flags,
                                                queue, st);
    // wide CTAs keep four entries per thread in flight only in the grouped layout (fewer
    // registers per entry there); otherwise two
    case 512:
      return (flags & TSPB_BATCH_GROUPED)
                 ? batch_two_opt_launch<MODE, 512, 4>(b, items, num_items, rows, phase, max_iter, max_n, smem, ctas,
                                                      flags, queue, st)
                 : batch_two_opt_launch<MODE, 512, 2>(b, items, num_items, rows, phase, max_iter, max_n, smem, ctas,
                                                      flags, queue, st);
    case 1024:
      return (flags & TSPB_BATCH_GROUPED)
                 ? batch_two_opt_launch<MODE, 1024, 4>(b, items, num_items, rows, phase, max_iter, max_n, smem, ctas,
                                                       flags, queue, st)
                 : batch_two_opt_launch<MODE, 1024, 2>(b, items, num_items, rows, phase, max_iter, max_n, smem, ctas,
                                                       flags, queue, st);
    default: return TSPB_ERR_ARG;
  }
}

template <int MODE>
static int batch_two_opt_occ_mode(int threads, size_t smem, bool rev, bool pair) {
  switch (threads) {
    case 64: return batch_two_opt_occ<MODE, 64, 4>(smem, rev, pair);
    case 128: return batch_two_opt_occ<MODE, 128, 4>(smem, rev, pair);
    case 256: return batch_two_opt_occ<MODE, 256, 4>(smem, rev, pair);
    case 512: return batch_two_opt_occ<MODE, 512, 4>(smem, rev, pair);
    case 1024: return batch_two_opt_occ<MODE, 1024, 4>(smem, rev, pair);
    default: return 0;
  }
}

}  // namespace tspb

using namespace tspb;

static bool batch_ok(const tspb_batch* b) {
  if (b == nullptr || b->num_instances < 0 || b->P < 2 || b->kt < 1 || b->elite < 0 || b->elite > b->P || b->G < 0)
    return false;
  if (b->rows_max < b->P) return false;
  if ((b->clean[0] == nullptr) != (b->clean[1] == nullptr)) return false;
  if (b->crossover != TSPB_XOVER_PMX && b->crossover != TSPB_XOVER_OX) return false;
  if (b->mutation != TSPB_MUT_INVERSION && b->mutation != TSPB_MUT_SWAP) return false;
  if (b->num_instances == 0) return true;
  return b->inst && b->pop[0] && b->pop[1] && b->fit[0] && b->fit[1] && b->off && b->off_fit && b->order && b->ctl &&
         b->best_cost && b->best_tour && b->history && b->ls_status;
}

static bool tape_ok(const tspb_batch* b) {
  return b->tape_tourn && b->tape_u && b->tape_inv_a && b->tape_inv_b && b->tape_cut_a && b->tape_cut_b && b->ties &&
         (b->clean[0] == nullptr || b->off_clean != nullptr);
}

extern "C" int tspb_batch_init(const tspb_batch* b, int32_t parity, int32_t set_best, void* stream) {
  if (!batch_ok(b) || (parity != 0 && parity != 1)) return TSPB_ERR_ARG;
  if (b->num_instances == 0) return TSPB_OK;
  const int row_blocks = (b->P + INIT_ROWS - 1) / INIT_ROWS;
  if (row_blocks > 65535) return TSPB_ERR_UNSUPPORTED;  // row blocks index grid.y
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const dim3 grid((unsigned)b->num_instances, (unsigned)row_blocks);
  batch_fitness_kernel<<<grid, 32 * INIT_ROWS, 0, st>>>(*b, parity);
  if (set_best) batch_init_kernel<<<b->num_instances, 256, 0, st>>>(*b, parity);
  return tspb_launch_status();
}

extern "C" int tspb_batch_offspring(const tspb_batch* b, const int32_t* items, int32_t num_items, int32_t max_n,
                                    int32_t threads, void* stream) {
  if (!batch_ok(b) || !tape_ok(b) || num_items < 0 || max_n < 1) return TSPB_ERR_ARG;
  if (threads < 32 || threads > 256 || threads % 32 != 0) return TSPB_ERR_ARG;
  if (num_items == 0 || b->G == 0) return TSPB_OK;
  if (!items) return TSPB_ERR_ARG;
  if ((long long)num_items * b->P > 0x7fffffffLL) return TSPB_ERR_UNSUPPORTED;
  const size_t smem = offspring_smem_bytes(max_n);
  if (smem > 200 * 1024) return TSPB_ERR_UNSUPPORTED;
  if (smem > 48 * 1024)
    TSPB_CUDA_CHECK(cudaFuncSetAttribute(batch_offspring_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  batch_offspring_kernel<<<num_items * b->P, threads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(*b, items, max_n);
  return tspb_launch_status();
}

extern "C" int tspb_batch_survival(const tspb_batch* b, void* stream) {
  if (!batch_ok(b) || !tape_ok(b)) return TSPB_ERR_ARG;
  if (b->num_instances == 0 || b->G == 0) return TSPB_OK;
  if ((long long)b->num_instances * b->P > 0x7fffffffLL || b->P > 3072) return TSPB_ERR_UNSUPPORTED;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int n2 = 1;
  while (n2 < 2 * b->P) n2 <<= 1;
  const size_t rank_smem = (size_t)12 * n2;
  if (n2 >= 64 && n2 <= 2048) {  // n2 / 2 threads, pairs in registers
    batch_survival_rank_reg_kernel<<<b->num_instances, n2 / 2, rank_smem, st>>>(*b, n2);
  } else {
    const int rank_threads = n2 >= 1024 ? 512 : (n2 / 2 > 32 ? n2 / 2 : 32);
    if (rank_smem > 48 * 1024)
      TSPB_CUDA_CHECK(cudaFuncSetAttribute(batch_survival_rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)rank_smem));
    batch_survival_rank_kernel<<<b->num_instances, rank_threads, rank_smem, st>>>(*b, n2);
  }
  batch_survival_gather_kernel<<<b->num_instances * b->P, 128, 0, st>>>(*b);
  return tspb_launch_status();
}

extern "C" int tspb_batch_two_opt_occupancy(int32_t max_n, int32_t mode, int32_t threads, int32_t flags) {
  if (max_n < 4 || (mode != TSPB_MODE_BEST && mode != TSPB_MODE_FIRST)) return 0;
  const bool rev = flags & TSPB_BATCH_INCREMENTAL;
  const bool pair = flags & TSPB_BATCH_PAIR;
  if (pair && (rev || mode != TSPB_MODE_BEST)) return 0;
  const size_t smem = scan_tour_state_bytes(max_n, mode, rev);
  if (smem > (size_t)smem_optin() - 2048) return 0;
  return mode == TSPB_MODE_BEST ? batch_two_opt_occ_mode<TSPB_MODE_BEST>(threads, smem, rev, pair)
                                : batch_two_opt_occ_mode<TSPB_MODE_FIRST>(threads, smem, rev, pair);
}

extern "C" int tspb_batch_two_opt(const tspb_batch* b, const int32_t* items, int32_t num_items, int32_t max_n,
                                  int32_t flags, int32_t phase, int32_t mode, int64_t max_iterations, int32_t threads,
                                  int32_t ctas, uint32_t* queue, void* stream) {
  if (!batch_ok(b) || num_items < 0 || max_n < 4 || !queue) return TSPB_ERR_ARG;
  if (flags & ~(TSPB_BATCH_COORDS | TSPB_BATCH_GROUPED | TSPB_BATCH_INCREMENTAL | TSPB_BATCH_PAIR)) return TSPB_ERR_ARG;
  if ((flags & TSPB_BATCH_PAIR) &&
      (mode != TSPB_MODE_BEST || !(flags & TSPB_BATCH_GROUPED) || (flags & TSPB_BATCH_INCREMENTAL)))
    return TSPB_ERR_ARG;
  const bool rev = flags & TSPB_BATCH_INCREMENTAL;
  if (rev && !(flags & TSPB_BATCH_GROUPED)) return TSPB_ERR_ARG;
  if (phase < TSPB_BATCH_PHASE_POSTINIT || phase > TSPB_BATCH_PHASE_OFFSPRING) return TSPB_ERR_ARG;
  if (mode != TSPB_MODE_BEST && mode != TSPB_MODE_FIRST) return TSPB_ERR_ARG;
  const int rows = (phase == TSPB_BATCH_PHASE_POSTINIT || phase == TSPB_BATCH_PHASE_OFFSPRING) ? b->P : b->elite;
  if (num_items == 0 || rows == 0 || max_iterations <= 0) return TSPB_OK;
  if (!items) return TSPB_ERR_ARG;
  if (phase == TSPB_BATCH_PHASE_RESUME && !b->host_elites) return TSPB_ERR_ARG;
  if ((long long)num_items * rows > 0x7fffffffLL || max_n > 65535) return TSPB_ERR_UNSUPPORTED;
  const size_t smem = scan_tour_state_bytes(max_n, mode, rev);
  if (smem > (size_t)smem_optin() - 2048) return TSPB_ERR_UNSUPPORTED;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (mode == TSPB_MODE_BEST)
    return batch_two_opt_mode<TSPB_MODE_BEST>(*b, items, num_items, rows, phase, max_iterations, max_n, threads, smem,
                                              ctas, flags, queue, st);
  return batch_two_opt_mode<TSPB_MODE_FIRST>(*b, items, num_items, rows, phase, max_iterations, max_n, threads, smem,
                                             ctas, flags, queue, st);
}

extern "C" int tspb_batch_track(const tspb_batch* b, int32_t phase, void* stream) {
  if (!batch_ok(b) || (phase != TSPB_BATCH_PHASE_RESUME && phase != TSPB_BATCH_PHASE_RUN)) return TSPB_ERR_ARG;
  if (b->num_instances == 0 || b->G == 0) return TSPB_OK;
  batch_track_kernel<<<b->num_instances, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*b, phase);
  return tspb_launch_status();
}
