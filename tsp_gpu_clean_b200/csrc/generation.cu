// One GA generation on the device, for graph capture: the fused offspring kernel
// (tournament selection, PMX crossover, inversion mutation, tour-length reduction), the
// (mu + lambda) survival gather, and best-so-far tracking with early stop.
//
// The random draws of every generation are pre-drawn on the host from the run's
// generator in the reference's order (tournament (P, k) -> PMX cut pairs (P/2) ->
// inversion u (P) -> inversion position pairs (P)) and uploaded once as a tape; the
// kernels read generation g's slice through a device counter that the tracking kernel
// advances, so one captured graph replays every generation unchanged. A device flag set
// by the tracker (patience exhausted) turns the remaining generations into no-ops.
//
// Reference semantics reproduced bit for bit:
//   SelectionCPUTournament.select_batch    (tournament_selection.py:98-128)
//   CrossoverCPUPermPartiallyMapped         (pmx_crossover.py:49-171, open permutations)
//   MutationCPUPermInversion.mutate_batch   (inversion_mutation.py:65-99)
//   evaluate_tour_cpu                       (tour_cost.py:17-29)
//   _select_survivors_assessed              (genetic_algorithm.py:618-706)
//   best tracking / patience                (genetic_algorithm.py:876-910)
#include "generation.cuh"

namespace tspb {

struct GenTape {
  const int32_t* tourn;   // [G][P][kt]
  const int32_t* cut_a;   // [G][P/2]
  const int32_t* cut_b;   // [G][P/2]
  const double* u;        // [G][P]
  const int32_t* inv_a;   // [G][P]
  const int32_t* inv_b;   // [G][P]
};

// CTA per child row of generation *gen.
__global__ void __launch_bounds__(256) offspring_kernel(const int32_t* __restrict__ pop, const double* __restrict__ fit,
                                                        int P, int n, int kt, GenTape tape, const int* __restrict__ gen,
                                                        const int* __restrict__ stopped, double rate, DistSrc ds,
                                                        int32_t* __restrict__ off, double* __restrict__ off_fit) {
  if (*stopped) return;
  extern __shared__ int sm[];
  const long long g = *gen;
  const int pairs = P >> 1;
  GenTapeSlice sl;
  sl.tourn = tape.tourn + g * P * kt;
  sl.cut_a = tape.cut_a ? tape.cut_a + g * pairs : nullptr;
  sl.cut_b = tape.cut_b ? tape.cut_b + g * pairs : nullptr;
  sl.u = tape.u + g * P;
  sl.inv_a = tape.inv_a + g * P;
  sl.inv_b = tape.inv_b + g * P;
  const int row = blockIdx.x;
  offspring_row(pop, fit, P, n, kt, sl, rate, ds, row, sm, off + (long long)row * n, off_fit + row);
}

// Stable rank of the 2P combined fitness (old population first), keep P.
__global__ void survival_rank_kernel(const double* __restrict__ fa, const double* __restrict__ fb, int P,
                                     const int* __restrict__ stopped, int32_t* __restrict__ order) {
  if (*stopped) return;
  __shared__ double tile[256];
  const int count = 2 * P;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double fi = i < count ? (i < P ? fa[i] : fb[i - P]) : 0.0;
  int rank = 0;
  for (int base = 0; base < count; base += blockDim.x) {
    const int j = base + threadIdx.x;
    if (j < count) tile[threadIdx.x] = j < P ? fa[j] : fb[j - P];
    __syncthreads();
    const int lim = min((int)blockDim.x, count - base);
    if (i < count)
      for (int t = 0; t < lim; ++t) {
        const double fj = tile[t];
        rank += (fj < fi) || (fj == fi && base + t < i);
      }
    __syncthreads();
  }
  if (i < count && rank < P) order[rank] = i;
}

// CTA per survivor: new_pop[r] = combined[order[r]]. A fitness tie across the elite edge
// sets tie_flags[g] and pauses the run (*stopped = 2): the elite membership then follows
// NumPy's unstable argsort, which the host decides before the run resumes.
__global__ void survival_gather_kernel(const int32_t* __restrict__ pop, const double* __restrict__ fit,
                                       const int32_t* __restrict__ off, const double* __restrict__ off_fit, int P, int n,
                                       const int32_t* __restrict__ order, int* __restrict__ stopped,
                                       const int* __restrict__ gen, int elite, int32_t* __restrict__ new_pop,
                                       double* __restrict__ new_fit, int32_t* __restrict__ tie_flags) {
  if (*stopped) return;
  const int r = blockIdx.x;
  const int o = order[r];
  const int32_t* src = o < P ? pop + (long long)o * n : off + (long long)(o - P) * n;
  int32_t* dst = new_pop + (long long)r * n;
  if ((n & 3) == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(dst);
    for (int t = threadIdx.x; t < (n >> 2); t += blockDim.x) d4[t] = s4[t];
  } else {
    for (int t = threadIdx.x; t < n; t += blockDim.x) dst[t] = src[t];
  }
  if (threadIdx.x == 0) {
    const double f = o < P ? fit[o] : off_fit[o - P];
    new_fit[r] = f;
    if (elite > 0 && elite < P && r == elite) {
      const int oe = order[elite - 1];
      const double fe = oe < P ? fit[oe] : off_fit[oe - P];
      tie_flags[*gen] = fe == f ? 1 : 0;
    }
  }
}

// After the gather (never inside it: its own CTAs read the flag at entry), a tie across
// the elite edge pauses the run for the host's elite decision.
__global__ void survival_pause_kernel(const int32_t* __restrict__ tie_flags, const int* __restrict__ gen,
                                      int* __restrict__ stopped) {
  if (*stopped == 0 && tie_flags[*gen] != 0) *stopped = 2;
}

// One CTA: argmin of fitness (first minimum), strict improvement by more than 1e-6 copies
// the tour, history[g + 1] = best so far, patience, then the generation counter advances.
__global__ void track_best_kernel(const double* __restrict__ fit, const int32_t* __restrict__ pop, int P, int n,
                                  int* __restrict__ gen, int* __restrict__ stopped, int* __restrict__ stall,
                                  long long patience, double* __restrict__ best_cost, int32_t* __restrict__ best_tour,
                                  double* __restrict__ history, int32_t* __restrict__ done_gens) {
  if (*stopped) return;
  __shared__ double sv[32];
  __shared__ int si[32];
  __shared__ int improve;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double bv = __longlong_as_double(0x7ff0000000000000LL);
  int bi = P;
  for (int i = tid; i < P; i += blockDim.x) {
    const double f = fit[i];
    if (f < bv || (f == bv && i < bi)) {
      bv = f;
      bi = i;
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
    improve = bv < *best_cost - 1e-6;
    if (improve) {
      *best_cost = bv;
      *stall = 0;
    } else {
      *stall += 1;
    }
    const int g = *gen;
    history[g + 1] = *best_cost;
    *done_gens = g + 1;
    if (*stall >= patience) *stopped = 1;
    *gen = g + 1;
  }
  __syncthreads();
  if (improve) {
    const int32_t* src = pop + (long long)si[0] * n;
    for (int t = tid; t < n; t += blockDim.x) best_tour[t] = src[t];
  }
}

// Rows [0, k) of the population get their fitness recomputed after the elite 2-opt.
__global__ void elite_cost_kernel(const int32_t* __restrict__ pop, int k, int n, DistSrc ds,
                                  const int* __restrict__ stopped, double* __restrict__ fit) {
  if (*stopped) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= k) return;
  const double f = warp_tour_length(pop + (long long)warp * n, n, ds);
  if ((threadIdx.x & 31) == 0) fit[warp] = f;
}

}  // namespace tspb

using namespace tspb;

static DistSrc gen_ds(const int32_t* dist, int64_t stride, const double* coords) {
  DistSrc d;
  d.dist = dist;
  d.stride = stride;
  d.coords = reinterpret_cast<const double2*>(coords);
  return d;
}

extern "C" int tspb_generation_offspring(const int32_t* pop, const double* fit, int32_t P, int32_t n, int32_t kt,
                                         const int32_t* tape_tourn, const int32_t* tape_cut_a, const int32_t* tape_cut_b,
                                         const double* tape_u, const int32_t* tape_inv_a, const int32_t* tape_inv_b,
                                         double rate, const int32_t* dist, int64_t dist_stride, const double* coords,
                                         const int32_t* gen, const int32_t* stopped, int32_t* off, double* off_fit,
                                         void* stream) {
  if (P < 1 || n < 1 || kt < 1) return TSPB_ERR_ARG;
  if (!pop || !fit || !tape_tourn || !tape_u || !tape_inv_a || !tape_inv_b || !gen || !stopped || !off || !off_fit)
    return TSPB_ERR_ARG;
  if (P >= 2 && (!tape_cut_a || !tape_cut_b)) return TSPB_ERR_ARG;
  if (!dist && !coords) return TSPB_ERR_ARG;
  const size_t smem = offspring_smem_bytes(n);
  if (smem > 200 * 1024) return TSPB_ERR_UNSUPPORTED;
  if (smem > 48 * 1024)
    TSPB_CUDA_CHECK(cudaFuncSetAttribute(offspring_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  GenTape tape{tape_tourn, tape_cut_a, tape_cut_b, tape_u, tape_inv_a, tape_inv_b};
  offspring_kernel<<<P, 256, smem, reinterpret_cast<cudaStream_t>(stream)>>>(pop, fit, P, n, kt, tape, gen, stopped, rate,
                                                                             gen_ds(dist, dist_stride, coords), off, off_fit);
  return tspb_launch_status();
}

extern "C" int tspb_generation_survival(const int32_t* pop, const double* fit, const int32_t* off, const double* off_fit,
                                        int32_t P, int32_t n, int32_t elite, const int32_t* gen, int32_t* stopped,
                                        int32_t* order, int32_t* new_pop, double* new_fit, int32_t* tie_flags,
                                        void* stream) {
  if (P < 1 || n < 1 || elite < 0) return TSPB_ERR_ARG;
  if (!pop || !fit || !off || !off_fit || !gen || !stopped || !order || !new_pop || !new_fit) return TSPB_ERR_ARG;
  if (elite > 0 && elite < P && !tie_flags) return TSPB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  survival_rank_kernel<<<(2 * P + 255) / 256, 256, 0, st>>>(fit, off_fit, P, stopped, order);
  survival_gather_kernel<<<P, 128, 0, st>>>(pop, fit, off, off_fit, P, n, order, stopped, gen, elite, new_pop, new_fit,
                                           tie_flags);
  if (elite > 0 && elite < P) survival_pause_kernel<<<1, 1, 0, st>>>(tie_flags, gen, stopped);
  return tspb_launch_status();
}

extern "C" int tspb_generation_elite_cost(const int32_t* pop, int32_t k, int32_t n, const int32_t* dist, int64_t dist_stride,
                                          const double* coords, const int32_t* stopped, double* fit, void* stream) {
  if (k < 0 || n < 1) return TSPB_ERR_ARG;
  if (k == 0) return TSPB_OK;
  if (!pop || !stopped || !fit || (!dist && !coords)) return TSPB_ERR_ARG;
  elite_cost_kernel<<<(k * 32 + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      pop, k, n, gen_ds(dist, dist_stride, coords), stopped, fit);
  return tspb_launch_status();
}

extern "C" int tspb_generation_track(const double* fit, const int32_t* pop, int32_t P, int32_t n, int32_t* gen,
                                     int32_t* stopped, int32_t* stall, int64_t patience, double* best_cost,
                                     int32_t* best_tour, double* history, int32_t* done_gens, void* stream) {
  if (P < 1 || n < 1) return TSPB_ERR_ARG;
  if (!fit || !pop || !gen || !stopped || !stall || !best_cost || !best_tour || !history || !done_gens) return TSPB_ERR_ARG;
  track_best_kernel<<<1, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(fit, pop, P, n, gen, stopped, stall, patience,
                                                                          best_cost, best_tour, history, done_gens);
  return tspb_launch_status();
}
