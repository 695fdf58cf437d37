// Random tape of the GA, drawn exactly as NumPy's Generator(PCG64) draws it.
//
// The reference draws every generation's random numbers from `context.rng`, a
// `np.random.Generator` on a PCG64 bit generator (src/utils/rng.py:48-64), in this order
// (tournament_selection.py:113, pmx_crossover.py:155, inversion_mutation.py:82,
// route_helpers.py:214):
//   integers(0, P, size=(P, kt), dtype=int32)      tournament contestants
//   sample_distinct_pairs(P // 2, 0, n)              PMX cut pairs
//   random(P)                                        inversion draws
//   sample_distinct_pairs(P, 0, n)                   inversion positions
// where sample_distinct_pairs draws first = integers(0, n, m), shifted = integers(0, n - 1, m)
// and pairs (first, shifted + (shifted >= first)).
//
// Published algorithms restated here:
// - PCG64 (O'Neill, "PCG: A Family of Simple Fast Space-Efficient Statistically Good
//   Algorithms for Random Number Generation"): 128-bit LCG state' = state * M + inc with the
//   128-bit default multiplier, output XSL-RR: rotr64(hi ^ lo, state >> 122);
// - NumPy's 32-bit draws take the low half of a 64-bit output and keep the high half for the
//   next 32-bit draw (`has_uint32`, `uinteger` in the generator state);
// - bounded integers by Lemire's multiply-and-reject method on 32-bit draws (the default
//   of Generator.integers for 32-bit dtypes);
// - doubles as (next64 >> 11) * 2^-53 (not touching the buffered half).
// The same code runs on the host (checked against NumPy in the CPU tests) and on the device
// (one thread per instance, writing the tape straight into HBM).
#include "common.cuh"

namespace tspb {

struct Pcg {
  uint64_t hi, lo, inc_hi, inc_lo;
  int has32;
  uint32_t buf32;
};

__host__ __device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * (unsigned __int128)b) >> 64);
#endif
}

__host__ __device__ __forceinline__ uint64_t pcg_next64(Pcg& g) {
  const uint64_t m_hi = 0x2360ED051FC65DA4ull, m_lo = 0x4385DF649FCCF645ull;
  const uint64_t lo = g.lo * m_lo;
  uint64_t hi = mulhi64(g.lo, m_lo) + g.lo * m_hi + g.hi * m_lo;
  const uint64_t nlo = lo + g.inc_lo;
  hi += g.inc_hi + (nlo < lo ? 1u : 0u);
  g.lo = nlo;
  g.hi = hi;
  const uint64_t x = hi ^ nlo;
  const unsigned rot = (unsigned)(hi >> 58);
  return (x >> rot) | (x << ((64u - rot) & 63u));
}

__host__ __device__ __forceinline__ uint32_t pcg_next32(Pcg& g) {
  if (g.has32) {
    g.has32 = 0;
    return g.buf32;
  }
  const uint64_t v = pcg_next64(g);
  g.has32 = 1;
  g.buf32 = (uint32_t)(v >> 32);
  return (uint32_t)(v & 0xffffffffu);
}

// Uniform integer in [0, rng] (rng = high - 1 - low of integers(low, high)).
__host__ __device__ __forceinline__ uint32_t pcg_bounded(Pcg& g, uint32_t rng) {
  if (rng == 0) return 0;
  if (rng == 0xffffffffu) return pcg_next32(g);
  const uint32_t ex = rng + 1u;
  uint64_t m = (uint64_t)pcg_next32(g) * ex;
  uint32_t left = (uint32_t)m;
  if (left < ex) {
    const uint32_t threshold = (uint32_t)(0u - ex) % ex;  // 2^32 mod ex
    while (left < threshold) {
      m = (uint64_t)pcg_next32(g) * ex;
      left = (uint32_t)m;
    }
  }
  return (uint32_t)(m >> 32);
}

__host__ __device__ __forceinline__ double pcg_double(Pcg& g) {
  return (double)(pcg_next64(g) >> 11) * (1.0 / 9007199254740992.0);
}

__host__ __device__ inline Pcg pcg_from(const tspb_pcg64& s) {
  Pcg g;
  g.hi = s.state_hi;
  g.lo = s.state_lo;
  g.inc_hi = s.inc_hi;
  g.inc_lo = s.inc_lo;
  g.has32 = s.has_uint32;
  g.buf32 = s.uinteger;
  return g;
}

__host__ __device__ inline void pcg_to(const Pcg& g, tspb_pcg64& s) {
  s.state_hi = g.hi;
  s.state_lo = g.lo;
  s.inc_hi = g.inc_hi;
  s.inc_lo = g.inc_lo;
  s.has_uint32 = g.has32;
  s.uinteger = g.buf32;
}

// pairs (first, second) of sample_distinct_pairs(m, 0, n): all firsts, then all shifted.
__host__ __device__ inline void draw_pairs(Pcg& g, int m, int n, int32_t* a, int32_t* b) {
  for (int j = 0; j < m; ++j) a[j] = (int32_t)pcg_bounded(g, (uint32_t)(n - 1));
  for (int j = 0; j < m; ++j) {
    const int32_t s = (int32_t)pcg_bounded(g, (uint32_t)(n - 2));
    b[j] = s + (s >= a[j] ? 1 : 0);
  }
}

// G generations of one run; arrays are that run's [G][...] slices.
__host__ __device__ inline void draw_tape(Pcg& g, int G, int P, int kt, int n, int32_t* tourn, int32_t* cut_a,
                                          int32_t* cut_b, double* u, int32_t* inv_a, int32_t* inv_b,
                                          tspb_pcg64* states) {
  const int half = P / 2;
  for (int gen = 0; gen < G; ++gen) {
    int32_t* t = tourn + (long long)gen * P * kt;
    for (int q = 0; q < P * kt; ++q) t[q] = (int32_t)pcg_bounded(g, (uint32_t)(P - 1));
    draw_pairs(g, half, n, cut_a + (long long)gen * half, cut_b + (long long)gen * half);
    double* uu = u + (long long)gen * P;
    for (int q = 0; q < P; ++q) uu[q] = pcg_double(g);
    draw_pairs(g, P, n, inv_a + (long long)gen * P, inv_b + (long long)gen * P);
    if (states) pcg_to(g, states[gen]);
  }
}

__global__ void tape_kernel(tspb_pcg64* __restrict__ gens, const int32_t* __restrict__ ns, int num, int G, int P,
                            int kt, int32_t* tourn, int32_t* cut_a, int32_t* cut_b, double* u, int32_t* inv_a,
                            int32_t* inv_b, tspb_pcg64* states) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= num) return;
  if (ns[i] < 2) return;  // sample_distinct_pairs needs two cities
  Pcg g = pcg_from(gens[i]);
  const long long gp = (long long)i * G;
  draw_tape(g, G, P, kt, ns[i], tourn + gp * P * kt, cut_a + gp * (P / 2), cut_b + gp * (P / 2), u + gp * P,
            inv_a + gp * P, inv_b + gp * P, states ? states + gp : nullptr);
  pcg_to(g, gens[i]);
}

}  // namespace tspb

using namespace tspb;

static bool tape_args_ok(int32_t G, int32_t P, int32_t kt) { return G >= 0 && P >= 2 && kt >= 1; }

extern "C" int tspb_tape_draw_host(tspb_pcg64* gen, int32_t G, int32_t P, int32_t kt, int32_t n, int32_t* tourn,
                                   int32_t* cut_a, int32_t* cut_b, double* u, int32_t* inv_a, int32_t* inv_b,
                                   tspb_pcg64* states) {
  if (!gen || !tape_args_ok(G, P, kt) || n < 2) return TSPB_ERR_ARG;
  if (G == 0) return TSPB_OK;
  if (!tourn || !cut_a || !cut_b || !u || !inv_a || !inv_b) return TSPB_ERR_ARG;
  Pcg g = pcg_from(*gen);
  draw_tape(g, G, P, kt, n, tourn, cut_a, cut_b, u, inv_a, inv_b, states);
  pcg_to(g, *gen);
  return TSPB_OK;
}

extern "C" int tspb_tape_draw(tspb_pcg64* gens, const int32_t* ns, int32_t num, int32_t G, int32_t P, int32_t kt,
                              int32_t* tourn, int32_t* cut_a, int32_t* cut_b, double* u, int32_t* inv_a,
                              int32_t* inv_b, tspb_pcg64* states, void* stream) {
  if (num < 0 || !tape_args_ok(G, P, kt)) return TSPB_ERR_ARG;
  if (num == 0 || G == 0) return TSPB_OK;
  if (!gens || !ns || !tourn || !cut_a || !cut_b || !u || !inv_a || !inv_b) return TSPB_ERR_ARG;
  const int threads = 32;
  tape_kernel<<<(num + threads - 1) / threads, threads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      gens, ns, num, G, P, kt, tourn, cut_a, cut_b, u, inv_a, inv_b, states);
  return tspb_launch_status();
}
