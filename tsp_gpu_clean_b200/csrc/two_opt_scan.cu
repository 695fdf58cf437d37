// Candidate-mode 2-opt (best / first), full rescan per pass: one CTA per tour.
//
// The per-tour body (scan_tour, two_opt_scan.cuh) follows the reference scan
// (src/algorithms/strategies/local_search/two_opt.py:347-367, 386-489, 565-595); this file
// holds the one-CTA-per-tour launch, its shared-memory carveout policy and the k-NN
// packing kernel.
#include <type_traits>

#include "two_opt_scan.cuh"

namespace tspb {

// SMEM: the tour state lives in shared memory (the compiler then addresses it with
// shared-memory instructions); otherwise in the per-tour global workspace slice.
// COUNT: first mode keeps the reference's pair count (launched when stats are requested).
template <int MODE, int THREADS, int U, int LAYOUT, bool SMEM, bool COUNT>
__global__ void __launch_bounds__(THREADS, ScanMinBlocks<THREADS>::value) two_opt_scan_kernel(const TwoOptArgs A) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ ScanSmem S;
  const int t = blockIdx.x;
  if (t >= A.num_tours) return;
  if (A.skip != nullptr && *A.skip != 0) return;
  ScanTour T;
  T.g_tour = A.tours + (long long)t * A.n;
  T.arrays = SMEM ? dsm : A.ws + (size_t)t * A.ws_tour_bytes;
  T.n = A.n;
  T.k = A.k;
  T.ds = A.ds;
  T.packed = A.cand_packed;
  T.cand = A.cand;
  T.cand_dist = A.cand_dist;
  T.max_iter = A.max_iter;
  T.status = A.status ? A.status + t : nullptr;
  T.stats = A.stats ? A.stats + (long long)t * 4 : nullptr;
  T.accumulate = 0;
  T.moved = nullptr;
  T.converged = nullptr;
  T.rev_off = A.rev_off;
  T.rev_idx = A.rev_idx;
  T.budget = A.budget;
  T.symmetric = A.symmetric;
  scan_tour<MODE, THREADS, U, LAYOUT, false, COUNT>(T, S);
}

size_t two_opt_scan_tour_bytes(int n, int mode) { return scan_tour_state_bytes(n, mode); }

// First mode without stats needs no per-row counts: 16n bytes instead of 20n.
static bool scan_counts(const TwoOptArgs& a, int mode) { return mode == TSPB_MODE_FIRST && a.stats != nullptr; }

// Shared-memory carveout (percent of the unified L1/shared array) that holds exactly
// `ctas_per_sm` CTAs of `smem_per_cta` dynamic bytes; the rest stays L1 for the k-NN
// tables. The default lets the driver take the largest split, which leaves too little L1.
// An attribute of the current device (queried on every call: a process may drive GPUs of
// different models, and the query is cheap next to a launch).
static int current_device_attr(cudaDeviceAttr attr) {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, attr, dev) != cudaSuccess) return 0;
  return v;
}

int carveout_for(int ctas_per_sm, size_t smem_per_cta) {
  const int smem_sm = current_device_attr(cudaDevAttrMaxSharedMemoryPerMultiprocessor);
  if (smem_sm <= 0 || ctas_per_sm <= 0) return -1;
  const long long need = (long long)ctas_per_sm * (long long)(smem_per_cta + sizeof(ScanSmem) + 1024);
  int pct = (int)((need * 100 + smem_sm - 1) / smem_sm);
  return pct < 1 ? 1 : (pct > 100 ? 100 : pct);
}

static int carveout_percent(int num_tours, size_t smem_per_cta, int max_ctas_per_sm) {
  const int sms = current_device_attr(cudaDevAttrMultiProcessorCount);
  if (sms <= 0) return -1;
  int per_sm = (num_tours + sms - 1) / sms;
  if (per_sm > max_ctas_per_sm) per_sm = max_ctas_per_sm;
  return carveout_for(per_sm, smem_per_cta);
}

template <int MODE, int THREADS, int U>
static int launch_scan(const TwoOptArgs& a, size_t smem, cudaStream_t st) {
  // the grouped layout loads U packed words at once: k % U == 0 and a U*4-byte aligned table
  const bool aligned = (reinterpret_cast<uintptr_t>(a.cand_packed) % (U * sizeof(uint32_t))) == 0;
  const int layout = a.cand_packed ? (a.k % U == 0 && aligned ? SCAN_GROUPED : SCAN_PACKED) : SCAN_PLAIN;
  // best mode has no per-row counts: one instance serves both
  constexpr bool CAN_SKIP = MODE == TSPB_MODE_FIRST;
  auto pick = [&](auto smem_tag, auto count_tag) {
    constexpr bool SM = decltype(smem_tag)::value;
    constexpr bool CT = decltype(count_tag)::value || !CAN_SKIP;
    return layout == SCAN_GROUPED  ? two_opt_scan_kernel<MODE, THREADS, U, SCAN_GROUPED, SM, CT>
           : layout == SCAN_PACKED ? two_opt_scan_kernel<MODE, THREADS, U, SCAN_PACKED, SM, CT>
                                   : two_opt_scan_kernel<MODE, THREADS, U, SCAN_PLAIN, SM, CT>;
  };
  const bool count = scan_counts(a, MODE);
  auto kern = a.arrays_in_smem ? (count ? pick(std::true_type{}, std::true_type{}) : pick(std::true_type{}, std::false_type{}))
                               : (count ? pick(std::false_type{}, std::true_type{}) : pick(std::false_type{}, std::false_type{}));
  if (smem > 48 * 1024) TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int pct = carveout_percent(a.num_tours, smem, ScanMinBlocks<THREADS>::value);
  if (pct > 0) TSPB_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  kern<<<a.num_tours, THREADS, smem, st>>>(a);
  return tspb_launch_status();
}

template <int MODE>
static int launch_scan_mode(const TwoOptArgs& a, int threads, size_t smem, cudaStream_t st) {
  switch (threads) {
    case 64: return launch_scan<MODE, 64, 4>(a, smem, st);
    case 128: return launch_scan<MODE, 128, 4>(a, smem, st);
    case 512: {  // four entries per thread in flight only where the grouped layout applies
      const bool grouped = a.cand_packed && a.k % 4 == 0 && (reinterpret_cast<uintptr_t>(a.cand_packed) % 16) == 0;
      return grouped ? launch_scan<MODE, 512, 4>(a, smem, st) : launch_scan<MODE, 512, 2>(a, smem, st);
    }
    default: return launch_scan<MODE, 256, 4>(a, smem, st);
  }
}

int launch_two_opt_scan(const TwoOptArgs& a, int mode, int threads, cudaStream_t st) {
  const size_t smem = a.arrays_in_smem ? scan_tour_state_bytes(a.n, mode, false, scan_counts(a, mode)) : 0;
  if (mode == TSPB_MODE_BEST) return launch_scan_mode<TSPB_MODE_BEST>(a, threads, smem, st);
  return launch_scan_mode<TSPB_MODE_FIRST>(a, threads, smem, st);
}

__global__ void cand_pack_kernel(const int32_t* __restrict__ cand, const int32_t* __restrict__ cd, long long total,
                                 uint32_t* __restrict__ out, int32_t* __restrict__ overflow) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int c = __ldg(cand + e), d = __ldg(cd + e);
  if ((unsigned)c > 0xffffu || (unsigned)d > 0xffffu) {
    atomicOr(overflow, 1);
    out[e] = 0xffffu;  // an id >= n: the entry is skipped
    return;
  }
  out[e] = (uint32_t)c | ((uint32_t)d << 16);
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_candidate_pack(const int32_t* cand, const int32_t* cand_dist, int32_t n, int32_t k, uint32_t* packed,
                                   int32_t* overflow, void* stream) {
  if (n < 0 || k < 0) return TSPB_ERR_ARG;
  if (!overflow || (n > 0 && k > 0 && (!cand || !cand_dist || !packed))) return TSPB_ERR_ARG;
  if (n > 65535) return TSPB_ERR_UNSUPPORTED;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  TSPB_CUDA_CHECK(cudaMemsetAsync(overflow, 0, sizeof(int32_t), st));
  const long long total = (long long)n * k;
  if (total > 0) cand_pack_kernel<<<(int)((total + 255) / 256), 256, 0, st>>>(cand, cand_dist, total, packed, overflow);
  return tspb_launch_status();
}
