// multi_move 2-opt without any device allocation by the caller or the library.
//
// tspb_two_opt needs a global workspace for multi_move (the per-tour buffer in which the
// improving moves of a pass are sorted). Some callers cannot provide one: code that runs
// where cudaMalloc is not allowed or not wanted, e.g. inside a host callback or a
// real-time loop that must not touch the allocator, or a plugin host that owns all
// device memory and hands out only the input and output buffers. This entry point runs
// the same multi_move kernel on a fixed scratch array compiled into the library.
//
// The array is a file-scope __device__ variable of TSPB_STATIC_SCRATCH_BYTES; every GPU
// that loads the library holds it until the process exits. Host code cannot use the
// array's name as a device address, so the first call on each device looks the address
// up with cudaGetSymbolAddress (with that device current) and caches it. All calls share
// the one array: two calls whose kernels overlap on the GPU (different streams, or
// different host threads on the same device) race on it and must be serialised by the
// caller. The kernel writes every scratch slot it reads within a call, so nothing has to
// be cleared between calls.
#include <mutex>

#include "two_opt.cuh"

namespace tspb {

constexpr size_t STATIC_SCRATCH_BYTES = (size_t)TSPB_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_two_opt_static_scratch[STATIC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
static void* g_scratch_addr[MAX_DEVICES];
static std::mutex g_scratch_lock;

// Device address of the scratch array on the current device (looked up once per device).
static int static_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return TSPB_ERR_CUDA;
  std::lock_guard<std::mutex> guard(g_scratch_lock);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_two_opt_static_scratch) != cudaSuccess || p == nullptr) return TSPB_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return TSPB_OK;
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_two_opt_multi_move_static(int32_t* tours, int32_t num_tours, int32_t n, const int32_t* dist,
                                              int64_t dist_stride, const double* coords, const int32_t* cand,
                                              const int32_t* cand_dist, int32_t k, int64_t max_iterations,
                                              int32_t block_threads, int64_t* stats, int32_t* status, void* stream) {
  if (num_tours < 0 || n < 0) return TSPB_ERR_ARG;
  const size_t need = tspb_two_opt_workspace_bytes(num_tours, n, cand != nullptr ? k : 0, TSPB_MODE_MULTI_MOVE, block_threads);
  if (need > STATIC_SCRATCH_BYTES) return TSPB_ERR_WORKSPACE;
  void* scratch = nullptr;
  if (need > 0) {
    const int rc = static_scratch(&scratch);
    if (rc != TSPB_OK) return rc;
  }
  return tspb_two_opt(tours, num_tours, n, dist, dist_stride, coords, cand, cand_dist, nullptr, nullptr, nullptr, k,
                      TSPB_MODE_MULTI_MOVE, max_iterations, block_threads, stats, status, scratch,
                      need > 0 ? STATIC_SCRATCH_BYTES : 0, stream);
}
