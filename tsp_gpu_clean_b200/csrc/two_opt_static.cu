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
// that loads this file's module holds it until the process exits. Under lazy module
// loading (CUDA_MODULE_LOADING=LAZY, the default) the module, and with it the array, is
// loaded on a device by the first address lookup there, so the first call on each device
// is the moment the memory is reserved; callers that cannot allocate later make that call
// during their set-up. Host code cannot use the array's name as a device address, so the
// call looks the address up with cudaGetSymbolAddress (with that device current) and keeps
// it per device, together with the identity of the device's current context: when the
// context changes (cudaDeviceReset, or a primary context released and created again) the
// module is loaded anew and the address is looked up again instead of reusing a stale one.
// All calls share the one array: two calls whose kernels overlap on the GPU (different
// streams, or different host threads on the same device) race on it and must be
// serialised by the caller. The kernel writes every scratch slot it reads within a call,
// so nothing has to be cleared between calls.
#include <cuda.h>  // CUcontext / CUresult for the two driver entry points below

#include <mutex>

#include "two_opt.cuh"

namespace tspb {

constexpr size_t STATIC_SCRATCH_BYTES = (size_t)TSPB_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_two_opt_static_scratch[STATIC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
struct ScratchSlot {
  void* addr;
  unsigned long long ctx_id;  // context the address belongs to (0: unknown)
};
static ScratchSlot g_scratch[MAX_DEVICES];
static std::mutex g_scratch_lock;

using CtxGetCurrentFn = CUresult(CUDAAPI*)(CUcontext*);
using CtxGetIdFn = CUresult(CUDAAPI*)(CUcontext, unsigned long long*);

// Identity of the calling thread's current context (0 when it cannot be told): resolved
// through the runtime's driver entry points, so the library does not link libcuda.
static unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {  // under g_scratch_lock
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0{}, q1{};
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000, cudaEnableDefault, &q0) == cudaSuccess &&
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
        q0 == cudaDriverEntryPointSuccess && q1 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
      get_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    cudaGetLastError();
    resolved = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array in the current device's context.
static int static_scratch(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return TSPB_ERR_CUDA;
  std::lock_guard<std::mutex> guard(g_scratch_lock);
  ScratchSlot& s = g_scratch[dev];
  const unsigned long long ctx = current_context_id();  // 0 before the runtime has made one current
  if (s.addr == nullptr || ctx == 0 || s.ctx_id != ctx) {
    void* p = nullptr;
    // initialises the device's context when none is current, and loads the module
    const cudaError_t e = cudaGetSymbolAddress(&p, g_two_opt_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();  // leave no sticky launch error for the caller's next call
      s.addr = nullptr;
      return e == cudaErrorMemoryAllocation ? TSPB_ERR_DEVICE_MEMORY : TSPB_ERR_CUDA;
    }
    s.addr = p;
    s.ctx_id = current_context_id();  // the context the lookup ran in
  }
  *out = s.addr;
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
