// CUDA graphs of the library's own launches, captured and replayed through the C ABI.
//
// The GA engines enqueue one generation as a handful of kernel launches and replay it
// hundreds of times. Only this library's kernels are captured: no memory is allocated
// during capture, so the graph needs none of a framework's allocator bookkeeping. A host
// that holds the launches' stream captures them with tspb_graph_capture_begin /
// tspb_graph_capture_end and replays the executable graph with tspb_graph_launch.
#include "common.cuh"

extern "C" {

int tspb_graph_capture_begin(void* stream) {
  if (stream == nullptr) return TSPB_ERR_ARG;  // the legacy default stream cannot be captured
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // relaxed: the launch functions query attributes and occupancy while the stream captures
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed) != cudaSuccess) return TSPB_ERR_CUDA;
  return TSPB_OK;
}

int tspb_graph_capture_end(void* stream, void** exec_out) {
  if (stream == nullptr || exec_out == nullptr) return TSPB_ERR_ARG;
  *exec_out = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (e != cudaSuccess || graph == nullptr) {
    if (graph != nullptr) cudaGraphDestroy(graph);
    cudaGetLastError();
    return TSPB_ERR_CUDA;
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiateWithFlags(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return TSPB_ERR_CUDA;
  }
  // upload once now, so the first replay does not pay for it inside a timed loop
  if (cudaGraphUpload(exec, s) != cudaSuccess) {
    cudaGraphExecDestroy(exec);
    return TSPB_ERR_CUDA;
  }
  *exec_out = exec;
  return TSPB_OK;
}

int tspb_graph_launch(void* exec, void* stream) {
  if (exec == nullptr) return TSPB_ERR_ARG;
  if (cudaGraphLaunch(static_cast<cudaGraphExec_t>(exec), static_cast<cudaStream_t>(stream)) != cudaSuccess)
    return TSPB_ERR_CUDA;
  return TSPB_OK;
}

int tspb_graph_destroy(void* exec) {
  // an executable graph still in flight is freed when its launches complete
  if (exec == nullptr) return TSPB_OK;
  return cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(exec)) == cudaSuccess ? TSPB_OK : TSPB_ERR_CUDA;
}

}  // extern "C"
