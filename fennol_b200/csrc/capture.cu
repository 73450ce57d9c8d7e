// CUDA-graph helper for the neighbour-list update inside a captured MD step.
//
// FeNNol's driver decides between a full rebuild and a skin update on the host
// every step (md/integrate.py:515-565).  Here the MD kernel raises a device
// flag when an atom has moved more than half the skin, and the captured step
// holds the rebuild kernels in the body of a conditional IF node: a one-thread
// kernel copies the flag into the node's condition, so a replay runs the
// rebuild only when it is due, with no host round trip and no launches of
// rebuild kernels that would return at once.
#include "common.cuh"

namespace {

__global__ void k_set_condition(cudaGraphConditionalHandle h, const int* __restrict__ flag) {
  cudaGraphSetConditional(h, *flag != 0 ? 1u : 0u);
}

}  // namespace

extern "C" int fennol_capture_if_begin(void* stream, const int* flag, void* body_stream) {
  if (!flag || !body_stream || body_stream == stream) return FENNOL_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  cudaStream_t bs = (cudaStream_t)body_stream;
  cudaStreamCaptureStatus status;
  cudaGraph_t graph;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  if (cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps) != cudaSuccess)
    return FENNOL_ERR_CUDA;
  if (status != cudaStreamCaptureStatusActive) return FENNOL_ERR_UNSUPPORTED;
  cudaStreamCaptureStatus body_status;
  if (cudaStreamIsCapturing(bs, &body_status) != cudaSuccess || body_status != cudaStreamCaptureStatusNone)
    return FENNOL_ERR_INVALID;
  // the condition is reset to 0 at every launch of the graph and set by the
  // kernel below before the node is reached
  cudaGraphConditionalHandle h;
  if (cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault) != cudaSuccess)
    return FENNOL_ERR_CUDA;
  k_set_condition<<<1, 1, 0, st>>>(h, flag);
  if (cudaGetLastError() != cudaSuccess) return FENNOL_ERR_CUDA;
  if (cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps) != cudaSuccess)
    return FENNOL_ERR_CUDA;
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  if (cudaGraphAddNode(&node, graph, deps, ndeps, &np) != cudaSuccess) return FENNOL_ERR_CUDA;
  if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
    return FENNOL_ERR_CUDA;
  cudaGraph_t body = np.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
    return FENNOL_ERR_CUDA;
  return FENNOL_OK;
}

extern "C" int fennol_capture_if_end(void* body_stream) {
  if (!body_stream) return FENNOL_ERR_INVALID;
  cudaGraph_t g = nullptr;
  if (cudaStreamEndCapture((cudaStream_t)body_stream, &g) != cudaSuccess) return FENNOL_ERR_CUDA;
  return FENNOL_OK;
}
