// Node kernel group for the SQ step of the FP32-mixed path (Lanczos vectors
// stored in FP32, FP64 moments): its own instantiation so the FP64 SQ
// kernel's register allocation does not carry it.
#include "sqb_node.cuh"

namespace sqb {

cudaError_t setup_node_sq32(int n) { return setup_kind<KIND_SQ32>(n); }

cudaError_t launch_node_sq32(const NodeArgs &args, int grid, int cols, cudaStream_t s) {
  return launch_kind<KIND_SQ32>(args, grid, cols, s);
}

}  // namespace sqb
