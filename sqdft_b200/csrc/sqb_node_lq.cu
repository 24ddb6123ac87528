// Node kernel group for the Lanczos-quadrature SQ step (bounds and Chebyshev
// moments from one FP64 Lanczos run per node): its own instantiation so the
// other groups' register allocation does not carry it.
#include "sqb_node.cuh"

namespace sqb {

cudaError_t setup_node_lq(int n) { return setup_kind<KIND_LQ>(n); }

cudaError_t launch_node_lq(const NodeArgs &args, int grid, int cols, cudaStream_t s) {
  return launch_kind<KIND_LQ>(args, grid, cols, s);
}

}  // namespace sqb
