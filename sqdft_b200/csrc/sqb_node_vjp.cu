// Node kernel group for the adjoint (reverse Chebyshev) gradient: its own
// instantiation so the SQ kernel's register allocation does not carry it.
#include "sqb_node.cuh"

namespace sqb {

cudaError_t setup_node_vjp(int n) { return setup_kind<KIND_VJP>(n); }

cudaError_t launch_node_vjp(const NodeArgs &args, int grid, int cols, cudaStream_t s) {
  return launch_kind<KIND_VJP>(args, grid, cols, s);
}

}  // namespace sqb
