// Node kernel group for the nonlocal forces (ForcesNonLocal): its own
// instantiation so the SQ kernel's register allocation does not carry it.
#include "sqb_node.cuh"

namespace sqb {

cudaError_t setup_node_forces(int n) { return setup_kind<KIND_FORCES>(n); }

cudaError_t launch_node_forces(const NodeArgs &args, int grid, int cols, cudaStream_t s) {
  return launch_kind<KIND_FORCES>(args, grid, cols, s);
}

}  // namespace sqb
