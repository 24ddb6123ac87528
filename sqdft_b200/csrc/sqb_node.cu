// Node kernel group for the SQ step (Lanczos + moments, moments with given
// bounds, window matvec) and the host-side launch dispatch of all groups.
#include "sqb_node.cuh"

namespace sqb {

int g_smem_optin = 0;

int node_kernel_threads(int n, int cols) { return threads_of(n, cols); }

namespace {

// Per-plane stage footprint, maximised over every window origin of the block
// and every global z-plane: the sum over replicas whose ball crosses the
// plane and meets the window of nproj padded table planes.
__global__ void plane_footprint_kernel(int n, int nloc, int ox0, int oy0, int nx, int ny, int z0, int nz, int n_rep,
                                       const int *rep_nn, const int *typ_nlocc, const int *typ_nproj,
                                       unsigned *out) {
  const long long total = (long long)nx * ny * nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((long long)nx * ny));
    const int ox = ox0 + ix, oy = oy0 + iy, zg = z0 + iz;
    unsigned sum = 0;
    for (int r = 0; r < n_rep; r++) {
      const int t = rep_nn[4 * r + 3], nl = typ_nlocc[t], np = typ_nproj[t];
      if (np == 0) continue;
      const int rz = rep_nn[4 * r + 2];
      if (rz - nl > zg || rz + nl < zg) continue;
      const int rx = rep_nn[4 * r], ry = rep_nn[4 * r + 1];
      const int bx = min(rx + nl, ox + n - 1) - max(rx - nl, ox) + 1;
      const int by = min(ry + nl, oy + n - 1) - max(ry - nl, oy) + 1;
      if (bx <= 0 || by <= 0) continue;
      const int Sd = 2 * nl + 1, r0 = max(ry - nl, oy) - (ry - nl), r1 = min(ry + nl, oy + n - 1) - (ry - nl);
      sum += (unsigned)(np * ((((r1 + 1) * Sd + 3) & ~3) - ((r0 * Sd) & ~3)));
    }
    atomicMax(out, sum);
  }
  (void)nloc;
}

}  // namespace

size_t node_kernel_stage_bytes(int n, long long elems) {
  (void)n;
  return ((size_t)(elems > 0 ? elems : 1) * sizeof(double) + 15) & ~size_t(15);
}

cudaError_t launch_plane_footprint(int n, int nloc, const int *np, const int *pnode_s, int n_rep, const int *rep_nn,
                                   const int *typ_nlocc, const int *typ_nproj, unsigned *d_out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(unsigned), s);
  if (e != cudaSuccess || n_rep == 0) return e;
  const int nz = np[2] + 2 * nloc;
  const long long total = (long long)np[0] * np[1] * nz;
  const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
  plane_footprint_kernel<<<blocks, 256, 0, s>>>(n, nloc, pnode_s[0] - nloc, pnode_s[1] - nloc, np[0], np[1],
                                                pnode_s[2] - nloc, nz, n_rep, rep_nn, typ_nlocc, typ_nproj, d_out);
  return cudaGetLastError();
}

cudaError_t node_kernel_setup(int n) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&g_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (n > MAXN || stage_bytes_max(n, 0) == 0) return cudaErrorInvalidValue;
  e = setup_kind<KIND_SQ>(n);
  if (e == cudaSuccess) e = setup_node_forces(n);
  if (e == cudaSuccess) e = setup_node_vjp(n);
  if (e == cudaSuccess) e = setup_node_sq32(n);
  if (e == cudaSuccess) e = setup_node_lq(n);
  return e;
}

cudaError_t launch_node_kernel(const NodeArgs &args, int grid, int cols, cudaStream_t s) {
  if (args.mode == MODE_FORCES) return launch_node_forces(args, grid, cols, s);
  if (args.mode == MODE_VJP) return launch_node_vjp(args, grid, cols == -2 ? 0 : cols, s);
  if (args.mixed && args.mode == MODE_SQ) return launch_node_sq32(args, grid, cols, s);
  if (args.lq && args.mode == MODE_SQ) return launch_node_lq(args, grid, cols, s);
  return launch_kind<KIND_SQ>(args, grid, cols, s);
}

}  // namespace sqb
