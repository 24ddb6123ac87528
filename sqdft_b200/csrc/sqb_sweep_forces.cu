// ForcesNonLocal on the sweep kernel (node_forces in sqb_sweep.cuh), in its
// own translation unit so its register allocation is its own.
#include "sqb_sweep.cuh"

namespace sqb {

namespace {

// as the SQ instantiations (sqb_sweep.cu)
constexpr int MAXT_A = 512, MAXT_B = 576, MAXT_C = 1024, MAXT_R3 = 384;

template <int PM, typename T, int MAXT, int RY>
cudaError_t set_attr(size_t smem) {
  return cudaFuncSetAttribute(sweep::sweep_force_kernel<PM, T, MAXT, RY>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int PM, typename T>
cudaError_t launch_t(const SweepArgs &a, int grid, int threads, size_t smem, cudaStream_t s) {
  if (a.ry == 3) {
    if (threads > MAXT_R3) return cudaErrorInvalidConfiguration;
    sweep::sweep_force_kernel<PM, T, MAXT_R3, 3><<<grid, threads, smem, s>>>(a);
  } else if (threads <= MAXT_A) sweep::sweep_force_kernel<PM, T, MAXT_A, 2><<<grid, threads, smem, s>>>(a);
  else if (threads <= MAXT_B) sweep::sweep_force_kernel<PM, T, MAXT_B, 2><<<grid, threads, smem, s>>>(a);
  else if (threads <= MAXT_C) sweep::sweep_force_kernel<PM, T, MAXT_C, 2><<<grid, threads, smem, s>>>(a);
  else return cudaErrorInvalidConfiguration;
  return cudaGetLastError();
}

template <int PM>
cudaError_t setup_pm(size_t smem) {
  cudaError_t r[8] = {set_attr<PM, double, MAXT_A, 2>(smem),  set_attr<PM, float, MAXT_A, 2>(smem),
                      set_attr<PM, double, MAXT_B, 2>(smem),  set_attr<PM, float, MAXT_B, 2>(smem),
                      set_attr<PM, double, MAXT_C, 2>(smem),  set_attr<PM, float, MAXT_C, 2>(smem),
                      set_attr<PM, double, MAXT_R3, 3>(smem), set_attr<PM, float, MAXT_R3, 3>(smem)};
  for (cudaError_t e : r)
    if (e != cudaSuccess) return e;
  return cudaSuccess;
}

}  // namespace

cudaError_t sweep_forces_setup(int n) {
  (void)n;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  e = setup_pm<1>((size_t)optin);
  if (e == cudaSuccess) e = setup_pm<3>((size_t)optin);
  return e;
}

cudaError_t launch_sweep_forces(const SweepArgs &a, int single, int grid, cudaStream_t s) {
  const int threads = sweep_threads(a.n, a.ry);
  if (a.n > MAXN || !sweep_rows_supported(a.n, a.ry) || threads != a.nsweep) return cudaErrorInvalidConfiguration;
  const size_t smem = sweep_smem(a.n, a.pmax, a.n_gproj, a.ry);
  if (a.pmax == 1) return single ? launch_t<1, float>(a, grid, threads, smem, s) : launch_t<1, double>(a, grid, threads, smem, s);
  if (a.pmax == 3) return single ? launch_t<3, float>(a, grid, threads, smem, s) : launch_t<3, double>(a, grid, threads, smem, s);
  return cudaErrorInvalidValue;
}

}  // namespace sqb
