// Sweep kernel group (sqb_sweep.cuh): instantiations, launch set-up, and the
// kernel that builds the layered projector fields from the projector tables.
#include "sqb_sweep.cuh"

namespace sqb {

namespace {

// Per replica and ball point: its projector values into the replica's layer
// of the fields, and its first projector id into the point's id word.  The
// balls of one layer do not overlap, so every field value has one writer.
__global__ void fill_layers_kernel(int n_rep, const int4 *rep_box, const int *rep_gpb, const int *typ_nlocc,
                                   const long long *rep_off, const double *tab64, int ex, int ey, int ez, int pmax,
                                   unsigned short *lay_id16, double *lay_chi) {
  const long long evol = (long long)ex * ey * ez;
  for (int r = blockIdx.x; r < n_rep; r += gridDim.x) {
    const int4 b = rep_box[r];
    const int x0 = (short)(b.x & 0xffff), y0 = (short)(b.y & 0xffff), z0 = (short)(b.z & 0xffff);
    const int k = b.w & 0xff, np = (b.w >> 8) & 0xff, t = (b.w >> 16) & 0xff;
    const int Sd = 2 * typ_nlocc[t] + 1, sp2 = plane_stride(Sd);
    const int nb = Sd * Sd * Sd;
    const double *U = tab64 + rep_off[r];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
      const int bx = i % Sd, by = (i / Sd) % Sd, bz = i / (Sd * Sd);
      const int X = x0 + bx, Yc = y0 + by, Z = z0 + bz;
      if (X < 0 || X >= ex || Yc < 0 || Yc >= ey || Z < 0 || Z >= ez) continue;
      const long long g = ((long long)Z * ey + Yc) * ex + X;
      lay_id16[g * 4 + k] = (unsigned short)rep_gpb[r];
      for (int q = 0; q < np && q < pmax; q++)
        lay_chi[(long long)(k * pmax + q) * evol + g] = U[(long long)(q * Sd + bz) * sp2 + by * Sd + bx];
    }
  }
}

__global__ void fill_empty_kernel(unsigned long long *lay_id, long long evol, unsigned long long empty) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < evol; i += (long long)gridDim.x * blockDim.x)
    lay_id[i] = empty;
}

// Launch bounds of the instantiations (the register budget per thread is
// set by the warps per SM sub-partition).  Two rows per thread: windows up
// to 31 wide run 512 threads (16 warps, 128 registers), 33 wide 576 (96), up
// to 43 wide 1024.  Three rows per thread: up to 33 wide, 384 threads (12
// warps, 168 registers), for fields whose many dot-product accumulators
// spill at the smaller budgets.
constexpr int MAXT_A = 512, MAXT_B = 576, MAXT_C = 1024, MAXT_R3 = 384;

template <int PM, int FORM, int MAXT, int RY>
cudaError_t set_attr(size_t smem) {
  return cudaFuncSetAttribute(sweep::sweep_kernel<PM, FORM, MAXT, RY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem);
}

template <int PM, int FORM>
cudaError_t launch_form(const SweepArgs &a, int grid, int threads, size_t smem, cudaStream_t s) {
  if (a.ry == 3) {
    if (threads > MAXT_R3) return cudaErrorInvalidConfiguration;
    sweep::sweep_kernel<PM, FORM, MAXT_R3, 3><<<grid, threads, smem, s>>>(a);
  } else if (threads <= MAXT_A) sweep::sweep_kernel<PM, FORM, MAXT_A, 2><<<grid, threads, smem, s>>>(a);
  else if (threads <= MAXT_B) sweep::sweep_kernel<PM, FORM, MAXT_B, 2><<<grid, threads, smem, s>>>(a);
  else if (threads <= MAXT_C) sweep::sweep_kernel<PM, FORM, MAXT_C, 2><<<grid, threads, smem, s>>>(a);
  else return cudaErrorInvalidConfiguration;
  return cudaGetLastError();
}

template <int PM>
cudaError_t launch_pm(const SweepArgs &a, int grid, int threads, size_t smem, cudaStream_t s) {
  if (a.form == 0) return launch_form<PM, 0>(a, grid, threads, smem, s);
  if (a.form == 1) return launch_form<PM, 1>(a, grid, threads, smem, s);
  return launch_form<PM, 2>(a, grid, threads, smem, s);
}

template <int PM>
cudaError_t setup_pm(size_t smem) {
  cudaError_t r[12] = {set_attr<PM, 0, MAXT_A, 2>(smem),  set_attr<PM, 1, MAXT_A, 2>(smem),
                       set_attr<PM, 2, MAXT_A, 2>(smem),  set_attr<PM, 0, MAXT_B, 2>(smem),
                       set_attr<PM, 1, MAXT_B, 2>(smem),  set_attr<PM, 2, MAXT_B, 2>(smem),
                       set_attr<PM, 0, MAXT_C, 2>(smem),  set_attr<PM, 1, MAXT_C, 2>(smem),
                       set_attr<PM, 2, MAXT_C, 2>(smem),  set_attr<PM, 0, MAXT_R3, 3>(smem),
                       set_attr<PM, 1, MAXT_R3, 3>(smem), set_attr<PM, 2, MAXT_R3, 3>(smem)};
  for (cudaError_t e : r)
    if (e != cudaSuccess) return e;
  return cudaSuccess;
}

}  // namespace

int sweep_threads(int n, int ry) { return sweep::sweep_threads_of(n, ry); }

bool sweep_rows_supported(int n, int ry) {
  if (ry == 2) return sweep::sweep_threads_of(n, 2) <= MAXT_C;
  if (ry == 3) return sweep::sweep_threads_of(n, 3) <= MAXT_R3;
  return false;
}

size_t sweep_smem(int n, int pmax, int n_gproj, int ry) {
  const int nt = sweep::sweep_threads_of(n, ry);
  return sweep::shared_fixed() + sweep::planes_bytes(n, ry) + sweep::ring_bytes(nt, pmax, ry) +
         sweep::accw_bytes(nt, pmax, ry) + (((size_t)(n_gproj + pmax) * sizeof(double) + 127) & ~size_t(127));
}

size_t sweep_scratch_bytes(int n, int pmax) {
  const size_t nw = (size_t)n * n * n;
  return ((3 * nw + sweep::flush_doubles(n, pmax)) * sizeof(double) + 255) & ~size_t(255);
}

cudaError_t sweep_setup(int n) {
  (void)n;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  e = setup_pm<1>((size_t)optin);
  if (e == cudaSuccess) e = setup_pm<3>((size_t)optin);
  return e;
}

cudaError_t launch_sweep(const SweepArgs &a, int grid, cudaStream_t s) {
  const int threads = sweep_threads(a.n, a.ry);
  if (a.n > MAXN || !sweep_rows_supported(a.n, a.ry) || threads != a.nsweep) return cudaErrorInvalidConfiguration;
  const size_t smem = sweep_smem(a.n, a.pmax, a.n_gproj, a.ry);
  if (a.pmax == 1) return launch_pm<1>(a, grid, threads, smem, s);
  if (a.pmax == 3) return launch_pm<3>(a, grid, threads, smem, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_fill_layers(int n_rep, const int4 *rep_box, const int *rep_gpb, const int *typ_nlocc,
                               const long long *rep_off, const double *tab64, int ex, int ey, int ez, int pmax,
                               int n_gproj, unsigned long long *lay_id, double *lay_chi, cudaStream_t s) {
  const long long evol = (long long)ex * ey * ez;
  cudaError_t e = cudaMemsetAsync(lay_chi, 0, (size_t)LAYERS * pmax * evol * sizeof(double), s);
  if (e != cudaSuccess) return e;
  const unsigned long long empty = 0x0001000100010001ull * (unsigned long long)n_gproj;
  fill_empty_kernel<<<1024, 256, 0, s>>>(lay_id, evol, empty);
  e = cudaGetLastError();
  if (e != cudaSuccess || n_rep == 0) return e;
  fill_layers_kernel<<<n_rep < 4096 ? n_rep : 4096, 256, 0, s>>>(n_rep, rep_box, rep_gpb, typ_nlocc, rep_off, tab64,
                                                                  ex, ey, ez, pmax,
                                                                  reinterpret_cast<unsigned short *>(lay_id), lay_chi);
  return cudaGetLastError();
}

}  // namespace sqb
