#pragma once
// Sweep kernel: the per-grid-node work of the SQ step (Lanczos bounds and
// Chebyshev moments, ClenshawCurtisSpectralQuadrature sq.cpp:530-661) on
// sm_100a, built around a branch-free nonlocal term.
//
// One persistent CTA per SM takes grid nodes from an atomic queue.  Every
// matvec H v = -1/2 Lap_h v + Veff v + Vnl v on a node's (2nloc+1)^3 window
// (HsubTimesVec sq.cpp:838-929, VnlocsubTimesVec nonlocal.cpp:20-215; v zero
// outside the window) is one sweep over the window's z-planes:
//   * each thread owns one window column x and RY adjacent rows y; it writes
//     its centre values into a shared-memory plane with a zero halo of 6, so
//     the x and y neighbours are unconditional loads (the window truncation
//     falls out of the halo); the RY rows share their y-arm loads;
//   * the 2 FDN + 1 planes of a column's stencil: the centre and the FDN
//     planes ahead in registers, the FDN planes behind in the thread's own
//     slots of a shared ring (no barrier: no other thread reads them);
//   * the shared planes rotate through three buffers under a split barrier:
//     a thread writes plane z + 1 and arrives on an mbarrier before it works
//     on plane z, and waits for that phase (bounded) only afterwards, so
//     warps drift by up to a plane instead of meeting at every plane;
//   * the nonlocal term reads the layered projector fields (sqb_internal.cuh):
//     per point and layer one 16-bit projector base and the projector values,
//     so the gather sum_J c_J chi_J(x) is a fixed loop over four layers with
//     no per-box control flow, c_J read from a shared array indexed by the
//     global projector id;
//   * the dot products chi_J . w of the sweep's output w, which the next
//     matvec needs, are accumulated per thread along z for each layer; when a
//     column leaves a ball (the layer's id changes) the column's partial sum
//     goes to the CTA's flush buffer in global memory, at the slot of (layer,
//     the ball's last window plane, column), which no other ball shares; after
//     the last plane every warp sums whole balls from it in a fixed order:
//     deterministic, one reduction per ball per sweep, none inside the plane
//     loop.
// Lanczos keeps the reference's recurrence, start vector and convergence test
// (sq.cpp:965-1092) with one sweep per step: the sweep forms the next
// unnormalised Lanczos vector from the stored vectors while loading it, and
// the block then finds the extreme eigenvalues of the tridiagonal (the
// quantities TridiagEigenSolve sq.cpp:1094-1180 returns) by a 257-way
// multisection.  Chebyshev moments use the reference's doubling identities
// (sq.cpp:564-655).  The Lanczos-quadrature form takes bounds and moments from
// one Lanczos run started at the node (Gauss-quadrature identity).
#include <cmath>
#include <cstdio>
#include <type_traits>

#include "sqb_internal.cuh"

namespace sqb {
namespace sweep {

constexpr int KL = LAYERS;
constexpr int RY_DEFAULT = 2;  // window rows per thread (3 for fields with three projectors per slot)

// Sweep kinds: the Lanczos start vector's projections only; a Lanczos step;
// a Chebyshev step; a Chebyshev step that also accumulates the density-matrix
// column D += c t_k+1 / h^3 (ForcesNonLocal).
enum : int { SK_ONES = 0, SK_LZF = 1, SK_CH = 2, SK_FD = 3 };

struct Shared {
  unsigned long long pbar;  // plane barrier of the sweeps (mbarrier, one arrival per thread and plane)
  unsigned pbar_phase;      // its phases completed so far
  int wabort;               // a plane wait ran out of time: later waits are skipped
  int node, qidx, gi, gj, gk;
  int n_ent, n_pi;
  int stop, count;
  double center_val;
  double scal[2];
  double red[32][2];
  double red3[32][3];
  double scal2[3];
  double aa[MAXL];
  double bb[MAXL];
  double eig[2], eprev[2];
  double wdel[2];   // last changes of the extremes (warm start of the next multisection)
  int warm;         // eig holds the extremes of the previous, one row smaller tridiagonal
  double br[2][2];  // multisection brackets (lambda_min, lambda_max)
  int wres[32];     // per-warp multisection results
  int scan[33];
  // boxes (replica balls meeting the window), window coordinates
  short e_x0[MAXE], e_x1[MAXE], e_y0[MAXE], e_y1[MAXE], e_z0[MAXE], e_z1[MAXE];
  unsigned char e_k[MAXE], e_np[MAXE], e_t[MAXE];
  short e_pb[MAXE];  // first local projector instance
  int e_gpb[MAXE];   // first global projector id
  int e_atom[MAXE];  // global atom (force passes)
  // local projector instances p < n_pi
  short pi_e[MAXP];
  int pi_g[MAXP];
  double p_nxt[MAXP];  // chi^T w of the sweep's output
  double p_in[MAXP];   // chi^T W of a Lanczos sweep's input (one projector per layer slot)
  double p_den[MAXP];
  double pw_cur[MAXP];   // Lanczos: chi^T W_m
  double pw_prev[MAXP];  // Lanczos: chi^T W_m-1
};

__host__ __device__ constexpr int plane_pitch(int n) { return n + 2 * FDN; }
// Halo'd planes of the stencil input: plane z lives in buffer z mod NPLANE.
// Three buffers let a thread write plane z + 1 before it works on plane z
// while the slowest thread may still read plane z - 1 (see sweep).
constexpr int NPLANE = 3;
// NPLANE halo'd planes, plus ry - 1 rows of slack: the shared y-arm loads of
// a row group whose last rows lie beyond the window read up to ry - 1 rows
// past the plane (into values that are not used)
__host__ __device__ inline size_t planes_bytes(int n, int ry) {
  const int P = plane_pitch(n);
  return ((size_t)(NPLANE * P * P + (ry - 1) * P + 8) * sizeof(double) + 127) & ~size_t(127);
}
// Lanczos sweeps of the one-projector fields also accumulate the dot products
// of their input (the exact chi^T W_m, see lanczos), flushed into a second
// set of the flush buffer.  The buffer (per CTA, after the three window
// vectors in the scratch) holds [set][layer][projector][plane][column].
__host__ __device__ constexpr bool input_dots(int pm) { return pm == 1; }
__host__ __device__ inline size_t flush_doubles(int n, int pm) {
  return (size_t)(input_dots(pm) ? 2 : 1) * KL * pm * n * n * n;
}
__host__ __device__ inline size_t shared_fixed() { return (sizeof(Shared) + 127) & ~size_t(127); }
// The threads' rings of the FDN planes behind (RSLOT slots, sized for FP64).
constexpr int RSLOT = 8;
__host__ __device__ constexpr bool uses_ring(int pm) { return pm >= 1; }
__host__ __device__ inline size_t ring_bytes(int nsweep, int pm, int ry) {
  return uses_ring(pm) ? (((size_t)RSLOT * ry * nsweep * sizeof(double) + 127) & ~size_t(127)) : 0;
}
// Lanczos sweeps' input-dot partials, one slot per (layer, row, thread): the
// owning thread accumulates, flushes and clears its own slots.
__host__ __device__ inline size_t accw_bytes(int nsweep, int pm, int ry) {
  return input_dots(pm) ? (((size_t)KL * ry * nsweep * sizeof(double) + 127) & ~size_t(127)) : 0;
}
__host__ __device__ inline int sweep_threads_of(int n, int ry) {
  const int groups = (n + ry - 1) / ry;
  const int t = n <= 32 ? 32 * groups : ((n * groups + 31) / 32) * 32;  // see the thread mapping in sweep
  return t < 64 ? 64 : t;  // two warps at least: the multisection's two extremes
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Barrier of the block's threads inside a sweep (named barrier 1).
__device__ __forceinline__ void bar_sweep(int nthreads) {
  asm volatile("bar.sync 1, %0;\n" ::"r"(nthreads) : "memory");
}

// The plane barrier: an mbarrier in shared memory that every thread of the
// block arrives on once per plane (release: its plane writes are visible to
// the threads whose wait on that phase returns, acquire).
__device__ __forceinline__ unsigned pbar_addr(const unsigned long long *bar) {
  return (unsigned)__cvta_generic_to_shared(bar);
}
__device__ __forceinline__ void pbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(pbar_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void pbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(pbar_addr(bar)) : "memory");
}
__device__ __forceinline__ bool pbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(pbar_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long gtimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Every thread of the block arrives once per plane, so a phase completes in
// microseconds; a wait that outlasts PBAR_WAIT_NS means a thread stopped
// arriving: the wait sets the status bit and the block's abort flag, after
// which no plane wait blocks (the step's results are then void and the call
// returns an error).
constexpr unsigned long long PBAR_WAIT_NS = 2000000000ull;
__device__ __forceinline__ void pbar_wait(Shared &S, int *status, unsigned phase) {
  if (*(volatile int *)&S.wabort) return;
  const unsigned parity = phase & 1u;
  if (pbar_try_wait(&S.pbar, parity)) return;
  const unsigned long long t0 = gtimer_ns();
  while (!pbar_try_wait(&S.pbar, parity)) {
    if (gtimer_ns() - t0 > PBAR_WAIT_NS) {
      *(volatile int *)&S.wabort = 1;
      atomicOr(status, ST_WAIT_LIMIT);
      return;
    }
  }
}
// Set up the plane barrier at the start of a kernel (before any sweep).
__device__ __forceinline__ void pbar_setup(Shared &S) {
  if (threadIdx.x == 0) {
    pbar_init(&S.pbar, blockDim.x);
    S.pbar_phase = 0u;
    S.wabort = 0;
  }
  __syncthreads();
}

template <typename T>
struct IO {
  const T *vin = nullptr;  // stencil input (LZF: Y = H W_m-1; CH: t_k)
  T *out = nullptr;        // output (LZF: H W_m; CH: t_k+1)
  const T *p1 = nullptr;   // LZF: W_m-1; CH: t_k-1
  const T *p2 = nullptr;   // LZF: W_m-2
  T *wout = nullptr;       // LZF: where the formed W_m is stored
  double s1 = 1.0;         // LZF: W_m = s1 (Y - ca W1) - cb W2
  double ca = 0.0, cb = 0.0;  // LZF: a, b s; CH: chi, zee
  double sin = 1.0;        // LZF konst 1: scale of the start vector
  double chk = 0.0;        // start vector 1 + chk (-1)^(x+y+z)
  int konst = 0;           // input generated: 1 the (scaled) start vector, 2 the node's unit vector e_c
  int p1_delta = 0;        // CH: t_k-1 is e_c
  int first = 0;           // CH: t_1 = (H t_0 - chi t_0) / zee (no t_k-1 term)
  int dbl = 0;             // CH: accumulate <t_k+1, t_k+1> and <t_k+1, t_k> (doubling)
  double *dacc = nullptr;  // FD: density-matrix column, FP64
  double cd = 0.0, ce = 0.0;  // FD: D += t_k+1 cd / h^3 (first: D = e_c ce / h^3 + t_1 cd / h^3)
};

// Lanczos start vector at window index g: 1 + chk (-1)^(x+y+z); the window
// edge n is odd, so x + y + z and g = (z n + y) n + x have the same parity.
__device__ __forceinline__ double start_val(double chk, int g) { return 1.0 + chk * (1.0 - 2.0 * (double)(g & 1)); }

__device__ __forceinline__ unsigned lay_of(unsigned long long w, int k) {
  return (unsigned)(w >> (16 * k)) & 0xffffu;
}

template <typename T>
__device__ __forceinline__ T *slot(const SweepArgs &a, int k) {
  const size_t nw = (size_t)a.n * a.n * a.n;
  return reinterpret_cast<T *>(a.scratch + blockIdx.x * a.scratch_stride + (size_t)k * nw * sizeof(double));
}

// Sum of one projector instance's flushed column partials over its box's
// columns, at the slots of its ball's last window plane (one warp, fixed
// order), into p_nxt; with IND also the input dots of the second set, into
// p_in.  The loads of a pass are independent, so they overlap.
template <int PM, bool IND>
__device__ __forceinline__ void reduce_instance(const SweepArgs &a, Shared &S, const double *fb, int p, int lane) {
  const int e = S.pi_e[p], q = p - S.e_pb[e], k = S.e_k[e];
  const int n = a.n, n2 = n * n;
  const int x0 = S.e_x0[e], y0 = S.e_y0[e];
  const int bx = S.e_x1[e] - x0 + 1, by = S.e_y1[e] - y0 + 1, cnt = bx * by;
  const int base = ((k * PM + q) * n + S.e_z1[e]) * n2 + y0 * n + x0, set = KL * PM * n * n2;
  const double *f = fb + base;
  const double *fw = f + set;
  (void)set;
  double s = 0.0, sw = 0.0;
#pragma unroll 4
  for (int i = lane; i < cnt; i += 32) {
    const int yy = i / bx, xx = i - yy * bx;
    const int o = SQB_IDX(base + yy * n + xx, set, a.status) - base;
    s += f[o];
    if constexpr (IND) sw += fw[o];
  }
  s = warp_sum(s);
  if constexpr (IND) sw = warp_sum(sw);
  if (lane == 0) {
    S.p_nxt[p] = s;
    if constexpr (IND) S.p_in[p] = sw;
  }
}

// One sweep over the window's z-planes (all threads of the block).  The
// stencil input of a thread's rows: with the ring, the centre and the FDN
// planes ahead in registers (fut[j][0] the centre, fut[j][s] plane z + s) and
// the FDN planes behind in the thread's own slots of a shared ring (plane
// z - s in slot (z - s) mod RSLOT); without it, all 2 FDN + 1 planes in
// registers (fut[j][FDN + s] plane z + s).
template <typename T, int PM, int SK, int RY>
__device__ __forceinline__ void sweep(const SweepArgs &a, Shared &S, unsigned char *dyn, const IO<T> &io,
                                      double &acc0, double &acc1) {
  constexpr bool STENCIL = SK != SK_ONES;
  constexpr bool CHEB = SK == SK_CH || SK == SK_FD;
  constexpr bool RING = uses_ring(PM);
  constexpr int F = RING ? FDN + 1 : 2 * FDN + 1;  // planes held in registers
  constexpr int C = RING ? 0 : FDN;                // register index of the centre
  constexpr bool CHR = PM == 1;  // projector values kept in registers from one plane to the next
  constexpr bool IND = SK == SK_LZF && input_dots(PM);  // dot products of the input too
  const int n = a.n, n2 = n * n, P = plane_pitch(n), P2 = P * P;
  const int tid = threadIdx.x, NS = a.nsweep, lane = tid & 31, warp = tid >> 5, nwarp = NS >> 5;
  // thread -> (column x, row group): windows up to 32 wide give each row
  // group a warp of its own (lane = column), so no warp straddles two row
  // groups and its shared-plane loads are one contiguous run (no bank
  // conflicts); wider windows pack the columns densely
  const int nrow = (n + RY - 1) / RY;
  const bool lanes = n <= 32;
  const int tx = lanes ? (tid & 31) : tid % n, tg = lanes ? (tid >> 5) : tid / n;
  const bool tv = tx < n && tg < nrow;
  const int x = tv ? tx : 0, yb = tv ? tg * RY : 0;
  const int nl = a.nloc, gc = (nl * n + nl) * n + nl;  // window index of the centre
  const int EP = a.ex * a.ey, EV = (int)a.evol;  // the extended grid fits 32-bit indices
  const unsigned dummy = (unsigned)a.n_gproj;
  const unsigned long long empty = 0x0001000100010001ull * (unsigned long long)dummy;  // no ball in any layer
  T *sm = reinterpret_cast<T *>(dyn);
  T *ring = reinterpret_cast<T *>(dyn + planes_bytes(n, RY));
  double *accw = reinterpret_cast<double *>(dyn + planes_bytes(n, RY) + ring_bytes(NS, PM, RY));
  const double *pcur =
      reinterpret_cast<const double *>(dyn + planes_bytes(n, RY) + ring_bytes(NS, PM, RY) + accw_bytes(NS, PM, RY));
  double *fb = slot<double>(a, 3);                // flush buffer: [set][layer][projector][plane][column]
  double *fbw = fb + (size_t)KL * PM * n * n2;  // IND: the input's set
  const double *veff = a.veff64;
  const unsigned long long *lid = a.lay_id;
  const double *lchi = a.lay_chi;
  const int NW = n * n2;                     // window points (vector length)
  int *const st = a.status;                  // (bounds-check build)
  (void)NW;
  (void)st;

  // zero the halo of the planes (the interior is written every plane)
  for (int i = tid; i < NPLANE * P2; i += NS) {
    const int r = (i % P2) / P, c = i % P;
    if (r < FDN || r >= n + FDN || c < FDN || c >= n + FDN) sm[i] = T(0);
  }

  int y[RY], col[RY];
  bool ok[RY];
  int xb[RY];
#pragma unroll
  for (int j = 0; j < RY; j++) {
    y[j] = yb + j;
    ok[j] = tv && y[j] < n;
    col[j] = ok[j] ? y[j] * n + x : 0;
    xb[j] = (S.gk * a.ey + (S.gj + (ok[j] ? y[j] : 0))) * a.ex + S.gi + x;
  }
  // ring slot of (row j, plane zz): ring[((zz mod RSLOT) * RY + j) * NS + tid]
  auto rslot = [&](int j, int zz) -> T & { return ring[(((zz + RSLOT) & (RSLOT - 1)) * RY + j) * NS + tid]; };

  // the stencil input of row j at plane zz (LZF: formed from the loaded operands)
  T fut[RY][F];
  T pf[RY], r1[RY], r2[RY];
  auto load_ops = [&](int j, int zz) {
    if (!ok[j] || zz >= n || io.konst) return;
    const int g = SQB_IDX(zz * n2 + col[j], NW, st);
    pf[j] = io.vin[g];
    if constexpr (SK == SK_LZF) {
      r1[j] = io.p1[g];
      r2[j] = io.p2[g];
    }
  };
  auto next_in = [&](int j, int zz) -> T {
    if (!ok[j] || zz >= n) return T(0);
    const int g = zz * n2 + col[j];
    T v;
    if (io.konst == 1) v = (T)(io.sin * start_val(io.chk, g));
    else if (io.konst == 2) v = (T)(g == gc ? 1.0 : 0.0);
    else if constexpr (SK == SK_LZF) v = (T)(io.s1 * ((double)pf[j] - io.ca * (double)r1[j]) - io.cb * (double)r2[j]);
    else v = pf[j];
    if constexpr (SK == SK_LZF) io.wout[SQB_IDX(g, NW, st)] = v;
    return v;
  };

  // per-plane point data, loaded one plane ahead
  double ve[RY];
  T q1[RY];
  double dq[RY];  // FD: D at the point, loaded one plane ahead
  unsigned long long idc[RY], idn[RY];
  double chc[RY][KL][PM];
  double acd[RY][KL][PM];
  // IND: the input's partial of (layer k, row j) lives in accw[(k RY + j) NS + tid]
  auto load_ids = [&](int j, int zz) -> unsigned long long {
    return (ok[j] && zz < n) ? __ldg(lid + SQB_IDX(xb[j] + zz * EP, EV, st)) : empty;
  };
  auto load_point = [&](int j, int zz) {
    if (!ok[j] || zz >= n) return;
    const int X = SQB_IDX(xb[j] + zz * EP, EV, st);
    if constexpr (STENCIL) ve[j] = __ldg(veff + X);
    if constexpr (CHEB) {
      if (!io.first)
        q1[j] = io.p1_delta ? (T)(zz * n2 + col[j] == gc ? 1.0 : 0.0) : io.p1[SQB_IDX(zz * n2 + col[j], NW, st)];
    }
    if constexpr (SK == SK_FD) dq[j] = io.first ? 0.0 : io.dacc[SQB_IDX(zz * n2 + col[j], NW, st)];
    if constexpr (CHR) {
#pragma unroll
      for (int k = 0; k < KL; k++)
        chc[j][k][0] = lay_of(idc[j], k) != dummy ? __ldg(lchi + k * EV + X) : 0.0;
    }
  };
  auto chi_at = [&](int j, int k, int q, int X) -> double {
    if constexpr (CHR) return chc[j][k][0];
    else return lay_of(idc[j], k) != dummy ? __ldg(lchi + (k * PM + q) * EV + X) : 0.0;
  };

#pragma unroll
  for (int j = 0; j < RY; j++) {
    ve[j] = 0.0;
    q1[j] = T(0);
    dq[j] = 0.0;
#pragma unroll
    for (int k = 0; k < KL; k++) {
      if constexpr (IND) accw[(k * RY + j) * NS + tid] = 0.0;
#pragma unroll
      for (int q = 0; q < PM; q++) acd[j][k][q] = chc[j][k][q] = 0.0;
    }
    idc[j] = load_ids(j, 0);
    idn[j] = load_ids(j, 1);
    if constexpr (STENCIL) {
      // planes behind the window are zero; planes 0..FDN enter it
      if constexpr (RING) {
#pragma unroll
        for (int s = 1; s <= FDN; s++) rslot(j, -s) = T(0);
      } else {
#pragma unroll
        for (int s = 0; s < FDN; s++) fut[j][s] = T(0);
      }
#pragma unroll
      for (int s = 0; s <= FDN; s++) {
        load_ops(j, s);
        fut[j][C + s] = next_in(j, s);
      }
      load_ops(j, FDN + 1);
    }
    load_point(j, 0);
  }
  const double c0 = 3.0 * a.coeff_lap[0];
  const double rcb = CHEB ? 1.0 / io.cb : 0.0;
  const double cdh = io.cd / a.h3, ceh = io.ce / a.h3;

  // Planes through the shared buffers with a split barrier: in step z a
  // thread first writes its centre values of plane z + 1 (buffer (z+1) mod 3)
  // and arrives, then works on plane z, and only then waits until every
  // thread has written plane z + 1.  A thread in step z has seen every thread
  // arrive in step z - 1, so the slowest is at worst in step z - 1, reading
  // buffer (z-1) mod 3: one buffer apart from the one written.  Warps drift
  // by up to a plane instead of meeting at every plane.
  const int sofs = (yb + FDN) * P + x + FDN;  // the thread's first row in a plane buffer
  if constexpr (STENCIL) {
#pragma unroll
    for (int j = 0; j < RY; j++)
      if (ok[j]) sm[sofs + j * P] = fut[j][C];
  }
  bar_sweep(NS);  // halo and plane 0 written; the previous sweep's phases are counted
  const unsigned ph0 = S.pbar_phase;
  int bz = 0;  // buffer of plane z
  for (int z = 0; z < n; z++) {
    T *smz = sm + bz * P2;
    const int bn = bz == NPLANE - 1 ? 0 : bz + 1;
    if constexpr (STENCIL) {
      if (z + 1 < n) {
#pragma unroll
        for (int j = 0; j < RY; j++)
          if (ok[j]) sm[bn * P2 + sofs + j * P] = fut[j][C + 1];
        pbar_arrive(&S.pbar);
      }
    }
    if (tv) {
      double hv[RY], v[RY];
      if constexpr (STENCIL) {
        // arm k of each point sums (x-k) + (x+k) + (y-k) + (y+k) + (z-k) + (z+k)
        // in that order before the coefficient, as HsubTimesVec does
        // (sq.cpp:894-897).  The RY rows y0..y0+RY-1 of a thread share their
        // y-arm loads: arm k loads rows y0-k (ym[k]) and y0+RY-1+k (yp[k]); row
        // j's y0+j-k is the centre of row j-k when j >= k, else ym[k-j], and
        // its y0+j+k the centre of row j+k when j+k < RY, else yp[j+k-RY+1].
        const T *cp0 = smz + (yb + FDN) * P + x + FDN;
        double temp[RY];
#pragma unroll
        for (int j = 0; j < RY; j++) temp[j] = (double)fut[j][C] * c0;
        if constexpr (RY == 2) {
          // the same, with the loads of the previous arm carried in two registers
          const T *c1p = cp0 + P;
          T prev_m = fut[0][C], prev_p = fut[1][C];
#pragma unroll
          for (int k = 1; k <= FDN; k++) {
            const T ym = cp0[-k * P], yp = c1p[k * P];
            const T zm0 = RING ? rslot(0, z - k) : fut[0][C - k], zm1 = RING ? rslot(1, z - k) : fut[1][C - k];
            const T s0 = cp0[-k] + cp0[k] + ym + prev_p + zm0 + fut[0][C + k];
            const T s1 = c1p[-k] + c1p[k] + prev_m + yp + zm1 + fut[1][C + k];
            temp[0] += (double)s0 * a.coeff_lap[k];
            temp[1] += (double)s1 * a.coeff_lap[k];
            prev_m = ym;
            prev_p = yp;
          }
        } else {
          T ym[FDN + 1], yp[FDN + 1];
#pragma unroll
          for (int k = 1; k <= FDN; k++) {
            ym[k] = cp0[-k * P];
            yp[k] = cp0[(RY - 1 + k) * P];
#pragma unroll
            for (int j = 0; j < RY; j++) {
              const T *cj = cp0 + j * P;
              const T ylo = j >= k ? fut[j - k][C] : ym[k - j];
              const T yhi = j + k < RY ? fut[j + k][C] : yp[j + k - RY + 1];
              const T zm = RING ? rslot(j, z - k) : fut[j][C - k];
              const T sj = cj[-k] + cj[k] + ylo + yhi + zm + fut[j][C + k];
              temp[j] += (double)sj * a.coeff_lap[k];
            }
          }
        }
#pragma unroll
        for (int j = 0; j < RY; j++) {
          const int X = xb[j] + z * EP;
          double vnl = 0.0;
#pragma unroll
          for (int k = 0; k < KL; k++) {
            const unsigned id = lay_of(idc[j], k);
#pragma unroll
            for (int q = 0; q < PM; q++) vnl += pcur[SQB_IDX(id + q, a.n_gproj + PM, st)] * chi_at(j, k, q, X);
          }
          v[j] = (double)fut[j][C];
          hv[j] = -0.5 * temp[j] + ve[j] * v[j] + vnl;
        }
      }
#pragma unroll
      for (int j = 0; j < RY; j++) {
        if (!ok[j]) continue;
        const int g = SQB_IDX(z * n2 + col[j], NW, st);
        double o;
        if constexpr (SK == SK_ONES) {
          o = start_val(io.chk, g);
        } else if constexpr (SK == SK_LZF) {
          const T ot = (T)hv[j];
          io.out[g] = ot;
          acc0 += v[j] * v[j];
          acc1 += v[j] * hv[j];
          o = (double)ot;
        } else {
          // sq.cpp:588, 615 divide by zee; the sweep multiplies by 1/zee
          // (one rounding apart, no FP64 division per point)
          double od;
          if (io.first) od = (hv[j] - io.ca * v[j]) * rcb;
          else od = (2.0 * (hv[j] - io.ca * v[j])) * rcb - (double)q1[j];
          const T ot = (T)od;
          io.out[g] = ot;
          o = (double)ot;
          if (io.dbl) {
            acc0 += o * o;
            acc1 += o * v[j];
          }
          if constexpr (SK == SK_FD) {  // forces.cpp:414-456 (Ci / h^3 formed once per sweep)
            if (io.first) io.dacc[g] = (g == gc ? ceh : 0.0) + o * cdh;
            else io.dacc[g] = dq[j] + o * cdh;
          }
        }
        if (g == gc) S.center_val = o;
        if (!isfinite(o)) atomicOr(a.status, ST_NONFINITE);
        const int X = xb[j] + z * EP;
#pragma unroll
        for (int k = 0; k < KL; k++) {
#pragma unroll
          for (int q = 0; q < PM; q++) acd[j][k][q] += chi_at(j, k, q, X) * o;
          if constexpr (IND) {
            if (lay_of(idc[j], k) != dummy) accw[(k * RY + j) * NS + tid] += chi_at(j, k, 0, X) * v[j];
          }
        }
        // a column that leaves a layer's ball after plane z flushes its partial
        // to the slot of (layer, z, column)
        const unsigned long long chg = idc[j] ^ idn[j];
        if (z + 1 < n && chg != 0ull) {
#pragma unroll
          for (int k = 0; k < KL; k++) {
            if (lay_of(chg, k) == 0u) continue;
            if (lay_of(idc[j], k) != dummy) {
#pragma unroll
              for (int q = 0; q < PM; q++) fb[SQB_IDX(((k * PM + q) * n + z) * n2 + col[j], KL * PM * NW, st)] = acd[j][k][q];
              if constexpr (IND) fbw[(k * n + z) * n2 + col[j]] = accw[(k * RY + j) * NS + tid];
            }
#pragma unroll
            for (int q = 0; q < PM; q++) acd[j][k][q] = 0.0;
            if constexpr (IND) accw[(k * RY + j) * NS + tid] = 0.0;
          }
        }
      }
    }
    // advance: ids, point data and the stencil input
#pragma unroll
    for (int j = 0; j < RY; j++) {
      idc[j] = idn[j];
      idn[j] = load_ids(j, z + 2);
      load_point(j, z + 1);
      if constexpr (STENCIL) {
        if constexpr (RING) rslot(j, z) = fut[j][0];  // plane z moves behind (its slot is free: RSLOT > FDN)
#pragma unroll
        for (int s = 0; s < F - 1; s++) fut[j][s] = fut[j][s + 1];
        fut[j][F - 1] = next_in(j, z + FDN + 1);
        load_ops(j, z + FDN + 2);
      }
    }
    if constexpr (STENCIL) {
      if (z + 1 < n) pbar_wait(S, a.status, ph0 + (unsigned)z);
    }
    bz = bn;
  }
  if constexpr (STENCIL) {
    // every thread read ph0 before its first arrival, and thread 0 passed
    // every wait of this sweep
    if (tid == 0) S.pbar_phase = ph0 + (unsigned)(n - 1);
  }
  // balls that end at the window's last plane: every layer's open partial (a
  // layer with no ball there writes a zero no reduction reads); then every
  // ball's columns are summed
  if (tv) {
#pragma unroll
    for (int j = 0; j < RY; j++) {
      if (!ok[j]) continue;
#pragma unroll
      for (int k = 0; k < KL; k++) {
#pragma unroll
        for (int q = 0; q < PM; q++) fb[((k * PM + q) * n + n - 1) * n2 + col[j]] = acd[j][k][q];
        if constexpr (IND) fbw[(k * n + n - 1) * n2 + col[j]] = accw[(k * RY + j) * NS + tid];
      }
    }
  }
  bar_sweep(NS);
  for (int p = warp; p < S.n_pi; p += nwarp) reduce_instance<PM, IND>(a, S, fb, p, lane);
  bar_sweep(NS);
}

// Sum of two values over the block into S.scal (deterministic).
static __device__ void sweep_sum2(Shared &S, double v0, double v1, int NS) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = NS >> 5;
  v0 = warp_sum(v0);
  v1 = warp_sum(v1);
  if (lane == 0) {
    S.red[warp][0] = v0;
    S.red[warp][1] = v1;
  }
  bar_sweep(NS);
  if (warp == 0) {
    double r0 = lane < nw ? S.red[lane][0] : 0.0;
    double r1 = lane < nw ? S.red[lane][1] : 0.0;
    r0 = warp_sum(r0);
    r1 = warp_sum(r1);
    if (lane == 0) {
      S.scal[0] = r0;
      S.scal[1] = r1;
    }
  }
  bar_sweep(NS);
}

// Sturm count: eigenvalues of the leading m x m tridiagonal (d, e) below x,
// from the sign changes of the characteristic-polynomial sequence
// p_i = (d_i - x) p_i-1 - e_i-1^2 p_i-2, rescaled by exact powers of two every
// eight rows (a row grows |p| by less than 2^64 here, far inside the range),
// which leaves every sign and rounding unchanged.  An exact zero counts as
// positive (a test point on an eigenvalue of a leading submatrix; the
// multisection's brackets tolerate the one-off count there).
static __device__ int sturm_count(const double *d, const double *e, int m, double x) {
  double p0 = 1.0, p1 = d[0] - x;
  int cnt = p1 < 0.0;
  for (int i = 1; i < m; i++) {
    const double p2 = (d[i] - x) * p1 - (e[i - 1] * e[i - 1]) * p0;
    cnt += (p2 < 0.0) != (p1 < 0.0);
    p0 = p1;
    p1 = p2;
    if ((i & 7) == 0) {
      const double mx = fmax(fabs(p0), fabs(p1));
      if (mx > 0x1p+600) {
        p0 *= 0x1p-600;
        p1 *= 0x1p-600;
      } else if (mx < 0x1p-600 && mx > 0.0) {
        p0 *= 0x1p+600;
        p1 *= 0x1p+600;
      }
    }
  }
  return cnt;
}

// Extreme eigenvalues of the m x m Lanczos tridiagonal (the quantities
// TridiagEigenSolve, sq.cpp:1094-1180, returns) into S.eig: the block's warps
// split into two groups, one per extreme, and each round every lane of a group
// evaluates a Sturm count at one of its 32 G points (G warps per group), so the
// bracket shrinks (32 G + 1)-fold per round, from the Gershgorin interval to
// four units in the last place.  All threads call it.
static __device__ void tridiag_extremes(Shared &S, int m) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int G = nw / 2, N = 32 * G;
  const int g = warp < G ? 0 : (warp < 2 * G ? 1 : 2);
  const int gi = warp - g * G;
  if (tid == 0) {
    const double *d = S.aa, *e = S.bb;
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < m; i++) {
      const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < m - 1 ? fabs(e[i]) : 0.0);
      lo = fmin(lo, d[i] - r);
      hi = fmax(hi, d[i] + r);
    }
    const double span = fmax(fabs(lo), fabs(hi));
    lo -= 1e-14 * span + 1e-300;
    hi += 1e-14 * span + 1e-300;
    S.br[0][0] = S.br[1][0] = lo;
    S.br[0][1] = S.br[1][1] = hi;
    if (S.warm) {
      // Warm start from the previous (one row smaller) tridiagonal's extremes:
      // by interlacing the new smallest lies at or below the old one and the
      // new largest at or above it; the other end of each bracket is the old
      // extreme moved by four times its last change, kept when a Sturm count
      // confirms that no eigenvalue lies beyond it.
      const double pad = 16.0 * 2.220446049250313e-16 * span;
      const double x0 = S.eig[0] - fmax(4.0 * S.wdel[0], 1e-9 * span), x1 = S.eig[1] + fmax(4.0 * S.wdel[1], 1e-9 * span);
      if (S.eig[0] + pad < hi) S.br[0][1] = S.eig[0] + pad;
      if (x0 > lo && sturm_count(d, e, m, x0) == 0) S.br[0][0] = x0;
      if (S.eig[1] - pad > lo) S.br[1][0] = S.eig[1] - pad;
      if (x1 < hi && sturm_count(d, e, m, x1) == m) S.br[1][1] = x1;
    }
  }
  __syncthreads();
  auto active = [&](int k) {
    const double lo = S.br[k][0], hi = S.br[k][1];
    return hi - lo > 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300;
  };
  for (int it = 0; it < 80; it++) {
    const bool a0 = active(0), a1 = active(1);
    if (!a0 && !a1) break;
    if (g < 2 && (g == 0 ? a0 : a1)) {
      const double lo = S.br[g][0], w = S.br[g][1] - lo;
      const int i = gi * 32 + lane;
      const int c = sturm_count(S.aa, S.bb, m, lo + w * (double)(i + 1) / (double)(N + 1));
      if (g == 0) {
        const unsigned below = __ballot_sync(0xffffffffu, c >= 1);
        if (lane == 0) S.wres[warp] = below ? gi * 32 + __ffs(below) - 1 : N;
      } else {
        const unsigned above = __ballot_sync(0xffffffffu, c < m);
        if (lane == 0) S.wres[warp] = above ? gi * 32 + 31 - __clz(above) : -1;
      }
    }
    __syncthreads();
    if (tid == 0) {
      const double inv = 1.0 / (double)(N + 1);
      if (a0) {  // smallest: the first point with an eigenvalue below it
        int f = N;
        for (int w = 0; w < G; w++) f = min(f, S.wres[w]);
        const double lo = S.br[0][0], w = S.br[0][1] - lo;
        if (f == N) {
          S.br[0][0] = lo + w * (double)N * inv;
        } else {
          S.br[0][1] = lo + w * (double)(f + 1) * inv;
          if (f > 0) S.br[0][0] = lo + w * (double)f * inv;
        }
      }
      if (a1) {  // largest: the last point with an eigenvalue above it
        int l = -1;
        for (int w = 0; w < G; w++) l = max(l, S.wres[G + w]);
        const double lo = S.br[1][0], w = S.br[1][1] - lo;
        if (l < 0) {
          S.br[1][1] = lo + w * inv;
        } else {
          if (l < N - 1) S.br[1][1] = lo + w * (double)(l + 2) * inv;
          S.br[1][0] = lo + w * (double)(l + 1) * inv;
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    S.eig[0] = 0.5 * (S.br[0][0] + S.br[0][1]);
    S.eig[1] = 0.5 * (S.br[1][0] + S.br[1][1]);
  }
  __syncthreads();
}

// The boxes of the replica balls meeting this node's window (the
// intersection test of nonlocal.cpp:66-108), their projector instances and
// the denominators.
static __device__ void setup_node(const SweepArgs &a, Shared &S) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int n = a.n;
  if (tid == 0) S.n_ent = 0;
  __syncthreads();
  for (int base = 0; base < a.n_rep; base += nt) {
    const int r = base + tid;
    bool hit = false;
    int4 b = make_int4(0, 0, 0, 0);
    int x0 = 0, x1 = 0, y0 = 0, y1 = 0, z0 = 0, z1 = 0;
    if (r < a.n_rep) {
      b = a.rep_box[r];
      x0 = max((int)(short)(b.x & 0xffff), S.gi) - S.gi;
      x1 = min(b.x >> 16, S.gi + n - 1) - S.gi;
      y0 = max((int)(short)(b.y & 0xffff), S.gj) - S.gj;
      y1 = min(b.y >> 16, S.gj + n - 1) - S.gj;
      z0 = max((int)(short)(b.z & 0xffff), S.gk) - S.gk;
      z1 = min(b.z >> 16, S.gk + n - 1) - S.gk;
      hit = x0 <= x1 && y0 <= y1 && z0 <= z1;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) S.scan[warp] = __popc(bal);
    __syncthreads();
    if (tid == 0) {
      int s = 0;
      for (int w = 0; w < nw; w++) {
        const int v = S.scan[w];
        S.scan[w] = s;
        s += v;
      }
      S.scan[32] = s;
    }
    __syncthreads();
    if (hit) {
      const int pos = S.n_ent + S.scan[warp] + __popc(bal & ((1u << lane) - 1u));
      if (pos < MAXE) {
        S.e_x0[pos] = (short)x0;
        S.e_x1[pos] = (short)x1;
        S.e_y0[pos] = (short)y0;
        S.e_y1[pos] = (short)y1;
        S.e_z0[pos] = (short)z0;
        S.e_z1[pos] = (short)z1;
        S.e_k[pos] = (unsigned char)(b.w & 0xff);
        S.e_np[pos] = (unsigned char)((b.w >> 8) & 0xff);
        S.e_t[pos] = (unsigned char)((b.w >> 16) & 0xff);
        S.e_gpb[pos] = a.rep_gpb[r];
        S.e_atom[pos] = a.rep_atom ? a.rep_atom[r] : -1;
      } else {
        atomicOr(a.status, ST_CAPACITY);
      }
    }
    __syncthreads();
    if (tid == 0) S.n_ent = min(S.n_ent + S.scan[32], MAXE);
    __syncthreads();
  }
  if (tid == 0) {
    int pb = 0, ne = S.n_ent;
    for (int e = 0; e < ne; e++) {
      if (pb + S.e_np[e] > MAXP) {
        atomicOr(a.status, ST_CAPACITY);
        ne = e;
        break;
      }
      S.e_pb[e] = (short)pb;
      pb += S.e_np[e];
    }
    S.n_ent = ne;
    S.n_pi = pb;
  }
  __syncthreads();
  for (int e = 0; e < S.n_ent; e++)
    for (int q = tid; q < S.e_np[e]; q += nt) {
      const int p = S.e_pb[e] + q;
      S.pi_e[p] = (short)e;
      S.pi_g[p] = S.e_gpb[e] + q;
      S.p_den[p] = a.proj_denom[S.e_t[e] * MAXPROJ_TYPE + q];
      S.p_nxt[p] = 0.0;
    }
  __syncthreads();
}

// chi^T e_c of every instance (the projector values at the window centre;
// zero for balls that do not hold it) into pw_cur, and c = chi^T e_c / Denom
// into the gather array.
static __device__ void centre_projections(const SweepArgs &a, Shared &S, double *pcur) {
  const int nl = a.nloc;
  const int X = ((S.gk + nl) * a.ey + (S.gj + nl)) * a.ex + S.gi + nl;
  for (int p = threadIdx.x; p < S.n_pi; p += blockDim.x) {
    const int e = S.pi_e[p], q = p - S.e_pb[e], k = S.e_k[e];
    const bool in = S.e_x0[e] <= nl && nl <= S.e_x1[e] && S.e_y0[e] <= nl && nl <= S.e_y1[e] && S.e_z0[e] <= nl &&
                    nl <= S.e_z1[e];
    const double c = in ? a.lay_chi[(k * a.pmax + q) * (int)a.evol + X] : 0.0;
    S.pw_cur[p] = c;
    S.pw_prev[p] = 0.0;
    pcur[S.pi_g[p]] = c / S.p_den[p];
  }
  __syncthreads();
}

// c_J = chi_J^T w / Denom_J of the last sweep's output into the gather array.
static __device__ void rotate(Shared &S, double *pcur) {
  for (int p = threadIdx.x; p < S.n_pi; p += blockDim.x) pcur[S.pi_g[p]] = S.p_nxt[p] / S.p_den[p];
  __syncthreads();
}

static __device__ void count_proj_points(const SweepArgs &a, Shared &S, long long steps, int cheb) {
  if (threadIdx.x != 0 || a.proj_points == nullptr) return;
  unsigned long long full = 0, win = 0;
  for (int e = 0; e < S.n_ent; e++) {
    const unsigned long long Sd = 2ull * a.typ_nlocc[S.e_t[e]] + 1ull;
    full += (unsigned long long)S.e_np[e] * Sd * Sd * Sd;
    win += (unsigned long long)S.e_np[e] * (S.e_x1[e] - S.e_x0[e] + 1) * (S.e_y1[e] - S.e_y0[e] + 1) *
           (S.e_z1[e] - S.e_z0[e] + 1);
  }
  atomicAdd(a.proj_points, full * (unsigned long long)steps);
  if (cheb) atomicAdd(a.proj_points + 1, full * (unsigned long long)steps);
  atomicAdd(a.proj_points + 2, win * (unsigned long long)steps);
}

// Lanczos bounds (sq.cpp:965-1092) in storage precision T, or (LQ) bounds and
// moments from one FP64 Lanczos run started at e_c.  Sweep m applies H to the
// unnormalised W_m = w_m-1 (v_m = s_m W_m), formed while it is loaded from the
// previous sweep's output Y_m-1 = H W_m-1 and the two previous W; it yields
// <W_m, W_m> = b_m-1^2 and <W_m, H W_m> = a_m b_m-1^2, so after sweep m the
// tridiagonal T_m+1 is complete and the reference's convergence test (both
// extremes moved by no more than the tolerance, at most 500 steps) applies.
// The projections chi^T W_m+1 the next gather needs follow from the recurrence
// on the dot products of the sweep's output.
template <typename T, int PM, bool LQ, int RY>
__device__ void lanczos(const SweepArgs &a, Shared &S, unsigned char *dyn, double *pcur, double &lmin_out,
                        double &lmax_out, int &rows_out) {
  const int tid = threadIdx.x;
  const double nw = (double)a.n * a.n * a.n;
  T *Y = slot<T>(a, 0);
  T *Wv[2] = {slot<T>(a, 1), slot<T>(a, 2)};
  const double chk = a.lz_chk;
  const double s0 = LQ ? 1.0 : 1.0 / sqrt(nw * (1.0 + chk * chk) + 2.0 * chk);
  const int kmin = a.npl / 2 + 1;
  double d0 = 0.0, d1 = 0.0;
  if constexpr (LQ) {
    centre_projections(a, S, pcur);  // W_0 = e_c
  } else {
    // chi^T W_0 for W_0 = (1 + chk (-1)^(x+y+z)) / norm (sq.cpp:538-546, 993-1004
    // with chk = 0)
    IO<T> io;
    io.chk = chk;
    sweep<T, PM, SK_ONES, RY>(a, S, dyn, io, d0, d1);
    __syncthreads();
    for (int p = tid; p < S.n_pi; p += blockDim.x) {
      S.pw_cur[p] = s0 * S.p_nxt[p];
      S.pw_prev[p] = 0.0;
      pcur[S.pi_g[p]] = S.pw_cur[p] / S.p_den[p];
    }
  }
  if (tid == 0) {
    S.stop = 0;
    S.count = 0;
    S.eprev[0] = S.eprev[1] = 0.0;
    S.warm = 0;
  }
  __syncthreads();
  double a_prev = 0.0, s_prev = 1.0, bs_prev = 0.0;
  for (int m = 0;; m++) {
    IO<T> io;
    io.out = Y;
    io.wout = Wv[m & 1];
    if (m == 0) {
      io.konst = LQ ? 2 : 1;
      io.chk = chk;
      io.sin = s0;
    } else {
      io.vin = Y;
      io.p1 = Wv[(m - 1) & 1];
      io.p2 = m >= 2 ? Wv[m & 1] : Wv[(m - 1) & 1];  // no third term in the first step (sq.cpp:1006-1014)
      io.s1 = s_prev;
      io.ca = a_prev;
      io.cb = bs_prev;
    }
    d0 = 0.0;
    d1 = 0.0;
    sweep<T, PM, SK_LZF, RY>(a, S, dyn, io, d0, d1);
    sweep_sum2(S, d0, d1, a.nsweep);
    // b_m-1 = |W_m| and a_m = <W_m, H W_m> / b_m-1^2 (W_0 is normalised)
    const double bm = m == 0 ? 1.0 : sqrt(S.scal[0]);
    const double am = S.scal[1] / (bm * bm);
    const double sm = 1.0 / bm;
    if (tid == 0) {
      S.aa[m] = am;
      if (m > 0) S.bb[m - 1] = bm;
    }
    __syncthreads();
    // after sweep m the tridiagonal has m + 1 rows (complete from m = 1; the
    // quadrature form follows its extremes from npl/2 rows on, so that the run
    // can stop at the npl/2 + 1 rows its moments need)
    const bool solve = LQ ? (m + 2 >= kmin) : (m >= 1);
    if (solve) {
      tridiag_extremes(S, m + 1);
      if (tid == 0) {
        const double dl = fabs(S.eig[0] - S.eprev[0]), dm = fabs(S.eig[1] - S.eprev[1]);
        S.eprev[0] = S.eig[0];
        S.eprev[1] = S.eig[1];
        S.wdel[0] = S.warm ? dl : 0.0;  // (the first solve's change is against zero)
        S.wdel[1] = S.warm ? dm : 0.0;
        S.warm = 1;
        const bool conv = !(dl > a.lanczos_tol || dm > a.lanczos_tol);
        if constexpr (LQ) {
          S.count = m + 1;  // rows of T; the first solve only sets the previous extremes
          S.stop = (m + 2 > kmin && conv) || S.count >= LANCZOS_MAX_ITER;
        } else {
          S.count = m;  // the reference's count after this step
          S.stop = conv || S.count >= LANCZOS_MAX_ITER;
        }
        if (S.count >= LANCZOS_MAX_ITER) atomicOr(a.status, ST_LANCZOS_MAXITER);
      }
      __syncthreads();
      if (S.stop) break;
    }
    // chi^T W_m+1 = s_m (chi^T Y_m - a_m chi^T W_m) - b_m-1 s_m-1 chi^T W_m-1.
    // With input dots the two older terms are the exact dot products of the
    // stored W_m and W_m-1, so only this step's rounding enters the gather of
    // the next sweep.  Without them (several projectors per layer slot) they
    // are the recurrence's own earlier values, whose rounding the three-term
    // recurrence amplifies like the Lanczos polynomials at 0: harmless for the
    // usual step counts when 0 lies inside the window's spectrum, growing
    // exponentially in the step count when it does not.
    const double bs_cur = m == 0 ? 0.0 : bm * s_prev;
    for (int p = tid; p < S.n_pi; p += blockDim.x) {
      const double wm = input_dots(PM) ? S.p_in[p] : S.pw_cur[p];
      const double nx = sm * (S.p_nxt[p] - am * wm) - bs_cur * S.pw_prev[p];
      S.pw_prev[p] = wm;
      S.pw_cur[p] = nx;
      pcur[S.pi_g[p]] = nx / S.p_den[p];
    }
    __syncthreads();
    a_prev = am;
    bs_prev = bs_cur;
    s_prev = sm;
  }
  lmin_out = S.eig[0] - a.lanczos_tol;
  lmax_out = S.eig[1] + a.lanczos_tol;
  rows_out = S.count;
}

// Chebyshev moments mu_j = e_c^T T_j((H - chi)/zee) e_c / h^3 (sq.cpp:564-655).
template <int PM, int RY>
__device__ void moments(const SweepArgs &a, Shared &S, unsigned char *dyn, double *pcur, double chi, double zee,
                        double *mu) {
  double *B0 = slot<double>(a, 0), *B1 = slot<double>(a, 1);
  double d0 = 0.0, d1 = 0.0;
  centre_projections(a, S, pcur);
  {  // t_1 = (H e_c - chi e_c) / zee
    IO<double> io;
    io.konst = 2;
    io.first = 1;
    io.out = B1;
    io.ca = chi;
    io.cb = zee;
    sweep<double, PM, SK_CH, RY>(a, S, dyn, io, d0, d1);
  }
  __syncthreads();
  rotate(S, pcur);
  const double htemp = S.center_val;
  if (threadIdx.x == 0) {
    mu[0] = (double)(1.0 / a.h3);
    mu[1] = (double)(htemp / a.h3);
  }
  double *t0 = B0, *t1 = B1;
  const int q1 = (int)rint(0.25 * a.npl), q2 = (int)rint(0.5 * a.npl);
  for (int nq = 2; nq <= q2; nq++) {
    {
      IO<double> io;
      io.vin = t1;
      io.p1 = t0;
      io.p1_delta = nq == 2;  // t_0 = e_c
      io.out = t0;
      io.ca = chi;
      io.cb = zee;
      io.dbl = nq > q1;
      d0 = 0.0;
      d1 = 0.0;
      sweep<double, PM, SK_CH, RY>(a, S, dyn, io, d0, d1);
      if (nq > q1) sweep_sum2(S, d0, d1, a.nsweep);
    }
    __syncthreads();
    rotate(S, pcur);
    if (threadIdx.x == 0) {
      mu[nq] = (double)(S.center_val / a.h3);
      if (nq > q1) {
        mu[2 * nq] = (double)((2 * S.scal[0] - 1) / a.h3);
        mu[2 * nq - 1] = (double)((2 * S.scal[1] - htemp) / a.h3);
      }
    }
    double *tt = t0;
    t0 = t1;
    t1 = tt;
  }
}

// Sum of three values over the block into S.scal2 (deterministic).
static __device__ void sweep_sum3(Shared &S, double v0, double v1, double v2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v0 = warp_sum(v0);
  v1 = warp_sum(v1);
  v2 = warp_sum(v2);
  if (lane == 0) {
    S.red3[warp][0] = v0;
    S.red3[warp][1] = v1;
    S.red3[warp][2] = v2;
  }
  __syncthreads();
  if (warp == 0) {
    double r0 = lane < nw ? S.red3[lane][0] : 0.0;
    double r1 = lane < nw ? S.red3[lane][1] : 0.0;
    double r2 = lane < nw ? S.red3[lane][2] : 0.0;
    r0 = warp_sum(r0);
    r1 = warp_sum(r1);
    r2 = warp_sum(r2);
    if (lane == 0) {
      S.scal2[0] = r0;
      S.scal2[1] = r1;
      S.scal2[2] = r2;
    }
  }
  __syncthreads();
}

// ForcesNonLocal for one node (forces.cpp:318-578): the density-matrix column
// D = sum_k Ci_k T_k((H - chi)/zee) e_c / h^3 by the full npl-step Chebyshev
// recursion (vectors in storage precision T, D in FP64, slot 2 of the
// scratch), then, on each ball that holds the window centre, the FD gradient
// of D (zero outside the window) contracted with the replica's projectors:
// f = -4 h^3 sum_q (chi_q . grad D) chi_q(centre) / Denom_q, into the node's
// force slots (atom, fx, fy, fz).
template <typename T, int PM, int RY>
__device__ void node_forces(const SweepArgs &a, Shared &S, unsigned char *dyn, double *pcur, double chi,
                            double zee, const double *ci, double *fslot) {
  T *B0 = slot<T>(a, 0), *B1 = slot<T>(a, 1);
  double *D = slot<double>(a, 2);
  double d0 = 0.0, d1 = 0.0;
  centre_projections(a, S, pcur);
  {  // t_1 = (H e_c - chi e_c) / zee; D = e_c Ci_0 / h^3 + t_1 Ci_1 / h^3
    IO<T> io;
    io.konst = 2;
    io.first = 1;
    io.out = B1;
    io.ca = chi;
    io.cb = zee;
    io.dacc = D;
    io.ce = ci[0];
    io.cd = ci[1];
    sweep<T, PM, SK_FD, RY>(a, S, dyn, io, d0, d1);
  }
  __syncthreads();
  rotate(S, pcur);
  T *t0 = B0, *t1 = B1;
  for (int nq = 2; nq <= a.npl; nq++) {  // t_nq = 2 (H - chi)/zee t_nq-1 - t_nq-2; D += t_nq Ci_nq / h^3
    IO<T> io;
    io.vin = t1;
    io.p1 = t0;
    io.p1_delta = nq == 2;  // t_0 = e_c
    io.out = t0;
    io.ca = chi;
    io.cb = zee;
    io.dacc = D;
    io.cd = ci[nq];
    sweep<T, PM, SK_FD, RY>(a, S, dyn, io, d0, d1);
    __syncthreads();
    rotate(S, pcur);
    T *tt = t0;
    t0 = t1;
    t1 = tt;
  }
  __threadfence_block();
  __syncthreads();
  const int n = a.n, nl = a.nloc, n2 = n * n, EV = (int)a.evol;
  int slotc = 0;
  for (int e = 0; e < S.n_ent; e++) {
    if (nl < S.e_x0[e] || nl > S.e_x1[e] || nl < S.e_y0[e] || nl > S.e_y1[e] || nl < S.e_z0[e] || nl > S.e_z1[e])
      continue;
    const int x0 = S.e_x0[e], y0 = S.e_y0[e], z0 = S.e_z0[e];
    const int bx = S.e_x1[e] - x0 + 1, by = S.e_y1[e] - y0 + 1, bz = S.e_z1[e] - z0 + 1, vol = bx * by * bz;
    const int k = S.e_k[e];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int q = 0; q < S.e_np[e]; q++) {
      const double *U = a.lay_chi + (size_t)(k * PM + q) * EV;
      double ax = 0.0, ay = 0.0, az = 0.0;
      for (int i = threadIdx.x; i < vol; i += blockDim.x) {
        const int x = x0 + i % bx, y = y0 + (i / bx) % by, z = z0 + i / (bx * by);
        const int w = SQB_IDX(z * n2 + y * n + x, n * n2, a.status);
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int kk = 1; kk <= FDN; kk++) {
          const double xm = x - kk >= 0 ? D[w - kk] : 0.0, xp = x + kk < n ? D[w + kk] : 0.0;
          const double ym = y - kk >= 0 ? D[w - kk * n] : 0.0, yp = y + kk < n ? D[w + kk * n] : 0.0;
          const double zm = z - kk >= 0 ? D[w - kk * n2] : 0.0, zp = z + kk < n ? D[w + kk * n2] : 0.0;
          gx += (-xm + xp) * a.coeff_grad[kk];
          gy += (-ym + yp) * a.coeff_grad[kk];
          gz += (-zm + zp) * a.coeff_grad[kk];
        }
        const double u = U[SQB_IDX(((S.gk + z) * a.ey + (S.gj + y)) * a.ex + S.gi + x, EV, a.status)];
        ax += u * gx;
        ay += u * gy;
        az += u * gz;
      }
      sweep_sum3(S, ax, ay, az);
      const double uc = U[((S.gk + nl) * a.ey + (S.gj + nl)) * a.ex + S.gi + nl];
      const double den = S.p_den[S.e_pb[e] + q];
      fx += S.scal2[0] / den * uc;
      fy += S.scal2[1] / den * uc;
      fz += S.scal2[2] / den * uc;
    }
    if (threadIdx.x == 0) {
      if (slotc < FSLOTS) {
        double *o = fslot + 4 * slotc;
        o[0] = (double)S.e_atom[e];
        o[1] = -4 * fx * a.h3;
        o[2] = -4 * fy * a.h3;
        o[3] = -4 * fz * a.h3;
      } else {
        atomicOr(a.status, ST_FSLOTS);
      }
    }
    slotc++;
    __syncthreads();
  }
  count_proj_points(a, S, a.npl, 1);
}

// The force pass over the listed nodes (bounds from chi, zee; Ci from ci).
template <int PM, typename T, int MAXT, int RY>
__global__ void __launch_bounds__(MAXT, 1) sweep_force_kernel(SweepArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  Shared &S = *reinterpret_cast<Shared *>(smem);
  unsigned char *dyn = smem + shared_fixed();
  double *pcur =
      reinterpret_cast<double *>(dyn + planes_bytes(a.n, RY) + ring_bytes(a.nsweep, PM, RY) + accw_bytes(a.nsweep, PM, RY));
  for (int i = threadIdx.x; i < a.n_gproj + PM; i += blockDim.x) pcur[i] = 0.0;  // [n_gproj..]: the empty id
  pbar_setup(S);
  for (;;) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(a.counter, 1);
      S.qidx = q;
      S.node = q < a.n_list ? a.node_list[q] : -1;
      if (S.node >= 0) {
        S.gi = S.node % a.np[0];
        S.gj = (S.node / a.np[0]) % a.np[1];
        S.gk = S.node / (a.np[0] * a.np[1]);
      }
    }
    __syncthreads();
    const int node = S.node;
    if (node < 0) break;
    double *fs = a.fslots + (size_t)S.qidx * FSLOTS * 4;
    for (int i = threadIdx.x; i < FSLOTS * 4; i += blockDim.x) fs[i] = (i % 4 == 0) ? -1.0 : 0.0;
    setup_node(a, S);
    node_forces<T, PM, RY>(a, S, dyn, pcur, a.chi[node], a.zee[node], a.ci + (size_t)node * (a.npl + 1), fs);
    __syncthreads();
  }
}

// Moments of the quadrature form: mu_j = e_1^T T_j((T_k - chi)/zee) e_1 / h^3
// on the k-row tridiagonal (one warp, k-vectors in the free window slots).
static __device__ void quadrature_moments(const SweepArgs &a, Shared &S, int k, double chi, double zee, double *mu) {
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  double *v0 = slot<double>(a, 0), *v1 = slot<double>(a, 1), *v2 = slot<double>(a, 2);
  for (int i = lane; i < k; i += 32) {
    v0[i] = i == 0 ? 1.0 : 0.0;
    v1[i] = i == 0 ? (S.aa[0] - chi) / zee : (i == 1 ? S.bb[0] / zee : 0.0);
  }
  __syncwarp();
  if (lane == 0) {
    mu[0] = 1.0 / a.h3;
    mu[1] = v1[0] / a.h3;
  }
  for (int j = 1; j < a.npl; j++) {
    for (int i = lane; i < k; i += 32) {
      double t = (S.aa[i] - chi) / zee * v1[i];
      if (i > 0) t += S.bb[i - 1] / zee * v1[i - 1];
      if (i + 1 < k) t += S.bb[i] / zee * v1[i + 1];
      v2[i] = 2.0 * t - v0[i];
    }
    __syncwarp();
    if (lane == 0) mu[j + 1] = v2[0] / a.h3;
    double *tt = v0;
    v0 = v1;
    v1 = v2;
    v2 = tt;
    __syncwarp();
  }
}

// FORM: 0 FP64, 1 FP32-mixed, 2 Lanczos quadrature.  MAXT bounds the block,
// which sets the register budget per thread.
template <int PM, int FORM, int MAXT, int RY>
__global__ void __launch_bounds__(MAXT, 1) sweep_kernel(SweepArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  Shared &S = *reinterpret_cast<Shared *>(smem);
  unsigned char *dyn = smem + shared_fixed();
  double *pcur =
      reinterpret_cast<double *>(dyn + planes_bytes(a.n, RY) + ring_bytes(a.nsweep, PM, RY) + accw_bytes(a.nsweep, PM, RY));
  for (int i = threadIdx.x; i < a.n_gproj + PM; i += blockDim.x) pcur[i] = 0.0;  // [n_gproj..]: the empty id
  pbar_setup(S);
  for (;;) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(a.counter, 1);
      S.qidx = q;
      S.node = q < a.n_list ? a.node_list[q] : -1;
      if (S.node >= 0) {
        S.gi = S.node % a.np[0];
        S.gj = (S.node / a.np[0]) % a.np[1];
        S.gk = S.node / (a.np[0] * a.np[1]);
      }
    }
    __syncthreads();
    const int node = S.node;
    if (node < 0) break;
    setup_node(a, S);
    double lmin = 0.0, lmax = 0.0;
    int rows = 0;
    double *mu = a.rho_pj + (size_t)node * (a.npl + 1);
    if constexpr (FORM == 2) {
      lanczos<double, PM, true, RY>(a, S, dyn, pcur, lmin, lmax, rows);
      const double chi = 0.5 * (lmax + lmin), zee = 0.5 * (lmax - lmin);
      if ((long long)rows <= (long long)a.n * a.n * a.n) quadrature_moments(a, S, rows, chi, zee, mu);
      else if (threadIdx.x == 0) atomicOr(a.status, ST_CAPACITY);
      count_proj_points(a, S, rows, 0);
      rows -= 1;  // reported as Lanczos iterations: matvecs = iterations + 1
    } else {
      using TL = typename std::conditional<FORM == 1, float, double>::type;
      lanczos<TL, PM, false, RY>(a, S, dyn, pcur, lmin, lmax, rows);
      const double chi = (lmax + lmin) / 2, zee = (lmax - lmin) / 2;  // sq.cpp:564-565
      count_proj_points(a, S, rows + 1, 0);
      // moments stay FP64 in both forms: FP32 storage of the Chebyshev vectors
      // grows a rounding error injected at step i like (k - i) by step k
      moments<PM, RY>(a, S, dyn, pcur, chi, zee, mu);
      count_proj_points(a, S, a.npl / 2, 1);
    }
    if (threadIdx.x == 0) {
      a.chi[node] = (lmax + lmin) / 2;
      a.zee[node] = (lmax - lmin) / 2;
      if (a.lmin) a.lmin[node] = lmin;
      if (a.lmax) a.lmax[node] = lmax;
      if (a.lanczos_iters) a.lanczos_iters[node] = rows;
    }
    __syncthreads();
  }
}

}  // namespace sweep
}  // namespace sqb
