#pragma once
// Node kernel: the per-grid-node work of the SQ step on sm_100a (device code,
// included by the translation units that instantiate its kernel groups).
//
// One persistent CTA works through a queue of grid nodes.  For each node it
// runs, on the node's (2nloc+1)^3 truncation window:
//   * the Lanczos spectral bounds of the sub-Hamiltonian (LanczosAlgorithm,
//     sq.cpp:965-1092; start vector of ones, sq.cpp:538-546);
//   * the Chebyshev moment recursion with the doubling identities
//     (sq.cpp:564-655), or, in force mode, the full npl-step recursion of the
//     density-matrix column and its nonlocal force contraction
//     (ForcesNonLocal, forces.cpp:318-578).
// Every matvec is H v = -1/2 Lap_h v + Veff v + Vnl v with v zero outside the
// window (HsubTimesVec, sq.cpp:838-929; VnlocsubTimesVec, nonlocal.cpp:20-215).
//
// Data movement.  A window vector lives in a per-CTA slot of global scratch
// (L2-resident for the CTAs in flight) and is streamed plane by plane along z:
// each thread owns one (x, y) column and keeps the 13 z-values its stencil
// needs in registers; the current z-plane is staged in shared memory inside a
// zero halo of 6 so the x and y neighbours are unconditional loads.  The
// nonlocal term is fused into the same plane sweep: bit masks of the
// projector boxes covering the warp's rows and crossing the plane drive the
// gather of sum_J c_J chi_J, and the dot products chi_J . v_new that the next matvec
// needs are accumulated from the freshly written plane by warp-owned atoms.
// The projector tables are stored with every z-plane of a ball padded to a
// multiple of four values, so the plane a box needs at a given z is one
// aligned contiguous block: it is copied into a three-stage ring in shared
// memory by one bulk asynchronous copy (cp.async.bulk, completion counted on
// the stage's mbarrier) issued one plane ahead, and the gather and the dot
// products read shared memory.  A plane that does not fit its stage is read
// from global memory instead.  The gather loops over the boxes covering the
// warp's rows (the same list for every lane), each lane testing its column.
#include <cmath>
#include <cstdio>
#include <type_traits>

#include "sqb_internal.cuh"

namespace sqb {

// Shared-memory limit per block of the current device (opt-in), set by
// node_kernel_setup.
extern int g_smem_optin;

enum : int { KIND_SQ = 0, KIND_FORCES = 1, KIND_VJP = 2, KIND_SQ32 = 3, KIND_LQ = 4 };

namespace {

enum PassKind : int {
  PK_ONES,   // v = 1 everywhere; projector dots of v
  PK_DELTA,  // v = e_centre; projector dots of v
  PK_DOTS,   // projector dots of an input vector (no output)
  PK_HV,     // out = H v, acc0 = <v, H v>                         (Lanczos step, sq.cpp:1029-1031)
  PK_LZB,    // w = o - a v_k - b v_k-1, acc0 = <w, w>; dots       (sq.cpp:1032-1043)
  PK_CH1,    // t1 = (H t0 - chi t0)/zee; dots; centre             (sq.cpp:579-591)
  PK_CH,     // t2 = 2(H t1 - chi t1)/zee - t0 in place of t0      (sq.cpp:603-616, 630-650)
  PK_FD01,   // D = t0 c0/h3 + t1 c1/h3                            (forces.cpp:414-441)
  PK_FD,     // PK_CH and D += t2 c_nq / h3                        (forces.cpp:443-456)
  PK_APPLY,  // out = H v                                          (HsubTimesVec)
  PK_ADJ,    // reverse Chebyshev (Clenshaw) step: out = 2(H a1 - chi a1)/zee
             // - s1 a2 + cd e_centre; dacc += ce a1 t (a1 = vin, a2 = p1, t = p2)
  PK_LZF,    // one Lanczos step in one sweep: the input W is formed on the
             // fly from the stored vectors, W = s1 (Y - ca W1) - cb W2 (or
             // the constant sin), written to wout; out = H W; acc0 = <W, W>,
             // acc1 = <W, H W>; dots of H W
};

struct NodeShared {
  unsigned long long mbar[4];  // per-stage mbarriers of the slice ring
  int node, qidx, gi, gj, gk;
  int n_ent, n_pi, stop, count;
  int ph;       // parity bits of the stage mbarriers
  int stalled;  // a stage wait ran out
  double center_val;
  double scal[4];
  double red[32][3];
  double aa[MAXL];
  double bb[MAXL];
  double eig[2];
  short e_x0[MAXE], e_x1[MAXE], e_y0[MAXE], e_y1[MAXE], e_z0[MAXE], e_z1[MAXE];
  short e_tx0[MAXE], e_ty0[MAXE], e_tz0[MAXE];  // table coordinates of the window origin
  int e_S[MAXE], e_sp2[MAXE], e_pb[MAXE], e_np[MAXE], e_nb[MAXE], e_atom[MAXE], e_type[MAXE];
  int e_ss[MAXE], e_sc[MAXE];  // staged part of a table plane: first value (multiple of 4) and count
  long long e_tab[MAXE];
  int4 e_geo[MAXE];  // packed: box x0,x1,y0,y1 | tx0,ty0 | Sd,np,pb | staged first value, count
  int scan[33];
  uint32_t rowmask[MAXN][4];  // boxes whose y range holds window row y
  uint32_t zmask[MAXN][4];    // boxes crossing window plane z
  int plane_tot[MAXN];        // staged values of plane z
  int ncross[MAXN];           // boxes crossing plane z
  int nitem[32];              // row layout: items of each warp
  uint32_t resid[32][4];      // row layout: boxes of each warp beyond its item list
  double p_cur[MAXP];
  double p_nxt[MAXP];
  double p_den[MAXP];
  double pw_cur[MAXP];   // Lanczos: chi^T W_m
  double pw_prev[MAXP];  // Lanczos: chi^T W_m-1
};

constexpr size_t kSharedFixed = (sizeof(NodeShared) + 127) & ~size_t(127);

template <typename T>
struct PassIO {
  const T *vin = nullptr;  // stencil input (or the pointwise main input)
  double sin = 1.0;        // lazy scale of vin (Lanczos normalisation)
  T *out = nullptr;        // output plane values
  const T *p1 = nullptr;   // pointwise input 1
  double s1 = 1.0;
  const T *p2 = nullptr;   // pointwise input 2
  double s2 = 1.0;
  double *dacc = nullptr;  // FP64 accumulator vector (density-matrix column)
  const double *din = nullptr;  // FP64 input (PK_DOTS / PK_APPLY from the caller)
  double *dout = nullptr;       // FP64 output (PK_APPLY)
  double ca = 0.0, cb = 0.0;    // a, b (PK_LZB) or chi, zee (Chebyshev)
  double cd = 0.0, ce = 0.0;    // D coefficients (forces)
  int dbl = 0;                  // accumulate the doubling dot products
  T *wout = nullptr;            // PK_LZF: where the formed input is stored
  int konst = 0;                // PK_LZF: the input is sin times the start vector
  double chk = 0.0;             // start vector 1 + chk (-1)^(x+y+z) (PK_ONES, PK_LZF konst)
  double *pg = nullptr;         // adjoint with atom gradients: dots with dchi/dR_alpha, [3][MAXP]
  const double *dtab = nullptr; // dchi/dR tables (3 x stride values)
  long long dstride = 0;
};


__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// mbarrier and bulk-copy primitives (PTX, sm_90 and later).
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// One contiguous global -> shared copy; both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Per-plane slice offsets (elements into the plane's stage): a box that does
// not cross the plane, and one that crosses it but did not fit the stage.
constexpr short OFF_NONE = -1;
constexpr short OFF_GLOBAL = -2;
constexpr int NSTAGE = 3;
// Time after which a stage wait is given up.  Copies of in-bounds data always
// complete (in microseconds), so reaching it means the hardware stopped
// making progress; the kernel then flags the stall and stops waiting.
constexpr unsigned long long WAIT_NS = 2000000000ull;
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Dynamic shared memory after NodeShared: two halo'd input planes and two
// output planes (sized for FP64; the row layout uses fixed pitches), the
// offset table [n][MAXE], the crossing lists [n][MAXE], the row layout's item
// lists, then NSTAGE slice stages of a.stage_bytes each.  `row` is the
// layout of the launch (NodeArgs::row_layout).
constexpr int ITEMS = 48;  // row layout: boxes listed per warp
__host__ __device__ __forceinline__ size_t planes_bytes(int n, int row) {
  const int P = n + 2 * FDN;
  const size_t v = row ? (size_t)(2 * (32 + 2 * FDN) * (32 + 2 * FDN) + 2 * 32 * 32) : (size_t)(2 * P * P + 2 * n * n);
  return (sizeof(double) * v + 15) & ~size_t(15);
}
__host__ __device__ __forceinline__ size_t offs_bytes(int n) { return (sizeof(short) * (size_t)n * MAXE + 15) & ~size_t(15); }
__host__ __device__ __forceinline__ size_t cross_bytes(int n) { return ((size_t)n * MAXE + 15) & ~size_t(15); }
__host__ __device__ __forceinline__ size_t offtab_bytes(int n, int row) {
  return offs_bytes(n) + cross_bytes(n) + (row ? sizeof(int4) * 16 * ITEMS : 0);
}
__device__ __forceinline__ short *off_table(const NodeArgs &a, unsigned char *dyn) {
  return reinterpret_cast<short *>(dyn + planes_bytes(a.n, a.row_layout));
}
// Boxes crossing plane z, in box order: cross_list(a, dyn)[z * MAXE + k], k < S.ncross[z].
__device__ __forceinline__ unsigned char *cross_list(const NodeArgs &a, unsigned char *dyn) {
  return dyn + planes_bytes(a.n, a.row_layout) + offs_bytes(a.n);
}
// Row layout item lists: row_items(a, dyn)[warp * ITEMS + i], i < S.nitem[warp].  An item is
//   x: box | z0 << 8 | z1 << 16 | nproj << 24
//   y: lane mask of the box's x range
//   z: (stage index of (x = 0, first row of the warp)) & 0xffff | Sd << 16 | row flags << 24
//   w: projector base | staged values per projector << 16
__device__ __forceinline__ int4 *row_items(const NodeArgs &a, unsigned char *dyn) {
  return reinterpret_cast<int4 *>(dyn + planes_bytes(a.n, a.row_layout) + offs_bytes(a.n) + cross_bytes(a.n));
}
template <typename T>
__device__ __forceinline__ T *stage_ptr(const NodeArgs &a, unsigned char *dyn, int k) {
  return reinterpret_cast<T *>(dyn + planes_bytes(a.n, a.row_layout) + offtab_bytes(a.n, a.row_layout) +
                               (size_t)k * a.stage_bytes);
}

// Lanes of a warp laid over a box cross-section row-wise: W lanes per row
// segment, R rows per warp step.
struct RowLanes {
  int W, R, lr, lx;
  __device__ __forceinline__ RowLanes(int bx, int lane) {
    W = bx < 32 ? bx : 32;
    R = 32 / W;
    lr = lane / W;
    lx = lane - lr * W;
  }
};

// Announce (one thread) the bytes plane zz's copies will bring into stage st.
// (not after a stall: the stage's barrier phase never completed, and a second
// arrival would overrun its count)
__device__ __forceinline__ void arm_plane(const NodeArgs &a, NodeShared &S, int zz, int st, size_t elem) {
  if (S.stalled) return;
  mbar_arrive_expect_tx(&S.mbar[st], (unsigned)(S.plane_tot[zz] * elem) + a.test_extra_tx);
}

// Issue the bulk copies of plane zz's table planes into stage st, spread
// over the warps: the k-th box crossing the plane goes to warp k % nw.
__device__ void issue_plane(const NodeArgs &a, NodeShared &S, unsigned char *dyn, int zz, int st) {
  if (S.stalled) return;  // no copies after a stall
  const int nw = blockDim.x >> 5;
  const int k = (threadIdx.x & 31) * nw + (threadIdx.x >> 5);
  if (k >= S.ncross[zz]) return;
  const int e = cross_list(a, dyn)[zz * MAXE + k];
  const int off = off_table(a, dyn)[zz * MAXE + e];
  if (off < 0) return;
  double *stage = stage_ptr<double>(a, dyn, st);
  const double *tab = a.at.tab64;
  const int Sd = S.e_S[e], sp2 = S.e_sp2[e], cnt = S.e_sc[e];
  const double *src = tab + S.e_tab[e] + (long long)(S.e_tz0[e] + zz) * sp2 + S.e_ss[e];
  // No proxy fence: every generic-proxy read of this stage (plane zz-3) was
  // consumed before the barrier that precedes this call.
  for (int q = 0; q < S.e_np[e]; q++)
    bulk_g2s(stage + off + q * cnt, src + (long long)q * Sd * sp2, (unsigned)(cnt * sizeof(double)), &S.mbar[st]);
}

// Wait for the copies of a stage (every thread); a wait that runs out of time
// (a.wait_ns, default WAIT_NS) gives the copies already issued a further
// GRACE_NS to land (in-bounds copies take microseconds), then sets the stall
// flag and the status bit, after which no copies are issued, no stage is armed
// or waited for, and the CTA leaves its node loop after the current node.
constexpr unsigned long long GRACE_NS = 1000000ull;
__device__ __forceinline__ void stage_wait(const NodeArgs &a, NodeShared &S, int st, int &ph) {
  if (!S.stalled) {
    const unsigned parity = (ph >> st) & 1;
    const unsigned long long limit = a.wait_ns ? a.wait_ns : WAIT_NS;
    bool done = mbar_try_wait(&S.mbar[st], parity);
    if (!done) {
      const unsigned long long t0 = global_ns();
      while (!(done = mbar_try_wait(&S.mbar[st], parity)))
        if (global_ns() - t0 > limit) break;
    }
    if (!done) {
      const unsigned long long t1 = global_ns();
      while (global_ns() - t1 < GRACE_NS) {
      }
      S.stalled = 1;
      atomicOr(a.status, ST_WAIT_LIMIT);
    }
  }
  ph ^= 1 << st;
}

// Slice offsets of every plane for this node's boxes, packed in box order.
__device__ void plane_offsets(const NodeArgs &a, NodeShared &S, short *off_tab, unsigned char *cross) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int cap = (int)(a.stage_bytes / sizeof(double));
  for (int zz = warp; zz < a.n; zz += nw) {
    int run = 0, nc = 0, tot = 0;
    for (int base = 0; base < S.n_ent; base += 32) {
      const int e = base + lane;
      bool crosses = false;
      int sz = 0;
      if (e < S.n_ent) {
        crosses = S.e_z0[e] <= zz && zz <= S.e_z1[e];
        if (crosses) sz = S.e_np[e] * S.e_sc[e];
      }
      int incl = sz;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      // staged boxes are packed in box order until the stage is full
      const int start = run + incl - sz;
      const bool fits = crosses && start + sz <= cap;
      if (e < S.n_ent) off_tab[zz * MAXE + e] = !crosses ? OFF_NONE : (fits ? (short)start : OFF_GLOBAL);
      tot += __reduce_add_sync(0xffffffffu, fits ? sz : 0);
      run += __shfl_sync(0xffffffffu, incl, 31);
      const unsigned cb = __ballot_sync(0xffffffffu, crosses);
      if (crosses) cross[zz * MAXE + nc + __popc(cb & ((1u << lane) - 1u))] = (unsigned char)e;
      nc += __popc(cb);
    }
    if (lane == 0) {
      S.plane_tot[zz] = tot;
      S.ncross[zz] = nc;
    }
  }
}

// Deterministic block sum of up to three values into S.scal[0..2].
__device__ void block_sum3(NodeShared &S, double v0, double v1, double v2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v0 = warp_sum(v0);
  v1 = warp_sum(v1);
  v2 = warp_sum(v2);
  if (lane == 0) {
    S.red[warp][0] = v0;
    S.red[warp][1] = v1;
    S.red[warp][2] = v2;
  }
  __syncthreads();
  if (warp == 0) {
    double r0 = lane < nw ? S.red[lane][0] : 0.0;
    double r1 = lane < nw ? S.red[lane][1] : 0.0;
    double r2 = lane < nw ? S.red[lane][2] : 0.0;
    r0 = warp_sum(r0);
    r1 = warp_sum(r1);
    r2 = warp_sum(r2);
    if (lane == 0) {
      S.scal[0] = r0;
      S.scal[1] = r1;
      S.scal[2] = r2;
    }
  }
  __syncthreads();
}

// Accumulate chi_J,q . plane into p_nxt for every projector box crossing
// plane zz (the k-th crossing box goes to warp k % nw); the table planes come
// from the plane's stage, or from global memory for a box that was not staged.
template <typename T>
__device__ __forceinline__ double box_dot(const T *pl, int pitch, const double *U, int Sd, int bx, int by, int lane) {
  double acc = 0.0;
  if (bx <= 16) {  // two rows per step: lanes 0-15 and 16-31
    const int lr = lane >> 4, lx = lane & 15;
    if (lx < bx) {
      const T *p = pl + lr * pitch + lx;
      const double *u = U + lr * Sd + lx;
      for (int y = lr; y < by; y += 2, p += 2 * pitch, u += 2 * Sd) acc += (double)*p * *u;
    }
  } else {
    const RowLanes L(bx, lane);
    if (L.lr < L.R) {
      for (int y = L.lr; y < by; y += L.R)
        for (int x = L.lx; x < bx; x += L.W) acc += (double)pl[y * pitch + x] * U[y * Sd + x];
    }
  }
  return acc;
}

template <typename T>
__device__ __forceinline__ double box_dot_d(const T *pl, int pitch, const double *U, int Sd, int bx, int by, int lane) {
  double acc = 0.0;
  const RowLanes L(bx, lane);
  if (L.lr < L.R) {
    for (int y = L.lr; y < by; y += L.R)
      for (int x = L.lx; x < bx; x += L.W) acc += (double)pl[y * pitch + x] * U[y * Sd + x];
  }
  return acc;
}

// pg != nullptr (adjoint with atom gradients): also the dot products with the
// derivative tables dchi/dR_alpha of every crossing box, added to pg[alpha][p]
// (read from global memory: this runs only in the adjoint kernel group).
template <typename T>
__device__ void dot_phase(NodeShared &S, const T *plane, int zz, int pitch, const double *tab, const short *offz,
                          const unsigned char *crossz, const double *stage, double *pg = nullptr,
                          const double *dtab = nullptr, long long dstride = 0) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = warp; k < S.ncross[zz]; k += nw) {
    const int e = crossz[k];
    const int off = offz[e];
    const int4 g = S.e_geo[e];
    const int x0 = g.x & 0xff, x1 = (g.x >> 8) & 0xff, y0 = (g.x >> 16) & 0xff, y1 = (g.x >> 24) & 0xff;
    const int tx0 = (short)(g.y & 0xffff), ty0 = g.y >> 16;
    const int Sd = g.z & 0xff, np = (g.z >> 8) & 0xff, pb = g.z >> 16, ss = g.w & 0xffff, cnt = g.w >> 16;
    const int bx = x1 - x0 + 1, by = y1 - y0 + 1;
    const int r0 = (ty0 + y0) * Sd + tx0 + x0;  // table index of the box corner
    const T *pl = plane + y0 * pitch + x0;
    for (int q = 0; q < np; q++) {
      double acc;
      if (off >= 0) {  // shared-memory stage (kept a separate pointer: shared loads)
        acc = box_dot<T>(pl, pitch, stage + off + q * cnt + r0 - ss, Sd, bx, by, lane);
      } else {
        const int sp2 = S.e_sp2[e];
        acc = box_dot<T>(pl, pitch, tab + S.e_tab[e] + (long long)(q * Sd + S.e_tz0[e] + zz) * sp2 + r0, Sd, bx, by,
                         lane);
      }
      acc = warp_sum(acc);
      if (lane == 0) S.p_nxt[pb + q] += acc;
      if (pg) {
        const double *Ud = dtab + S.e_tab[e] + (long long)(q * Sd + S.e_tz0[e] + zz) * S.e_sp2[e] + r0;
#pragma unroll
        for (int al = 0; al < 3; al++) {
          double ad = box_dot_d<T>(pl, pitch, Ud + al * dstride, Sd, bx, by, lane);
          ad = warp_sum(ad);
          if (lane == 0) pg[al * MAXP + pb + q] += ad;
        }
      }
    }
  }
}

// After a pass that accumulated projector dots: c_J,q = scale * dot / Denom.
__device__ void rotate_proj(NodeShared &S, double scale) {
  for (int p = threadIdx.x; p < S.n_pi; p += blockDim.x) {
    S.p_cur[p] = scale * S.p_nxt[p] / S.p_den[p];
    S.p_nxt[p] = 0.0;
  }
  __syncthreads();
}

// PK_LZF input at window index g from its loaded operands y = Y[g],
// w1 = W1[g], w2 = W2[g]: the next (unnormalised) Lanczos vector
// W = s1 (Y - ca W1) - cb W2, i.e. u - a v_k - b v_k-1 with u = s1 Y,
// v_k = s1 W1, v_k-1 = s2 W2 and cb = b s2 (LanczosAlgorithm, sq.cpp:1032-1036);
// stored in wout, in place of W2.  The operands are loaded one plane before
// they are combined, so the loads' latency overlaps a plane of work.
// Lanczos start vector at window index g: 1 + chk (-1)^(x+y+z); the window
// edge n is odd, so x + y + z and g = (z n + y) n + x have the same parity.
__device__ __forceinline__ double start_val(double chk, size_t g) { return 1.0 + chk * (1.0 - 2.0 * (double)(g & 1)); }

template <typename T>
__device__ __forceinline__ T form_w(const PassIO<T> &io, size_t g, T y, T w1, T w2) {
  const T f = io.konst ? (T)(io.sin * start_val(io.chk, g))
                       : (T)(io.s1 * ((double)y - io.ca * (double)w1) - io.cb * (double)w2);
  io.wout[g] = f;
  return f;
}

// One sweep over the window's z-planes.
template <typename T, int C, int PK>
__device__ void pass(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const PassIO<T> &io,
                     const uint32_t (&wmask)[4], double &acc0, double &acc1) {
  constexpr bool STENCIL = (PK == PK_HV || PK == PK_CH1 || PK == PK_CH || PK == PK_FD || PK == PK_APPLY ||
                           PK == PK_LZF || PK == PK_ADJ);
  constexpr bool DOTS = (PK == PK_ONES || PK == PK_DELTA || PK == PK_DOTS || PK == PK_LZB || PK == PK_CH1 ||
                         PK == PK_CH || PK == PK_FD || PK == PK_LZF || PK == PK_ADJ);
  const int n = a.n, n2 = n * n, P = n + 2 * FDN, P2 = P * P;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int centre_col = a.nloc * n + a.nloc;
  T *sm_in = reinterpret_cast<T *>(dyn);
  T *sm_out = sm_in + 2 * P2;
  const double *veff = a.veff64;  // Veff and projector tables stay FP64 in both paths
  const double *tab = a.at.tab64;
  const size_t vplane = (size_t)a.ex * a.ey;
  const short *off_tab = off_table(a, dyn);
  const bool staged = (STENCIL || DOTS) && S.n_ent > 0;

  if (STENCIL) {
    for (int i = tid; i < 2 * P2; i += nt) sm_in[i] = T(0);
  }
  if (staged && tid == 0) arm_plane(a, S, 0, 0, sizeof(double));
  __syncthreads();
  int ph = S.ph;
  if (staged) issue_plane(a, S, dyn, 0, 0);

  int col[C], cx[C], cy[C];
  bool ok[C];
  size_t vb[C];
#pragma unroll
  for (int c = 0; c < C; c++) {
    col[c] = tid + c * nt;
    ok[c] = col[c] < n2;
    cx[c] = ok[c] ? col[c] % n : 0;
    cy[c] = ok[c] ? col[c] / n : 0;
    vb[c] = ((size_t)(S.gk) * a.ey + (S.gj + cy[c])) * a.ex + (S.gi + cx[c]);
  }
  const T sin = (T)io.sin;
  auto ld_in = [&](int c, int z) -> T {
    if (!ok[c] || z >= n) return T(0);
    if constexpr (PK == PK_DOTS || PK == PK_APPLY) return (T)io.din[(size_t)z * n2 + col[c]];
    else return io.vin[(size_t)z * n2 + col[c]] * sin;
  };

  T win[C][2 * FDN + 1];
  T pf[C];
  T rw1[C], rw2[C];  // PK_LZF: W1, W2 of the prefetched plane (pf holds its Y)
  auto lzf_load = [&](int c, int z) {
    if (ok[c] && z < n && !io.konst) {
      const size_t g = (size_t)z * n2 + col[c];
      pf[c] = io.vin[g];
      rw1[c] = io.p1[g];
      rw2[c] = io.p2[g];
    }
  };
  auto lzf_form = [&](int c, int z) -> T {
    if (!ok[c] || z >= n) return T(0);
    return form_w<T>(io, (size_t)z * n2 + col[c], pf[c], rw1[c], rw2[c]);
  };
  T q_p1[C], q_p2[C];
  double q_ve[C];
  double q_d[C];
  auto ld_point = [&](int c, int z) {
    if (!ok[c] || z >= n) return;
    const size_t g = (size_t)z * n2 + col[c];
    if constexpr (STENCIL) q_ve[c] = veff[vb[c] + (size_t)z * vplane];
    if constexpr (PK == PK_LZB || PK == PK_CH || PK == PK_FD || PK == PK_FD01 || PK == PK_ADJ)
      q_p1[c] = io.p1[g] * (T)io.s1;
    if constexpr (PK == PK_LZB || PK == PK_FD01 || PK == PK_ADJ) q_p2[c] = io.p2[g] * (T)io.s2;
    if constexpr (PK == PK_LZB || PK == PK_DOTS) pf[c] = ld_in(c, z);
    if constexpr (PK == PK_FD || PK == PK_ADJ) q_d[c] = io.dacc[g];
  };
#pragma unroll
  for (int c = 0; c < C; c++) {
    if constexpr (PK == PK_LZF) {
      // planes 0..FDN enter the window: their operands are loaded four planes
      // at a time before any is combined (the stores of W would otherwise
      // order every load after the previous plane's store)
#pragma unroll
      for (int s = 0; s < FDN; s++) win[c][s] = T(0);
#pragma unroll
      for (int z0 = 0; z0 <= FDN; z0 += 4) {
        T ty[4], t1[4], t2[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int z = z0 + q;
          ty[q] = t1[q] = t2[q] = T(0);
          if (z <= FDN && ok[c] && z < n && !io.konst) {
            const size_t g = (size_t)z * n2 + col[c];
            ty[q] = io.vin[g];
            t1[q] = io.p1[g];
            t2[q] = io.p2[g];
          }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int z = z0 + q;
          if (z <= FDN)
            win[c][FDN + z] = (ok[c] && z < n) ? form_w<T>(io, (size_t)z * n2 + col[c], ty[q], t1[q], t2[q]) : T(0);
        }
      }
      lzf_load(c, FDN + 1);
    } else if constexpr (STENCIL) {
#pragma unroll
      for (int s = 0; s <= 2 * FDN; s++) win[c][s] = s < FDN ? T(0) : ld_in(c, s - FDN);
      pf[c] = ld_in(c, FDN + 1);
    }
    ld_point(c, 0);
  }

  // Arithmetic is FP64 for both storage types: with FP32 storage (mixed
  // path) the six neighbour pairs of each stencil arm are summed in FP32 and
  // everything after that -- the 7-term stencil sum, Veff, the nonlocal
  // gather and the recursion update -- in FP64, so the rounding left is the
  // FP32 storage of the vectors.
  const double chi = io.ca, zee = io.cb;

  // Stage ring: plane z in stage st, plane z-1 (dot phase) in the previous
  // one; warp 0 issues the copies for plane z+1 into the third after the
  // barrier that ends every read of plane z-2.
  int st = 0;
  for (int z = 0; z <= n; z++) {
    T *smz = sm_in + (z & 1) * P2;
    T *smo = sm_out + (z & 1) * n2;
    if (STENCIL && z < n) {
#pragma unroll
      for (int c = 0; c < C; c++)
        if (ok[c]) smz[(cy[c] + FDN) * P + cx[c] + FDN] = win[c][FDN];
    }
    const int st_next = st == NSTAGE - 1 ? 0 : st + 1, st_prev = st == 0 ? NSTAGE - 1 : st - 1;
    if (staged && z < n) stage_wait(a, S, st, ph);
    if (staged && tid == 0 && z + 1 < n) arm_plane(a, S, z + 1, st_next, sizeof(double));
    __syncthreads();
    if (DOTS && z >= 1 && S.n_ent > 0)
      dot_phase<T>(S, sm_out + ((z - 1) & 1) * n2, z - 1, n, tab, off_tab + (z - 1) * MAXE,
                   cross_list(a, dyn) + (z - 1) * MAXE, stage_ptr<double>(a, dyn, st_prev), io.pg, io.dtab, io.dstride);
    if (staged && z + 1 < n) issue_plane(a, S, dyn, z + 1, st_next);
    if (z == n) break;
    // Nonlocal gather: the boxes covering this warp's rows and crossing plane
    // z, the same list for every lane; each lane adds the boxes that cover
    // its column.
    double vnl[C];
#pragma unroll
    for (int c = 0; c < C; c++) vnl[c] = 0.0;
    if (STENCIL && S.n_ent > 0) {
      const short *offz = off_tab + z * MAXE;
      const double *stg = stage_ptr<double>(a, dyn, st);
#pragma unroll
      for (int w = 0; w < 4; w++) {
        uint32_t m = wmask[w] & S.zmask[z][w];
        while (m) {
          const int e = w * 32 + __ffs(m) - 1;
          m &= m - 1;
          const int off = offz[e];
          const int4 g = S.e_geo[e];
          const int x0 = g.x & 0xff, x1 = (g.x >> 8) & 0xff, y0 = (g.x >> 16) & 0xff, y1 = (g.x >> 24) & 0xff;
          const int tx0 = (short)(g.y & 0xffff), ty0 = g.y >> 16;
          const int Sd = g.z & 0xff, np = (g.z >> 8) & 0xff, pb = g.z >> 16, ss = g.w & 0xffff, cnt = g.w >> 16;
          if (off >= 0) {  // shared-memory stage: its own pointer, so the loads stay shared loads
            const double *base = stg + off - ss;
#pragma unroll
            for (int c = 0; c < C; c++) {
              if (!ok[c] || cx[c] < x0 || cx[c] > x1 || cy[c] < y0 || cy[c] > y1) continue;
              const double *u = base + (ty0 + cy[c]) * Sd + tx0 + cx[c];
              for (int q = 0; q < np; q++) vnl[c] += S.p_cur[pb + q] * u[q * cnt];
            }
          } else {
            const int sp2 = S.e_sp2[e];
            const double *base = tab + S.e_tab[e] + (long long)(S.e_tz0[e] + z) * sp2;
#pragma unroll
            for (int c = 0; c < C; c++) {
              if (!ok[c] || cx[c] < x0 || cx[c] > x1 || cy[c] < y0 || cy[c] > y1) continue;
              const double *u = base + (ty0 + cy[c]) * Sd + tx0 + cx[c];
              for (int q = 0; q < np; q++) vnl[c] += S.p_cur[pb + q] * u[(long long)q * Sd * sp2];
            }
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < C; c++) {
      if (!ok[c]) continue;
      const size_t g = (size_t)z * n2 + col[c];
      double hv = 0.0, v = 0.0;
      if constexpr (STENCIL) {
        v = (double)win[c][FDN];
        const int idx = (cy[c] + FDN) * P + cx[c] + FDN;
        double temp = v * 3.0 * a.coeff_lap[0];
#pragma unroll
        for (int k = 1; k <= FDN; k++) {
          T s = smz[idx - k] + smz[idx + k] + smz[idx - k * P] + smz[idx + k * P] + win[c][FDN - k] + win[c][FDN + k];
          temp += (double)s * a.coeff_lap[k];
        }
        hv = -0.5 * temp + q_ve[c] * v + vnl[c];
      }
      T o = T(0);
      if constexpr (PK == PK_ONES) {
        o = (T)start_val(io.chk, g);
        io.out[g] = o;
      } else if constexpr (PK == PK_DELTA) {
        o = (col[c] == centre_col && z == a.nloc) ? T(1) : T(0);
        io.out[g] = o;
      } else if constexpr (PK == PK_DOTS) {
        o = pf[c];
      } else if constexpr (PK == PK_HV) {
        o = (T)hv;
        io.out[g] = o;
        acc0 += v * hv;
      } else if constexpr (PK == PK_LZB) {
        o = q_p1[c] - (T)io.ca * pf[c] - (T)io.cb * q_p2[c];
        io.out[g] = o;
        acc0 += (double)o * (double)o;
      } else if constexpr (PK == PK_CH1) {
        o = (T)((hv - chi * v) / zee);
        io.out[g] = o;
      } else if constexpr (PK == PK_CH || PK == PK_FD) {
        const double od = (2.0 * (hv - chi * v)) / zee - (double)q_p1[c];
        o = (T)od;
        io.out[g] = o;
        if (io.dbl) {
          acc0 += (double)o * (double)o;
          acc1 += (double)o * v;
        }
        if constexpr (PK == PK_FD) io.dacc[g] = q_d[c] + (double)o * io.cd / a.h3;
      } else if constexpr (PK == PK_FD01) {
        io.dacc[g] = 0.0 + (double)q_p1[c] * io.cd / a.h3 + (double)q_p2[c] * io.ce / a.h3;
      } else if constexpr (PK == PK_APPLY) {
        io.dout[g] = hv;
      } else if constexpr (PK == PK_LZF) {
        o = (T)hv;
        io.out[g] = o;
        acc0 += v * v;
        acc1 += v * hv;
      } else if constexpr (PK == PK_ADJ) {
        double od = (2.0 * (hv - chi * v)) / zee - (double)q_p1[c];
        if (col[c] == centre_col && z == a.nloc) od += io.cd;
        o = (T)od;
        io.out[g] = o;
        io.dacc[g] = q_d[c] + io.ce * v * (double)q_p2[c];
      }
      if constexpr (DOTS) smo[col[c]] = o;
      if (col[c] == centre_col && z == a.nloc) S.center_val = (double)o;
      if (!isfinite((double)o)) atomicOr(a.status, ST_NONFINITE);
    }
    // advance the register windows and prefetch the next plane's operands
#pragma unroll
    for (int c = 0; c < C; c++) {
      if constexpr (PK == PK_LZF) {
#pragma unroll
        for (int s = 0; s < 2 * FDN; s++) win[c][s] = win[c][s + 1];
        win[c][2 * FDN] = lzf_form(c, z + FDN + 1);
        lzf_load(c, z + FDN + 2);
      } else if constexpr (STENCIL) {
#pragma unroll
        for (int s = 0; s < 2 * FDN; s++) win[c][s] = win[c][s + 1];
        win[c][2 * FDN] = pf[c];
        pf[c] = ld_in(c, z + FDN + 2);
      }
      ld_point(c, z + 1);
    }
    st = st_next;
  }
  __syncthreads();
  if (tid == 0) S.ph = ph;
}

// Row layout of the plane loop, for windows up to 32 wide: warp w owns the
// RY adjacent rows y = RY*w + j, lane x owns column x.  The halo'd input
// plane has the compile-time pitch RP, so every stencil neighbour is an
// immediate offset from the lane's centre; with RY = 2 the two rows share
// the loads of their y arms.  The projector boxes covering the warp's rows
// are one list for all its lanes.
constexpr int RP = 32 + 2 * FDN;         // pitch of the input planes
constexpr int RPLANE = RP * RP;          // one input plane (rows 0..n+2FDN-1 used)
constexpr int OPLANE = 32 * 32;          // one output plane, pitch 32

template <typename T, int RY, int PK>
__device__ void pass_rows(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const PassIO<T> &io,
                          const uint32_t (&wmask)[4], double &acc0, double &acc1) {
  constexpr bool STENCIL = (PK == PK_HV || PK == PK_CH1 || PK == PK_CH || PK == PK_FD || PK == PK_APPLY ||
                           PK == PK_LZF || PK == PK_ADJ);
  constexpr bool DOTS = (PK == PK_ONES || PK == PK_DELTA || PK == PK_DOTS || PK == PK_LZB || PK == PK_CH1 ||
                         PK == PK_CH || PK == PK_FD || PK == PK_LZF || PK == PK_ADJ);
  constexpr bool P1 = (PK == PK_LZB || PK == PK_CH || PK == PK_FD || PK == PK_FD01 || PK == PK_ADJ);
  constexpr bool P2 = (PK == PK_LZB || PK == PK_FD01 || PK == PK_ADJ);
  constexpr bool PF = (PK == PK_LZB || PK == PK_DOTS);
  const int n = a.n, n2 = n * n;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int x = lane;
  T *sm_in = reinterpret_cast<T *>(dyn);
  T *sm_out = sm_in + 2 * RPLANE;
  const double *veff = a.veff64;  // Veff and projector tables stay FP64 in both paths
  const double *tab = a.at.tab64;
  const size_t vplane = (size_t)a.ex * a.ey;
  const short *off_tab = off_table(a, dyn);
  const bool staged = (STENCIL || DOTS) && S.n_ent > 0;

  if (STENCIL) {
    for (int i = tid; i < 2 * RPLANE; i += nt) sm_in[i] = T(0);
  }
  if (staged && tid == 0) arm_plane(a, S, 0, 0, sizeof(double));
  __syncthreads();
  int ph = S.ph;
  if (staged) issue_plane(a, S, dyn, 0, 0);

  int y[RY];
  bool ok[RY];
  size_t col[RY];    // y*n + x
  size_t vb[RY];     // Veff index of (x, y, 0)
#pragma unroll
  for (int j = 0; j < RY; j++) {
    y[j] = warp * RY + j;
    ok[j] = x < n && y[j] < n;
    col[j] = ok[j] ? (size_t)y[j] * n + x : 0;
    vb[j] = ((size_t)S.gk * a.ey + (S.gj + (ok[j] ? y[j] : 0))) * a.ex + (S.gi + (ok[j] ? x : 0));
  }
  const T sin = (T)io.sin;
  auto ld_in = [&](int j, int z) -> T {
    if (!ok[j] || z >= n) return T(0);
    if constexpr (PK == PK_DOTS || PK == PK_APPLY) return (T)io.din[(size_t)z * n2 + col[j]];
    else return io.vin[(size_t)z * n2 + col[j]] * sin;
  };
  T win[RY][2 * FDN + 1];
  T pf[RY], q_p1[RY], q_p2[RY];
  double q_ve[RY];
  T rw1[RY], rw2[RY];  // PK_LZF: W1, W2 of the prefetched plane (pf holds its Y)
  auto lzf_load = [&](int j, int z) {
    if (ok[j] && z < n && !io.konst) {
      const size_t g = (size_t)z * n2 + col[j];
      pf[j] = io.vin[g];
      rw1[j] = io.p1[g];
      rw2[j] = io.p2[g];
    }
  };
  auto lzf_form = [&](int j, int z) -> T {
    if (!ok[j] || z >= n) return T(0);
    return form_w<T>(io, (size_t)z * n2 + col[j], pf[j], rw1[j], rw2[j]);
  };
  double q_d[RY];
  auto ld_point = [&](int j, int z) {
    if (!ok[j] || z >= n) return;
    const size_t g = (size_t)z * n2 + col[j];
    if constexpr (STENCIL) q_ve[j] = veff[vb[j] + (size_t)z * vplane];
    if constexpr (P1) q_p1[j] = io.p1[g] * (T)io.s1;
    if constexpr (P2) q_p2[j] = io.p2[g] * (T)io.s2;
    if constexpr (PF) pf[j] = ld_in(j, z);
    if constexpr (PK == PK_FD || PK == PK_ADJ) q_d[j] = io.dacc[g];
  };
#pragma unroll
  for (int j = 0; j < RY; j++) {
    if constexpr (PK == PK_LZF) {
#pragma unroll
      for (int s = 0; s < FDN; s++) win[j][s] = T(0);
#pragma unroll
      for (int z0 = 0; z0 <= FDN; z0 += 4) {
        T ty[4], t1[4], t2[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int z = z0 + q;
          ty[q] = t1[q] = t2[q] = T(0);
          if (z <= FDN && ok[j] && z < n && !io.konst) {
            const size_t g = (size_t)z * n2 + col[j];
            ty[q] = io.vin[g];
            t1[q] = io.p1[g];
            t2[q] = io.p2[g];
          }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int z = z0 + q;
          if (z <= FDN)
            win[j][FDN + z] = (ok[j] && z < n) ? form_w<T>(io, (size_t)z * n2 + col[j], ty[q], t1[q], t2[q]) : T(0);
        }
      }
      lzf_load(j, FDN + 1);
    } else if constexpr (STENCIL) {
#pragma unroll
      for (int s = 0; s <= 2 * FDN; s++) win[j][s] = s < FDN ? T(0) : ld_in(j, s - FDN);
      pf[j] = ld_in(j, FDN + 1);
    }
    ld_point(j, 0);
  }
  const double chi = io.ca, zee = io.cb;
  const double c0 = 3.0 * a.coeff_lap[0];

  int st = 0;
  for (int z = 0; z <= n; z++) {
    T *smz = sm_in + (z & 1) * RPLANE;
    T *smo = sm_out + (z & 1) * OPLANE;
    if (STENCIL && z < n) {
#pragma unroll
      for (int j = 0; j < RY; j++)
        if (ok[j]) smz[(y[j] + FDN) * RP + x + FDN] = win[j][FDN];
    }
    const int st_next = st == NSTAGE - 1 ? 0 : st + 1, st_prev = st == 0 ? NSTAGE - 1 : st - 1;
    if (staged && z < n) stage_wait(a, S, st, ph);
    if (staged && tid == 0 && z + 1 < n) arm_plane(a, S, z + 1, st_next, sizeof(double));
    __syncthreads();
    if (DOTS && z >= 1 && S.n_ent > 0)
      dot_phase<T>(S, sm_out + ((z - 1) & 1) * OPLANE, z - 1, 32, tab, off_tab + (z - 1) * MAXE,
                   cross_list(a, dyn) + (z - 1) * MAXE, stage_ptr<double>(a, dyn, st_prev), io.pg, io.dtab, io.dstride);
    if (staged && z + 1 < n) issue_plane(a, S, dyn, z + 1, st_next);
    if (z == n) break;

    double vnl[RY];
#pragma unroll
    for (int j = 0; j < RY; j++) vnl[j] = 0.0;
    if (STENCIL && S.n_ent > 0) {
      const short *offz = off_tab + z * MAXE;
      const double *stg = stage_ptr<double>(a, dyn, st);
      if constexpr (RY == 2) {
        // the boxes of this warp's item list that cross plane z
        const int4 *it = row_items(a, dyn) + warp * ITEMS;
        const int ni = S.nitem[warp];
        for (int i = 0; i < ni; i++) {
          const int4 g = it[i];
          if (z < ((g.x >> 8) & 0xff) || z > ((g.x >> 16) & 0xff)) continue;
          if (!((g.y >> lane) & 1)) continue;
          const int e = g.x & 0xff, np = (g.x >> 24) & 0xff;
          const int rb = (short)(g.z & 0xffff) + x, Sd = (g.z >> 16) & 0xff, fl = (g.z >> 24) & 0xff;
          const int pb = g.w & 0xffff, cnt = g.w >> 16;
          const int off = offz[e];
          if (off >= 0) {  // shared-memory stage: its own pointer, so the loads stay shared loads
            const double *u = stg + off + rb;
            for (int q = 0; q < np; q++) {
              const double pc = S.p_cur[pb + q];
              if (fl & 1) vnl[0] += pc * (double)u[q * cnt];
              if (fl & 2) vnl[1] += pc * (double)u[q * cnt + Sd];
            }
          } else {
            const int sp2 = S.e_sp2[e];
            const double *u = tab + S.e_tab[e] + (long long)(S.e_tz0[e] + z) * sp2 + rb + S.e_ss[e];
            for (int q = 0; q < np; q++) {
              const double pc = S.p_cur[pb + q];
              if (fl & 1) vnl[0] += pc * (double)u[(long long)q * Sd * sp2];
              if (fl & 2) vnl[1] += pc * (double)u[(long long)q * Sd * sp2 + Sd];
            }
          }
        }
      }
      // boxes not in an item list (RY != 2, or a list that overflowed)
#pragma unroll
      for (int w = 0; w < 4; w++) {
        uint32_t m = (RY == 2 ? S.resid[warp][w] : wmask[w]) & S.zmask[z][w];
        while (m) {
          const int e = w * 32 + __ffs(m) - 1;
          m &= m - 1;
          const int off = offz[e];
          const int4 g = S.e_geo[e];
          const int x0 = g.x & 0xff, x1 = (g.x >> 8) & 0xff, y0 = (g.x >> 16) & 0xff, y1 = (g.x >> 24) & 0xff;
          if (x < x0 || x > x1) continue;
          const int tx0 = (short)(g.y & 0xffff), ty0 = g.y >> 16;
          const int Sd = g.z & 0xff, np = (g.z >> 8) & 0xff, pb = g.z >> 16, ss = g.w & 0xffff, cnt = g.w >> 16;
          if (off >= 0) {
            const double *base = stg + off - ss + tx0 + x;
#pragma unroll
            for (int j = 0; j < RY; j++) {
              if (!ok[j] || y[j] < y0 || y[j] > y1) continue;
              const double *u = base + (ty0 + y[j]) * Sd;
              for (int q = 0; q < np; q++) vnl[j] += S.p_cur[pb + q] * (double)u[q * cnt];
            }
          } else {
            const int sp2 = S.e_sp2[e];
            const double *base = tab + S.e_tab[e] + (long long)(S.e_tz0[e] + z) * sp2 + tx0 + x;
#pragma unroll
            for (int j = 0; j < RY; j++) {
              if (!ok[j] || y[j] < y0 || y[j] > y1) continue;
              const double *u = base + (ty0 + y[j]) * Sd;
              for (int q = 0; q < np; q++) vnl[j] += S.p_cur[pb + q] * (double)u[(long long)q * Sd * sp2];
            }
          }
        }
      }
    }

    double hvj[RY], vj[RY];
    if constexpr (STENCIL) {
      // Arm k of each point sums (x-k) + (x+k) + (y-k) + (y+k) + (z-k) + (z+k)
      // in that order before the coefficient, as HsubTimesVec does
      // (sq.cpp:894-897).
      const T *cc = smz + (y[0] + FDN) * RP + x + FDN;  // centre of row y[0]
      double temp[RY];
#pragma unroll
      for (int j = 0; j < RY; j++) temp[j] = (double)win[j][FDN] * c0;
      if constexpr (RY == 2) {
        // rows y0-k and y0+1+k are loaded once: row y0-k is point 0's minus
        // side at arm k and point 1's at arm k+1, row y0+1+k point 1's plus
        // side at arm k and point 0's at arm k+1.
        const T *c1 = cc + RP;
        T prev_m = win[0][FDN], prev_p = win[1][FDN];
#pragma unroll
        for (int k = 1; k <= FDN; k++) {
          const T ym = cc[-k * RP], yp = cc[(k + 1) * RP];
          const T s0 = cc[-k] + cc[k] + ym + prev_p + win[0][FDN - k] + win[0][FDN + k];
          const T s1 = c1[-k] + c1[k] + prev_m + yp + win[1][FDN - k] + win[1][FDN + k];
          temp[0] += (double)s0 * a.coeff_lap[k];
          temp[1] += (double)s1 * a.coeff_lap[k];
          prev_m = ym;
          prev_p = yp;
        }
      } else {
#pragma unroll
        for (int j = 0; j < RY; j++) {
          const T *cj = cc + j * RP;
#pragma unroll
          for (int k = 1; k <= FDN; k++) {
            const T sk = cj[-k] + cj[k] + cj[-k * RP] + cj[k * RP] + win[j][FDN - k] + win[j][FDN + k];
            temp[j] += (double)sk * a.coeff_lap[k];
          }
        }
      }
#pragma unroll
      for (int j = 0; j < RY; j++) {
        vj[j] = (double)win[j][FDN];
        hvj[j] = -0.5 * temp[j] + q_ve[j] * vj[j] + vnl[j];
      }
    }

#pragma unroll
    for (int j = 0; j < RY; j++) {
      if (!ok[j]) continue;
      const size_t g = (size_t)z * n2 + col[j];
      const double hv = STENCIL ? hvj[j] : 0.0, v = STENCIL ? vj[j] : 0.0;
      T o = T(0);
      if constexpr (PK == PK_ONES) {
        o = (T)start_val(io.chk, g);
        io.out[g] = o;
      } else if constexpr (PK == PK_DELTA) {
        o = (x == a.nloc && y[j] == a.nloc && z == a.nloc) ? T(1) : T(0);
        io.out[g] = o;
      } else if constexpr (PK == PK_DOTS) {
        o = pf[j];
      } else if constexpr (PK == PK_HV) {
        o = (T)hv;
        io.out[g] = o;
        acc0 += v * hv;
      } else if constexpr (PK == PK_LZB) {
        o = q_p1[j] - (T)io.ca * pf[j] - (T)io.cb * q_p2[j];
        io.out[g] = o;
        acc0 += (double)o * (double)o;
      } else if constexpr (PK == PK_CH1) {
        o = (T)((hv - chi * v) / zee);
        io.out[g] = o;
      } else if constexpr (PK == PK_CH || PK == PK_FD) {
        const double od = (2.0 * (hv - chi * v)) / zee - (double)q_p1[j];
        o = (T)od;
        io.out[g] = o;
        if (io.dbl) {
          acc0 += (double)o * (double)o;
          acc1 += (double)o * v;
        }
        if constexpr (PK == PK_FD) io.dacc[g] = q_d[j] + (double)o * io.cd / a.h3;
      } else if constexpr (PK == PK_FD01) {
        io.dacc[g] = 0.0 + (double)q_p1[j] * io.cd / a.h3 + (double)q_p2[j] * io.ce / a.h3;
      } else if constexpr (PK == PK_APPLY) {
        io.dout[g] = hv;
      } else if constexpr (PK == PK_LZF) {
        o = (T)hv;
        io.out[g] = o;
        acc0 += v * v;
        acc1 += v * hv;
      } else if constexpr (PK == PK_ADJ) {
        double od = (2.0 * (hv - chi * v)) / zee - (double)q_p1[j];
        if (x == a.nloc && y[j] == a.nloc && z == a.nloc) od += io.cd;
        o = (T)od;
        io.out[g] = o;
        io.dacc[g] = q_d[j] + io.ce * v * (double)q_p2[j];
      }
      if constexpr (DOTS) smo[y[j] * 32 + x] = o;
      if (x == a.nloc && y[j] == a.nloc && z == a.nloc) S.center_val = (double)o;
      if (!isfinite((double)o)) atomicOr(a.status, ST_NONFINITE);
    }
#pragma unroll
    for (int j = 0; j < RY; j++) {
      if constexpr (PK == PK_LZF) {
#pragma unroll
        for (int s = 0; s < 2 * FDN; s++) win[j][s] = win[j][s + 1];
        win[j][2 * FDN] = lzf_form(j, z + FDN + 1);
        lzf_load(j, z + FDN + 2);
      } else if constexpr (STENCIL) {
#pragma unroll
        for (int s = 0; s < 2 * FDN; s++) win[j][s] = win[j][s + 1];
        win[j][2 * FDN] = pf[j];
        pf[j] = ld_in(j, z + FDN + 2);
      }
      ld_point(j, z + 1);
    }
    st = st_next;
  }
  __syncthreads();
  if (tid == 0) S.ph = ph;
}

// Layout dispatch: L > 0 is the column layout with L columns per thread,
// L < 0 the row layout with -L rows per warp.
template <typename T, int L, int PK>
__device__ __forceinline__ void run_pass(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const PassIO<T> &io,
                                         const uint32_t (&wmask)[4], double &acc0, double &acc1) {
  if constexpr (L > 0) pass<T, L, PK>(a, S, dyn, io, wmask, acc0, acc1);
  else pass_rows<T, -L, PK>(a, S, dyn, io, wmask, acc0, acc1);
}

// Sturm count: eigenvalues of the leading m x m tridiagonal (aa, bb) below x,
// from the sign changes of the characteristic-polynomial sequence, rescaled
// by exact powers of two to stay in range.
__device__ int sturm_count(const double *d, const double *e, int m, double x) {
  double p0 = 1.0, p1 = d[0] - x;
  int s_prev = 1, cnt = 0;
  int s1 = p1 > 0.0 ? 1 : (p1 < 0.0 ? -1 : -s_prev);
  cnt += (s1 != s_prev);
  s_prev = s1;
  for (int i = 1; i < m; i++) {
    double p2 = (d[i] - x) * p1 - (e[i - 1] * e[i - 1]) * p0;
    int s2 = p2 > 0.0 ? 1 : (p2 < 0.0 ? -1 : -s_prev);
    cnt += (s2 != s_prev);
    s_prev = s2;
    p0 = p1;
    p1 = p2;
    double mx = fmax(fabs(p0), fabs(p1));
    if (mx > 0x1p+600) {
      p0 *= 0x1p-600;
      p1 *= 0x1p-600;
    } else if (mx < 0x1p-600 && mx > 0.0) {
      p0 *= 0x1p+600;
      p1 *= 0x1p+600;
    }
  }
  return cnt;
}

// Extreme eigenvalues of the Lanczos tridiagonal (the quantities
// TridiagEigenSolve, sq.cpp:1094-1180, returns) by 33-way multisection:
// warp 0 finds the smallest, warp 1 the largest.
__device__ void tridiag_extremes(NodeShared &S, int m) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp > 1) return;
  const double *d = S.aa, *e = S.bb;
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < m; i++) {
    double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < m - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
  }
  const double span = fmax(fabs(lo), fabs(hi));
  lo -= 1e-14 * span + 1e-300;
  hi += 1e-14 * span + 1e-300;
  for (int it = 0; it < 80; it++) {
    const double w = hi - lo;
    if (w <= 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300) break;
    const double x = lo + w * (double)(lane + 1) / 33.0;
    const int c = sturm_count(d, e, m, x);
    if (warp == 0) {
      const unsigned below = __ballot_sync(0xffffffffu, c >= 1);
      if (below == 0) lo = lo + w * 32.0 / 33.0;
      else {
        const int f = __ffs(below) - 1;
        const double nhi = lo + w * (double)(f + 1) / 33.0;
        if (f > 0) lo = lo + w * (double)f / 33.0;
        hi = nhi;
      }
    } else {
      const unsigned above = __ballot_sync(0xffffffffu, c < m);
      if (above == 0) hi = lo + w / 33.0;
      else {
        const int l = 31 - __clz(above);
        const double nlo = lo + w * (double)(l + 1) / 33.0;
        if (l < 31) hi = lo + w * (double)(l + 2) / 33.0;
        lo = nlo;
      }
    }
  }
  if (lane == 0) S.eig[warp] = 0.5 * (lo + hi);
}

// Block-wide ordered compaction of the replicas whose projector ball meets
// this node's window (the intersection test of nonlocal.cpp:66-108).
__device__ void setup_node(const NodeArgs &a, NodeShared &S) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int gx = a.pnode_s[0] + S.gi, gy = a.pnode_s[1] + S.gj, gz = a.pnode_s[2] + S.gk;
  const int ox = gx - a.nloc, oy = gy - a.nloc, oz = gz - a.nloc, n = a.n;
  if (tid == 0) S.n_ent = 0;
  __syncthreads();
  for (int base = 0; base < a.at.n_rep; base += nt) {
    const int r = base + tid;
    bool hit = false;
    int x0 = 0, x1 = 0, y0 = 0, y1 = 0, z0 = 0, z1 = 0, t = 0, nlocc = 0;
    int inn = 0, jnn = 0, knn = 0;
    if (r < a.at.n_rep) {
      inn = a.at.rep_nn[4 * r];
      jnn = a.at.rep_nn[4 * r + 1];
      knn = a.at.rep_nn[4 * r + 2];
      t = a.at.rep_nn[4 * r + 3];
      nlocc = a.at.typ_nlocc[t];
      x0 = max(inn - nlocc, ox) - ox;
      x1 = min(inn + nlocc, ox + n - 1) - ox;
      y0 = max(jnn - nlocc, oy) - oy;
      y1 = min(jnn + nlocc, oy + n - 1) - oy;
      z0 = max(knn - nlocc, oz) - oz;
      z1 = min(knn + nlocc, oz + n - 1) - oz;
      hit = x0 <= x1 && y0 <= y1 && z0 <= z1 && a.at.typ_nproj[t] > 0;
    }
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) S.scan[warp] = __popc(b);
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
      const int pos = S.n_ent + S.scan[warp] + __popc(b & ((1u << lane) - 1u));
      if (pos < MAXE) {
        const int Sd = 2 * nlocc + 1;
        S.e_x0[pos] = (short)x0;
        S.e_x1[pos] = (short)x1;
        S.e_y0[pos] = (short)y0;
        S.e_y1[pos] = (short)y1;
        S.e_z0[pos] = (short)z0;
        S.e_z1[pos] = (short)z1;
        S.e_S[pos] = Sd;
        S.e_sp2[pos] = plane_stride(Sd);
        S.e_nb[pos] = Sd * Sd * Sd;
        S.e_tx0[pos] = (short)(ox - inn + nlocc);
        S.e_ty0[pos] = (short)(oy - jnn + nlocc);
        S.e_tz0[pos] = (short)(oz - knn + nlocc);
        S.e_tab[pos] = a.at.rep_off[r];
        S.e_np[pos] = a.at.typ_nproj[t];
        S.e_atom[pos] = a.at.rep_atom[r];
        S.e_type[pos] = t;
      } else {
        atomicOr(a.status, ST_CAPACITY);
      }
    }
    __syncthreads();
    if (tid == 0) S.n_ent = min(S.n_ent + S.scan[32], MAXE);
    __syncthreads();
  }
  if (tid == 0) {
    int pb = 0;
    for (int e = 0; e < S.n_ent; e++) {
      S.e_pb[e] = pb;
      pb += S.e_np[e];
    }
    if (pb > MAXP) {
      atomicOr(a.status, ST_CAPACITY);
      pb = MAXP;
      int k = 0, acc = 0;
      while (k < S.n_ent && acc + S.e_np[k] <= MAXP) acc += S.e_np[k++];
      S.n_ent = k;
    }
    S.n_pi = pb;
  }
  __syncthreads();
  for (int e = 0; e < S.n_ent; e++)
    for (int q = tid; q < S.e_np[e]; q += nt) {
      S.p_den[S.e_pb[e] + q] = a.at.proj_denom[S.e_type[e] * MAXPROJ_TYPE + q];
      S.p_cur[S.e_pb[e] + q] = 0.0;
      S.p_nxt[S.e_pb[e] + q] = 0.0;
    }
  // Staged part of each table plane: the table rows of the box's window y
  // range, widened to multiples of 4 values (16-byte copy granularity).
  for (int e = tid; e < S.n_ent; e += nt) {
    const int Sd = S.e_S[e];
    S.e_ss[e] = ((S.e_ty0[e] + S.e_y0[e]) * Sd) & ~3;
    S.e_sc[e] = (((S.e_ty0[e] + S.e_y1[e] + 1) * Sd + 3) & ~3) - S.e_ss[e];
  }
  __syncthreads();
  for (int e = tid; e < S.n_ent; e += nt)
    S.e_geo[e] = make_int4(S.e_x0[e] | (S.e_x1[e] << 8) | (S.e_y0[e] << 16) | (S.e_y1[e] << 24),
                           (S.e_tx0[e] & 0xffff) | ((int)S.e_ty0[e] << 16), S.e_S[e] | (S.e_np[e] << 8) | (S.e_pb[e] << 16),
                           S.e_ss[e] | (S.e_sc[e] << 16));
  // Row and plane masks of the boxes: bit e of rowmask[y] (zmask[z]) is set
  // when box e's y (z) range holds window row y (plane z).
  for (int i = tid; i < 2 * n * 4; i += nt) {
    const int w = i & 3, k = (i >> 2) % n, zrow = i / (4 * n);
    uint32_t m = 0u;
    for (int b = 0; b < 32; b++) {
      const int e = w * 32 + b;
      if (e >= S.n_ent) break;
      const bool in = zrow ? (S.e_z0[e] <= k && k <= S.e_z1[e]) : (S.e_y0[e] <= k && k <= S.e_y1[e]);
      if (in) m |= 1u << b;
    }
    if (zrow) S.zmask[k][w] = m;
    else S.rowmask[k][w] = m;
  }
  __syncthreads();
}

// Row layout (two rows per warp): each warp lists the boxes that cover its
// rows; boxes beyond ITEMS go to the warp's residual mask.
__device__ void build_items(const NodeArgs &a, NodeShared &S, int4 *items) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n = a.n;
  const int y0 = 2 * warp, y1 = y0 + 1;
  int cnt = 0;
  uint32_t resid[4] = {0u, 0u, 0u, 0u};
  for (int base = 0; base < S.n_ent; base += 32) {
    const int e = base + lane;
    bool c0 = false, c1 = false;
    if (e < S.n_ent) {
      c0 = y0 < n && S.e_y0[e] <= y0 && y0 <= S.e_y1[e];
      c1 = y1 < n && S.e_y0[e] <= y1 && y1 <= S.e_y1[e];
    }
    const bool has = c0 || c1;
    const unsigned b = __ballot_sync(0xffffffffu, has);
    const int idx = cnt + __popc(b & ((1u << lane) - 1u));
    if (has) {
      if (idx < ITEMS) {
        const int Sd = S.e_S[e], x0 = S.e_x0[e], x1 = S.e_x1[e];
        const uint32_t xm = (x1 >= 31 ? 0xffffffffu : ((1u << (x1 + 1)) - 1u)) & ~((1u << x0) - 1u);
        const int rb0 = (S.e_ty0[e] + y0) * Sd + S.e_tx0[e] - S.e_ss[e];  // relative to the staged first value
        items[warp * ITEMS + idx] = make_int4(e | (S.e_z0[e] << 8) | (S.e_z1[e] << 16) | (S.e_np[e] << 24), (int)xm,
                                              (rb0 & 0xffff) | (Sd << 16) | ((c0 ? 1 : 0) | (c1 ? 2 : 0)) << 24,
                                              S.e_pb[e] | (S.e_sc[e] << 16));
      } else {
        resid[e >> 5] |= 1u << (e & 31);
      }
    }
    cnt += __popc(b);
  }
#pragma unroll
  for (int w = 0; w < 4; w++) resid[w] = __reduce_or_sync(0xffffffffu, resid[w]);
  if (lane == 0) {
    S.nitem[warp] = cnt < ITEMS ? cnt : ITEMS;
    for (int w = 0; w < 4; w++) S.resid[warp][w] = resid[w];
  }
}

// Boxes covering any row this warp's columns lie in (uniform over the warp).
template <int L>
__device__ void warp_masks(const NodeArgs &a, const NodeShared &S, uint32_t (&wmask)[4]) {
  const int n = a.n, n2 = n * n;
  uint32_t m[4] = {0u, 0u, 0u, 0u};
  if constexpr (L > 0) {
#pragma unroll
    for (int c = 0; c < L; c++) {
      const int col = threadIdx.x + c * blockDim.x;
      if (col >= n2) continue;
#pragma unroll
      for (int w = 0; w < 4; w++) m[w] |= S.rowmask[col / n][w];
    }
  } else {
    const int lane = threadIdx.x & 31, y = (threadIdx.x >> 5) * (-L) + lane;
    if (lane < -L && y < n) {
#pragma unroll
      for (int w = 0; w < 4; w++) m[w] = S.rowmask[y][w];
    }
  }
#pragma unroll
  for (int w = 0; w < 4; w++) wmask[w] = __reduce_or_sync(0xffffffffu, m[w]);
}

template <typename T>
__device__ __forceinline__ T *slot(const NodeArgs &a, int k) {
  const size_t nw = (size_t)a.n * a.n * a.n;
  return reinterpret_cast<T *>(a.scratch + blockIdx.x * a.scratch_stride + (size_t)k * nw * sizeof(double));
}

// Projector-ball points of the boxes meeting this window times the matvec
// steps taken: slot 0 all steps, slot 1 the Chebyshev steps only.
__device__ void count_proj_points(const NodeArgs &a, NodeShared &S, int passes, int cheb) {
  if (threadIdx.x != 0 || a.proj_points == nullptr) return;
  unsigned long long s = 0;
  for (int e = 0; e < S.n_ent; e++) s += (unsigned long long)S.e_np[e] * S.e_nb[e];
  atomicAdd(a.proj_points, s * (unsigned long long)passes);
  if (cheb) atomicAdd(a.proj_points + 1, s * (unsigned long long)passes);
}

// Lanczos bounds, sq.cpp:965-1092, one sweep per Lanczos step; vectors stored
// in T (FP32 in the mixed path), recurrences, dots and T_m in FP64.
//
// The reference's step k computes u = H v_k+1, a = <v_k+1, u>, w = u - a v_k+1
// - b v_k, b' = |w|, v_k+2 = w / b'.  Here sweep m applies H to the
// unnormalised vector W_m = w_m-1 (v_m = s_m W_m, s_m = 1/b_m-1), formed while
// it is loaded from the previous sweep's output Y_m-1 = H W_m-1 and the two
// previous W; the sweep accumulates <W_m, W_m> = b_m-1^2 and <W_m, H W_m> =
// a_m b_m-1^2, so after sweep m the tridiagonal T_m+1 of the reference's step
// m-1 is complete and its extreme eigenvalues decide convergence there.
// The nonlocal gather of sweep m needs chi^T W_m before the sweep; it follows
// from the same recurrence on the projections: chi^T W_m+1 = s_m (chi^T Y_m -
// a_m chi^T W_m) - b_m-1 s_m-1 chi^T W_m-1, with chi^T Y_m the dot products
// of the sweep's output.  The matvec count is the reference's (count + 1).
template <typename T, int C>
__device__ void lanczos(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const uint32_t (&mask)[4],
                        double &lmin_out, double &lmax_out, int &iters) {
  const double nw = (double)a.n * a.n * a.n;
  T *Y = slot<T>(a, 0);
  T *W[2] = {slot<T>(a, 1), slot<T>(a, 2)};
  double d0 = 0.0, d1 = 0.0;
  // chi^T W_0 with W_0 = v_0 = ones / |ones| (sq.cpp:538-546, 993-1004); the
  // mixed path may add a checkerboard, v_0 = (1 + c (-1)^(x+y+z)) / norm, whose
  // overlap with the top of the stencil's spectrum lets lambda_max converge in
  // fewer steps (|v|^2 = nw (1 + c^2) + 2c: one more even than odd point)
  const double chk = a.lz_chk;
  const double s0 = 1.0 / sqrt(nw * (1.0 + chk * chk) + 2.0 * chk);
  {
    PassIO<T> io;
    io.out = W[1];  // scratch: W[1] is overwritten before it is read
    io.chk = chk;
    run_pass<T, C, PK_ONES>(a, S, dyn, io, mask, d0, d1);
    for (int p = threadIdx.x; p < S.n_pi; p += blockDim.x) {
      S.pw_cur[p] = s0 * S.p_nxt[p];
      S.pw_prev[p] = 0.0;
      S.p_cur[p] = S.pw_cur[p] / S.p_den[p];
      S.p_nxt[p] = 0.0;
    }
    __syncthreads();
  }
  // state of the recurrence before sweep m: a = a_m-1, s = s_m-1, bs = b_m-2 s_m-2
  double a_prev = 0.0, s_prev = 1.0, bs_prev = 0.0;
  double lmin_prev = 0.0, lmax_prev = 0.0;
  if (threadIdx.x == 0) {
    S.count = 0;
    S.stop = 0;
  }
  __syncthreads();
  for (int m = 0;; m++) {
    PassIO<T> io;
    io.out = Y;
    io.wout = W[m & 1];
    if (m == 0) {
      io.konst = 1;
      io.chk = chk;
      io.sin = s0;
    } else {
      io.vin = Y;
      io.p1 = W[(m - 1) & 1];
      io.p2 = m >= 2 ? W[m & 1] : W[(m - 1) & 1];  // no third term in the first step (sq.cpp:1006-1014)
      io.s1 = s_prev;
      io.ca = a_prev;
      io.cb = bs_prev;
    }
    d0 = 0.0;
    d1 = 0.0;
    run_pass<T, C, PK_LZF>(a, S, dyn, io, mask, d0, d1);
    block_sum3(S, d0, d1, 0.0);
    // b_m-1 = |W_m| and a_m = <W_m, H W_m> / b_m-1^2 (W_0 is normalised)
    const double bm = m == 0 ? 1.0 : sqrt(S.scal[0]);
    const double am = S.scal[1] / (bm * bm);
    const double sm = 1.0 / bm;  // s_m: v_m = s_m W_m
    if (threadIdx.x == 0) {
      S.aa[m] = am;
      if (m > 0) S.bb[m - 1] = bm;
    }
    // chi^T W_m+1 = s_m (chi^T Y_m - a_m chi^T W_m) - b_m-1 s_m-1 chi^T W_m-1
    const double bs_cur = m == 0 ? 0.0 : bm * s_prev;
    for (int p = threadIdx.x; p < S.n_pi; p += blockDim.x) {
      const double nx = sm * (S.p_nxt[p] - am * S.pw_cur[p]) - bs_cur * S.pw_prev[p];
      S.pw_prev[p] = S.pw_cur[p];
      S.pw_cur[p] = nx;
      S.p_cur[p] = nx / S.p_den[p];
      S.p_nxt[p] = 0.0;
    }
    __syncthreads();
    a_prev = am;
    bs_prev = bs_cur;
    s_prev = sm;
    if (m == 0) continue;
    // the reference's step m-1: extreme eigenvalues of T_m+1 (sq.cpp:1050-1059)
    tridiag_extremes(S, m + 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      const double lmin = S.eig[0], lmax = S.eig[1];
      const double dl = fabs(lmin - lmin_prev), dm = fabs(lmax - lmax_prev);
      lmin_prev = lmin;
      lmax_prev = lmax;
      S.count = m;
      S.stop = !(S.count < LANCZOS_MAX_ITER && (dl > a.lanczos_tol || dm > a.lanczos_tol));
      if (S.count >= LANCZOS_MAX_ITER) atomicOr(a.status, ST_LANCZOS_MAXITER);
    }
    __syncthreads();
    if (S.stop) break;
  }
  lmin_out = S.eig[0] - a.lanczos_tol;
  lmax_out = S.eig[1] + a.lanczos_tol;
  iters = S.count;
  count_proj_points(a, S, S.count + 1, 0);  // Lanczos: iterations + the first matvec
}

// Moments and bounds from one FP64 Lanczos run started at the node's unit
// vector e_c (the quantities of sq.cpp:564-655, computed another way).  With
// Q_m the Lanczos basis (q_1 = e_c) and T_m its tridiagonal, p(H) e_c = Q_m
// p(T_m) e_1 for degree < m, hence e_c^T p(H) e_c = e_1^T p(T_m) e_1 for
// degree <= 2m - 1 (the Gauss-quadrature identity): m >= npl/2 + 1 steps give
// every Chebyshev moment mu_j = e_c^T T_j((H - chi)/zee) e_c, j <= npl, at any
// bounds, from a recurrence on the m x m tridiagonal.  The bounds are the
// extreme Ritz values of T_m -/+ lanczos_tol once both move by less than
// lanczos_tol between steps (sq.cpp:1050-1092's test), which for high npl the
// npl/2 + 1 steps usually already meet.  One sweep per step replaces the
// Lanczos sweeps for the bounds plus the npl/2 Chebyshev sweeps.
template <int C>
__device__ void lanczos_quadrature(const NodeArgs &a, NodeShared &S, unsigned char *dyn,
                                   const uint32_t (&mask)[4], double &lmin_out, double &lmax_out, int &iters,
                                   double *mu) {
  const int n = a.n;
  const int kmin = a.npl / 2 + 1;
  double *Y = slot<double>(a, 0);
  double *W[2] = {slot<double>(a, 1), slot<double>(a, 2)};
  double d0 = 0.0, d1 = 0.0;
  {  // e_c into Y, and chi^T e_c
    PassIO<double> io;
    io.out = Y;
    run_pass<double, C, PK_DELTA>(a, S, dyn, io, mask, d0, d1);
    for (int p = threadIdx.x; p < S.n_pi; p += blockDim.x) {
      S.pw_cur[p] = S.p_nxt[p];
      S.pw_prev[p] = 0.0;
      S.p_cur[p] = S.pw_cur[p] / S.p_den[p];
      S.p_nxt[p] = 0.0;
    }
    __syncthreads();
  }
  double a_prev = 0.0, s_prev = 1.0, bs_prev = 0.0;
  double lmin_prev = 0.0, lmax_prev = 0.0;
  if (threadIdx.x == 0) {
    S.count = 0;
    S.stop = 0;
  }
  __syncthreads();
  for (int m = 0;; m++) {
    PassIO<double> io;
    io.out = Y;
    io.wout = W[m & 1];
    io.vin = Y;
    if (m == 0) {  // W_0 = 1 (e_c - 0 e_c) - 0 e_c, exactly e_c
      io.p1 = Y;
      io.p2 = Y;
      io.s1 = 1.0;
    } else {
      io.p1 = W[(m - 1) & 1];
      io.p2 = m >= 2 ? W[m & 1] : W[(m - 1) & 1];
      io.s1 = s_prev;
      io.ca = a_prev;
      io.cb = bs_prev;
    }
    d0 = 0.0;
    d1 = 0.0;
    run_pass<double, C, PK_LZF>(a, S, dyn, io, mask, d0, d1);
    block_sum3(S, d0, d1, 0.0);
    const double bm = m == 0 ? 1.0 : sqrt(S.scal[0]);
    const double am = S.scal[1] / (bm * bm);
    const double sm = 1.0 / bm;
    if (threadIdx.x == 0) {
      S.aa[m] = am;
      if (m > 0) S.bb[m - 1] = bm;
    }
    const double bs_cur = m == 0 ? 0.0 : bm * s_prev;
    for (int p = threadIdx.x; p < S.n_pi; p += blockDim.x) {
      const double nx = sm * (S.p_nxt[p] - am * S.pw_cur[p]) - bs_cur * S.pw_prev[p];
      S.pw_prev[p] = S.pw_cur[p];
      S.pw_cur[p] = nx;
      S.p_cur[p] = nx / S.p_den[p];
      S.p_nxt[p] = 0.0;
    }
    __syncthreads();
    a_prev = am;
    bs_prev = bs_cur;
    s_prev = sm;
    // after sweep m the tridiagonal T_m+1 is complete; its extremes are
    // followed from npl/2 rows on, so that the run can stop at the npl/2 + 1
    // rows the moments need when the bounds have settled by then
    if (m + 2 < kmin) continue;
    tridiag_extremes(S, m + 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      const double lmin = S.eig[0], lmax = S.eig[1];
      const bool first = (m + 2 == kmin);
      const double dl = fabs(lmin - lmin_prev), dm = fabs(lmax - lmax_prev);
      lmin_prev = lmin;
      lmax_prev = lmax;
      S.count = m + 1;  // rows of T
      S.stop = !first && !(S.count < LANCZOS_MAX_ITER && (dl > a.lanczos_tol || dm > a.lanczos_tol));
      if (S.count >= LANCZOS_MAX_ITER) {
        S.stop = 1;
        atomicOr(a.status, ST_LANCZOS_MAXITER);
      }
    }
    __syncthreads();
    if (S.stop) break;
  }
  const int k = S.count;
  lmin_out = S.eig[0] - a.lanczos_tol;
  lmax_out = S.eig[1] + a.lanczos_tol;
  iters = k - 1;  // matvecs = iters + 1, as for the reference's Lanczos
  count_proj_points(a, S, k, 0);
  // mu_j = e_1^T T_j(That) e_1, That = (T_k - chi) / zee: the Chebyshev
  // recurrence on k-vectors, one warp, in the (now free) window-vector slots
  // (k <= n^3: Lanczos on the window cannot take more steps than its size)
  const double chi = 0.5 * (lmax_out + lmin_out), zee = 0.5 * (lmax_out - lmin_out);
  if (threadIdx.x < 32 && (long long)k <= (long long)n * n * n) {
    const int lane = threadIdx.x;
    double *v0 = Y, *v1 = W[0], *v2 = W[1];
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
  } else if (threadIdx.x == 0 && (long long)k > (long long)n * n * n) {
    atomicOr(a.status, ST_CAPACITY);  // the moment recurrence's k-vectors do not fit the window slots
  }
  __syncthreads();
}

// Chebyshev moments (sq.cpp:564-655) in precision T.
template <typename T, int C>
__device__ void moments(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const uint32_t (&mask)[4],
                        double chi, double zee, double *mu) {
  T *B0 = slot<T>(a, 0), *B1 = slot<T>(a, 1);
  double d0 = 0.0, d1 = 0.0;
  {
    PassIO<T> io;
    io.out = B0;
    run_pass<T, C, PK_DELTA>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
  }
  {
    PassIO<T> io;
    io.vin = B0;
    io.out = B1;
    io.ca = chi;
    io.cb = zee;
    run_pass<T, C, PK_CH1>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
  }
  const double htemp = S.center_val;
  if (threadIdx.x == 0) {
    mu[0] = (double)(1.0 / a.h3);
    mu[1] = (double)(htemp / a.h3);
  }
  T *t0 = B0, *t1 = B1;
  const int q1 = (int)rint(0.25 * a.npl), q2 = (int)rint(0.5 * a.npl);
  for (int nq = 2; nq <= q2; nq++) {
    PassIO<T> io;
    io.vin = t1;
    io.p1 = t0;
    io.out = t0;
    io.ca = chi;
    io.cb = zee;
    io.dbl = nq > q1;
    d0 = 0.0;
    d1 = 0.0;
    run_pass<T, C, PK_CH>(a, S, dyn, io, mask, d0, d1);
    if (nq > q1) block_sum3(S, d0, d1, 0.0);
    rotate_proj(S, 1.0);
    if (threadIdx.x == 0) {
      mu[nq] = (double)(S.center_val / a.h3);
      if (nq > q1) {
        mu[2 * nq] = (double)((2 * S.scal[0] - 1) / a.h3);
        mu[2 * nq - 1] = (double)((2 * S.scal[1] - htemp) / a.h3);
      }
    }
    T *tt = t0;
    t0 = t1;
    t1 = tt;
  }
  count_proj_points(a, S, q2, 1);  // Chebyshev: npl/2 matvecs
}

// ForcesNonLocal for one node (forces.cpp:318-578).
template <typename T, int C>
__device__ void node_forces(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const uint32_t (&mask)[4],
                            double chi, double zee, const double *ci, double *fslot) {
  T *B0 = slot<T>(a, 0), *B1 = slot<T>(a, 1);
  double *D = slot<double>(a, 3);
  double d0 = 0.0, d1 = 0.0;
  {
    PassIO<T> io;
    io.out = B0;
    run_pass<T, C, PK_DELTA>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
  }
  {
    PassIO<T> io;
    io.vin = B0;
    io.out = B1;
    io.ca = chi;
    io.cb = zee;
    run_pass<T, C, PK_CH1>(a, S, dyn, io, mask, d0, d1);
  }
  {
    PassIO<T> io;
    io.p1 = B0;
    io.p2 = B1;
    io.dacc = D;
    io.cd = ci[0];
    io.ce = ci[1];
    run_pass<T, C, PK_FD01>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
  }
  T *t0 = B0, *t1 = B1;
  for (int nq = 2; nq <= a.npl; nq++) {
    PassIO<T> io;
    io.vin = t1;
    io.p1 = t0;
    io.out = t0;
    io.ca = chi;
    io.cb = zee;
    io.dacc = D;
    io.cd = ci[nq];
    run_pass<T, C, PK_FD>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
    T *tt = t0;
    t0 = t1;
    t1 = tt;
  }
  __threadfence_block();
  __syncthreads();
  // Gradient of D (zero outside the window) on each ball that holds the
  // window centre, contracted with that replica's projectors.
  const int n = a.n, nl = a.nloc, n2 = n * n;
  const double *Dc = D;
  int slotc = 0;
  for (int e = 0; e < S.n_ent; e++) {
    if (nl < S.e_x0[e] || nl > S.e_x1[e] || nl < S.e_y0[e] || nl > S.e_y1[e] || nl < S.e_z0[e] || nl > S.e_z1[e])
      continue;
    const int x0 = S.e_x0[e], y0 = S.e_y0[e], z0 = S.e_z0[e];
    const int bx = S.e_x1[e] - x0 + 1, by = S.e_y1[e] - y0 + 1, bz = S.e_z1[e] - z0 + 1;
    const int Sd = S.e_S[e], sp2 = S.e_sp2[e], vol = bx * by * bz;
    const int tx0 = S.e_tx0[e], ty0 = S.e_ty0[e], tz0 = S.e_tz0[e];
    const double *U = a.at.tab64 + S.e_tab[e];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int q = 0; q < S.e_np[e]; q++) {
      double ax = 0.0, ay = 0.0, az = 0.0;
      for (int i = threadIdx.x; i < vol; i += blockDim.x) {
        const int x = x0 + i % bx, y = y0 + (i / bx) % by, z = z0 + i / (bx * by);
        const size_t w = (size_t)z * n2 + y * n + x;
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int k = 1; k <= FDN; k++) {
          const double xm = x - k >= 0 ? Dc[w - k] : 0.0, xp = x + k < n ? Dc[w + k] : 0.0;
          const double ym = y - k >= 0 ? Dc[w - (size_t)k * n] : 0.0, yp = y + k < n ? Dc[w + (size_t)k * n] : 0.0;
          const double zm = z - k >= 0 ? Dc[w - (size_t)k * n2] : 0.0, zp = z + k < n ? Dc[w + (size_t)k * n2] : 0.0;
          gx += (-xm + xp) * a.coeff_grad[k];
          gy += (-ym + yp) * a.coeff_grad[k];
          gz += (-zm + zp) * a.coeff_grad[k];
        }
        const double u = U[(long long)(q * Sd + tz0 + z) * sp2 + (ty0 + y) * Sd + tx0 + x];
        ax += u * gx;
        ay += u * gy;
        az += u * gz;
      }
      block_sum3(S, ax, ay, az);
      const double uc = U[(long long)(q * Sd + tz0 + nl) * sp2 + (ty0 + nl) * Sd + tx0 + nl];
      const double den = S.p_den[S.e_pb[e] + q];
      fx += S.scal[0] / den * uc;
      fy += S.scal[1] / den * uc;
      fz += S.scal[2] / den * uc;
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

// Gradient of L = sum_j g_j mu_j (mu_j = e_c^T T_j(Ht) e_c / h^3, the node's
// Chebyshev moments, Ht = (H - chi)/zee with chi, zee held fixed) with respect
// to Veff on the node's window, added into a.g_veff, and (a.g_atoms set) with
// respect to the replica positions through the projectors, added into the
// gradient of each replica's atom.  Forward recursion t_0 = e_c, t_1 = Ht t_0,
// t_k+1 = 2 Ht t_k - t_k-1 (sq.cpp:579-616) with the pair (t_sK, t_sK+1) and
// the projections of t_sK+1 checkpointed every K steps; reverse Clenshaw
// recursion a_k = (g_k/h^3) e_c + 2 Ht a_k+1 - a_k+2 from k = npl down to 1,
// segment by segment, recomputing each segment's vectors from its checkpoint;
// dL/dHt = a_1 t_0^T + 2 sum_k a_k+1 t_k^T, so
//   dL/dVeff(x) = (a_1 t_0 + 2 sum_k a_k+1 t_k)(x) / zee and, with
//   dVnl/dR = sum_q (dchi_q chi_q^T + chi_q dchi_q^T) / Denom_q,
//   dL/dR = sum_k c_k sum_q [(a_k+1.dchi_q)(chi_q.t_k) + (a_k+1.chi_q)(dchi_q.t_k)]
//           / (Denom_q zee),  c_k = 2 (k >= 1), 1 (k = 0).
template <int C>
__device__ void node_vjp(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const uint32_t (&mask)[4],
                         double chi, double zee, const double *g) {
  const int n = a.n, npl = a.npl, K = VJP_K, nseg = (npl + K - 1) / K;
  const size_t nw = (size_t)n * n * n;
  const bool at = a.g_atoms != nullptr;
  double *ck = a.vjp + (size_t)blockIdx.x * a.vjp_stride;  // [nseg][2][nw]
  double *seg = ck + (size_t)nseg * 2 * nw;                  // [K][nw]
  double *A = seg + (size_t)K * nw;                          // [3][nw]
  double *G = A + 3 * nw;                                    // [nw]
  double *ckp = G + nw;                                      // [nseg][MAXP]
  // atom gradients: chi / dchi dots of the segment's t ([K][MAXP], [K][3][MAXP]),
  // dchi dots of a_k+1 (pgA), of the output being formed (pgN), saved (pgS),
  // and the per-projector sums (dRp)
  double *Tt = at ? a.vjp_at + (size_t)blockIdx.x * a.vjp_at_stride : nullptr;
  double *Tg = at ? Tt + (size_t)K * MAXP : nullptr;
  double *pgA = at ? Tg + (size_t)3 * K * MAXP : nullptr;
  double *pgN = at ? pgA + 3 * MAXP : nullptr, *pgS = at ? pgN + 3 * MAXP : nullptr;
  double *dRp = at ? pgS + 3 * MAXP : nullptr;
  const int npi = S.n_pi;
  double d0 = 0.0, d1 = 0.0;
  for (size_t i = threadIdx.x; i < nw; i += blockDim.x) G[i] = 0.0;
  if (at)
    for (int i = threadIdx.x; i < 3 * MAXP; i += blockDim.x) {
      dRp[i] = 0.0;
      pgN[i] = 0.0;
    }
  __syncthreads();
  auto gradio = [&](PassIO<double> &io) {
    if (at) {
      io.pg = pgN;
      io.dtab = a.dtab;
      io.dstride = a.dtab_stride;
    }
  };
  // forward: checkpoints only
  {
    PassIO<double> io;
    io.out = ck;
    run_pass<double, C, PK_DELTA>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
  }
  {
    PassIO<double> io;
    io.vin = ck;
    io.out = ck + nw;
    io.ca = chi;
    io.cb = zee;
    run_pass<double, C, PK_CH1>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
    for (int p = threadIdx.x; p < npi; p += blockDim.x) ckp[p] = S.p_cur[p];
  }
  const double *tm1 = ck, *tk = ck + nw;
  for (int k = 1; k + 1 <= npl - 1; k++) {
    const int kk = k + 1, sg = kk / K, r = kk % K;
    double *out = r == 0 ? ck + (size_t)(2 * sg) * nw : (r == 1 ? ck + (size_t)(2 * sg + 1) * nw : seg + r * nw);
    PassIO<double> io;
    io.vin = tk;
    io.p1 = tm1;
    io.out = out;
    io.ca = chi;
    io.cb = zee;
    run_pass<double, C, PK_CH>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
    if (r == 1)
      for (int p = threadIdx.x; p < npi; p += blockDim.x) ckp[(size_t)sg * MAXP + p] = S.p_cur[p];
    tm1 = tk;
    tk = out;
  }
  // dchi dots of the output just formed -> dst (scaled), pgN cleared
  auto take_pg = [&](double *dst, double scale) {
    for (int i = threadIdx.x; i < 3 * MAXP; i += blockDim.x) {
      dst[i] = scale * pgN[i];
      pgN[i] = 0.0;
    }
  };
  // backward: a_npl = (g_npl / h^3) e_c (stored as e_c with a lazy scale), a_npl+1 = 0
  const double h3 = a.h3;
  double *an1 = A, *an2 = A, *afree = A + nw, *aspare = A + 2 * nw;
  double sc1 = g[npl] / h3, sc2 = 0.0;
  {
    PassIO<double> io;
    io.out = A;
    gradio(io);
    run_pass<double, C, PK_DELTA>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, sc1);
    if (at) take_pg(pgA, sc1);
    __syncthreads();
  }
  for (int sg = nseg - 1; sg >= 0; sg--) {
    const int lo = sg * K, hi = min(lo + K - 1, npl - 1);
    if (hi < 1) break;
    const double *tv[VJP_K];
    tv[0] = ck + (size_t)(2 * sg) * nw;
    if (hi >= lo + 1) tv[1] = ck + (size_t)(2 * sg + 1) * nw;
    for (int j = 2; j < K; j++) tv[j] = seg + j * nw;
    const bool recompute = hi >= lo + 2;
    if (recompute || at) {
      // keep the adjoint's projections aside
      for (int p = threadIdx.x; p < npi; p += blockDim.x) S.pw_prev[p] = S.p_cur[p];
      if (at)
        for (int i = threadIdx.x; i < 3 * MAXP; i += blockDim.x) pgS[i] = pgA[i];
      __syncthreads();
    }
    if (at) {
      // chi and dchi dots of the checkpointed t_lo, t_lo+1
      for (int j = 0; j < 2 && lo + j <= hi; j++) {
        for (int p = threadIdx.x; p < npi; p += blockDim.x) S.p_nxt[p] = 0.0;
        __syncthreads();
        PassIO<double> io;
        io.din = tv[j];
        gradio(io);
        run_pass<double, C, PK_DOTS>(a, S, dyn, io, mask, d0, d1);
        for (int p = threadIdx.x; p < npi; p += blockDim.x) Tt[(size_t)j * MAXP + p] = S.p_nxt[p];
        take_pg(Tg + (size_t)j * 3 * MAXP, 1.0);
        __syncthreads();
      }
    }
    if (recompute) {
      // recompute t_lo+2 .. t_hi from the checkpoint
      for (int p = threadIdx.x; p < npi; p += blockDim.x) {
        S.p_cur[p] = ckp[(size_t)sg * MAXP + p];
        S.p_nxt[p] = 0.0;
      }
      __syncthreads();
      for (int k = lo + 1; k + 1 <= hi; k++) {
        PassIO<double> io;
        io.vin = tv[k - lo];
        io.p1 = tv[k - 1 - lo];
        io.out = seg + (size_t)(k + 1 - lo) * nw;
        io.ca = chi;
        io.cb = zee;
        gradio(io);
        run_pass<double, C, PK_CH>(a, S, dyn, io, mask, d0, d1);
        if (at) {
          for (int p = threadIdx.x; p < npi; p += blockDim.x) Tt[(size_t)(k + 1 - lo) * MAXP + p] = S.p_nxt[p];
          take_pg(Tg + (size_t)(k + 1 - lo) * 3 * MAXP, 1.0);
        }
        rotate_proj(S, 1.0);
      }
    }
    if (recompute || at) {
      for (int p = threadIdx.x; p < npi; p += blockDim.x) {
        S.p_cur[p] = S.pw_prev[p];
        S.p_nxt[p] = 0.0;
      }
      if (at)
        for (int i = threadIdx.x; i < 3 * MAXP; i += blockDim.x) pgA[i] = pgS[i];
      __syncthreads();
    }
    for (int k = hi; k >= lo && k >= 1; k--) {
      // a_k = (g_k/h^3) e_c + 2 Ht a_k+1 - a_k+2 in place of a_k+2 (or a free
      // slot while a_k+2 is zero); G += 2 a_k+1 t_k
      double *out = sc2 != 0.0 ? an2 : afree;
      PassIO<double> io;
      io.vin = an1;
      io.sin = sc1;
      io.p1 = sc2 != 0.0 ? an2 : an1;
      io.s1 = sc2;
      io.p2 = tv[k - lo];
      io.out = out;
      io.ca = chi;
      io.cb = zee;
      io.cd = g[k] / h3;
      io.ce = 2.0;
      io.dacc = G;
      gradio(io);
      run_pass<double, C, PK_ADJ>(a, S, dyn, io, mask, d0, d1);
      if (at) {
        // step k's term: a_k+1 (projections in p_cur, dchi dots in pgA) with t_k
        for (int p = threadIdx.x; p < npi; p += blockDim.x) {
          const double D = S.p_den[p], Ak = S.p_cur[p] * D, Tk = Tt[(size_t)(k - lo) * MAXP + p];
#pragma unroll
          for (int al = 0; al < 3; al++)
            dRp[al * MAXP + p] +=
                2.0 * (pgA[al * MAXP + p] * Tk + Ak * Tg[((size_t)(k - lo) * 3 + al) * MAXP + p]) / D;
        }
        __syncthreads();
        take_pg(pgA, 1.0);
      }
      rotate_proj(S, 1.0);
      if (out == afree) {
        afree = aspare;
        aspare = nullptr;
      }
      an2 = an1;
      sc2 = sc1;
      an1 = out;
      sc1 = 1.0;
    }
  }
  __syncthreads();
  // a_1 t_0 (t_0 = e_c): the last step's centre value; for the atoms, a_1
  // with t_0's dots (segment 0, kept in Tt[0], Tg[0])
  if (threadIdx.x == 0) G[(size_t)(a.nloc * n + a.nloc) * n + a.nloc] += S.center_val;
  if (at)
    for (int p = threadIdx.x; p < npi; p += blockDim.x) {
      const double D = S.p_den[p], A1 = S.p_cur[p] * D, T0 = Tt[p];
#pragma unroll
      for (int al = 0; al < 3; al++) dRp[al * MAXP + p] += (pgA[al * MAXP + p] * T0 + A1 * Tg[al * MAXP + p]) / D;
    }
  __syncthreads();
  // dL/dVeff on the block with halo: the window of node (gi, gj, gk) starts at
  // (gi, gj, gk) in the halo'd block
  const double iz = 1.0 / zee;
  for (size_t i = threadIdx.x; i < nw; i += blockDim.x) {
    const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((size_t)n * n));
    const size_t ve = ((size_t)(S.gk + z) * a.ey + (S.gj + y)) * a.ex + (S.gi + x);
    atomicAdd(&a.g_veff[ve], G[i] * iz);
  }
  // dL/dR: each box's projectors summed into its replica's atom
  if (at)
    for (int i = threadIdx.x; i < S.n_ent * 3; i += blockDim.x) {
      const int e = i / 3, al = i % 3;
      double sum = 0.0;
      for (int q = 0; q < S.e_np[e]; q++) sum += dRp[al * MAXP + S.e_pb[e] + q];
      atomicAdd(&a.g_atoms[(size_t)S.e_atom[e] * 3 + al], sum * iz);
    }
  count_proj_points(a, S, 2 * npl, 1);
}

// L is the plane-loop layout (L > 0: L columns per thread; L < 0: -L rows
// per warp); MAXT is the launch bound, which sets the register budget per
// thread (64K / MAXT); KIND selects the modes the instantiation carries
// (KIND_SQ: SQ, moments with given bounds, matvec; KIND_SQ32: SQ of the
// FP32-mixed path, Lanczos vectors in FP32; KIND_FORCES; KIND_VJP), so the
// register allocation of each is its own.
template <int C, int MAXT, int KIND>
__global__ void __launch_bounds__(MAXT, 1) node_kernel(NodeArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  NodeShared &S = *reinterpret_cast<NodeShared *>(smem);
  unsigned char *dyn = smem + kSharedFixed;
  if (threadIdx.x == 0) {
    for (int k = 0; k < NSTAGE; k++) mbar_init(&S.mbar[k], 1);
    mbar_fence_init();
    S.ph = 0;
    S.stalled = 0;
  }
  __syncthreads();
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
    if (node < 0 || S.stalled) break;
    setup_node(a, S);
    plane_offsets(a, S, off_table(a, dyn), cross_list(a, dyn));
    __syncthreads();
    uint32_t mask[4];
    warp_masks<C>(a, S, mask);
    if constexpr (C == -2) {
      build_items(a, S, row_items(a, dyn));
      __syncthreads();
    }
    if constexpr (KIND == KIND_LQ) {
      double lmin = 0.0, lmax = 0.0;
      int iters = 0;
      double *mu = a.rho_pj + (size_t)node * (a.npl + 1);
      lanczos_quadrature<C>(a, S, dyn, mask, lmin, lmax, iters, mu);
      if (threadIdx.x == 0) {
        a.chi[node] = 0.5 * (lmax + lmin);
        a.zee[node] = 0.5 * (lmax - lmin);
        if (a.lmin) a.lmin[node] = lmin;
        if (a.lmax) a.lmax[node] = lmax;
        if (a.lanczos_iters) a.lanczos_iters[node] = iters;
      }
    } else if constexpr (KIND == KIND_SQ || KIND == KIND_SQ32) {
      using TV = typename std::conditional<KIND == KIND_SQ32, float, double>::type;
      if (a.mode == MODE_SQ || a.mode == MODE_MOMENTS) {
        // SQ: Lanczos bounds then moments; MODE_MOMENTS: moments with given bounds
        double lmin = 0.0, lmax = 0.0, chi, zee;
        int iters = 0;
        if (a.mode == MODE_SQ) {
          lanczos<TV, C>(a, S, dyn, mask, lmin, lmax, iters);
          chi = (lmax + lmin) / 2;  // sq.cpp:564-565
          zee = (lmax - lmin) / 2;
        } else {
          chi = a.chi_in[node];
          zee = a.zee_in[node];
        }
        double *mu = a.rho_pj + (size_t)node * (a.npl + 1);
        // moments stay FP64 in both paths: FP32 storage of the Chebyshev
        // vectors grows a rounding error injected at step i like (k - i) by
        // step k, ~5e-6 of max rho after 48 steps, above the mixed budget
        moments<double, C>(a, S, dyn, mask, chi, zee, mu);
        if (a.mode == MODE_SQ && threadIdx.x == 0) {
          a.chi[node] = chi;
          a.zee[node] = zee;
          if (a.lmin) a.lmin[node] = lmin;
          if (a.lmax) a.lmax[node] = lmax;
          if (a.lanczos_iters) a.lanczos_iters[node] = iters;
        }
      } else if constexpr (KIND == KIND_SQ) {
        const size_t nw = (size_t)a.n * a.n * a.n;
        double d0 = 0.0, d1 = 0.0;
        PassIO<double> io;
        io.din = a.apply_in + (size_t)S.qidx * nw;
        run_pass<double, C, PK_DOTS>(a, S, dyn, io, mask, d0, d1);
        rotate_proj(S, 1.0);
        io.dout = a.apply_out + (size_t)S.qidx * nw;
        run_pass<double, C, PK_APPLY>(a, S, dyn, io, mask, d0, d1);
      }
    } else if constexpr (KIND == KIND_FORCES) {
      double *fs = a.fslots + (size_t)S.qidx * FSLOTS * 4;
      for (int i = threadIdx.x; i < FSLOTS * 4; i += blockDim.x) fs[i] = (i % 4 == 0) ? -1.0 : 0.0;
      __syncthreads();
      const double *ci = a.ci + (size_t)node * (a.npl + 1);
      if (a.mixed) node_forces<float, C>(a, S, dyn, mask, a.chi_in[node], a.zee_in[node], ci, fs);
      else node_forces<double, C>(a, S, dyn, mask, a.chi_in[node], a.zee_in[node], ci, fs);
    } else {
      node_vjp<C>(a, S, dyn, mask, a.chi_in[node], a.zee_in[node], a.gmu + (size_t)node * (a.npl + 1));
    }
    __syncthreads();
  }
}


// Layout of a launch: cols == 0 picks the column layout with one column per
// thread when the window has at most 1024 columns, two otherwise; 1 or 2
// force that many columns per thread; -2 selects the row layout (two window
// rows per warp, windows up to 32 wide).
inline int layout_of(int n, int cols) {
  if (cols == 0) return n * n <= 1024 ? 1 : 2;
  return cols;
}

inline int threads_of(int n, int cols) {
  const int L = layout_of(n, cols);
  if (L < 0) return 32 * ((n + (-L) - 1) / (-L));
  const int per = (n * n + L - 1) / L;
  return ((per + 31) / 32) * 32;
}

inline size_t smem_limit() { return g_smem_optin > 0 ? (size_t)g_smem_optin : 232448; }
inline size_t smem_base(int n, int row) { return kSharedFixed + planes_bytes(n, row) + offtab_bytes(n, row); }

// Largest slice stage the block's shared memory leaves room for (offsets are
// int16 element counts).
inline size_t stage_bytes_max(int n, int row) {
  const size_t base = smem_base(n, row), limit = smem_limit();
  if (base + NSTAGE * 256 > limit) return 0;
  const size_t sb = ((limit - base) / NSTAGE) & ~size_t(15);
  const size_t cap = ((size_t)32767 * sizeof(double)) & ~size_t(15);
  return sb < cap ? sb : cap;
}

template <int C, int MAXT, int KIND>
cudaError_t set_smem_attr(int n) {
  const int row = C < 0;
  if (row && n > 32) return cudaSuccess;
  return cudaFuncSetAttribute(node_kernel<C, MAXT, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(smem_base(n, row) + NSTAGE * stage_bytes_max(n, row)));
}

// Shared-memory attributes of every layout variant of one kernel group.
template <int KIND>
cudaError_t setup_kind(int n) {
  cudaError_t r[4] = {set_smem_attr<-2, 512, KIND>(n), set_smem_attr<1, 1024, KIND>(n),
                      set_smem_attr<2, 576, KIND>(n), set_smem_attr<2, 1024, KIND>(n)};
  for (cudaError_t x : r)
    if (x != cudaSuccess) return x;
  return cudaSuccess;
}

// Launch one kernel group with the layout `cols` asks for.
template <int KIND>
cudaError_t launch_kind(const NodeArgs &args, int grid, int cols, cudaStream_t s) {
  const int threads = threads_of(args.n, cols);
  if (threads > 1024 || threads < 64) return cudaErrorInvalidConfiguration;
  NodeArgs a = args;
  const int L = layout_of(a.n, cols);
  a.row_layout = L < 0;
  const size_t mx = stage_bytes_max(a.n, a.row_layout);
  if (a.n > MAXN || mx == 0) return cudaErrorInvalidValue;
  if (a.stage_bytes == 0 || a.stage_bytes > mx) a.stage_bytes = mx;
  a.stage_bytes = (a.stage_bytes + 15) & ~size_t(15);
  const size_t smem = smem_base(a.n, a.row_layout) + NSTAGE * a.stage_bytes;
  if (L == -2) {
    if (a.n > 32 || threads > 512) return cudaErrorInvalidConfiguration;
    node_kernel<-2, 512, KIND><<<grid, threads, smem, s>>>(a);
  } else if (L == 1) {
    node_kernel<1, 1024, KIND><<<grid, threads, smem, s>>>(a);
  } else if (L == 2) {
    if (threads <= 576) node_kernel<2, 576, KIND><<<grid, threads, smem, s>>>(a);
    else node_kernel<2, 1024, KIND><<<grid, threads, smem, s>>>(a);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

}  // namespace sqb
