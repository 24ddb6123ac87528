// Node kernel: the per-grid-node work of the SQ step on sm_100a.
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
// nonlocal term is fused into the same plane sweep: a per-column bit mask of
// the projector boxes covering the column drives the gather of
// sum_J c_J chi_J, and the dot products chi_J . v_new that the next matvec
// needs are accumulated from the freshly written plane by warp-owned atoms.
#include <cmath>
#include <cstdio>

#include "sqb_internal.cuh"

namespace sqb {

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
};

struct NodeShared {
  int node, qidx, gi, gj, gk;
  int n_ent, n_pi, stop, count;
  double center_val;
  double scal[4];
  double red[32][3];
  double aa[MAXL];
  double bb[MAXL];
  double eig[2];
  short e_x0[MAXE], e_x1[MAXE], e_y0[MAXE], e_y1[MAXE], e_z0[MAXE], e_z1[MAXE];
  int e_base[MAXE], e_S[MAXE], e_pb[MAXE], e_np[MAXE], e_nb[MAXE], e_atom[MAXE], e_type[MAXE];
  long long e_tab[MAXE];
  int scan[33];
  double p_cur[MAXP];
  double p_nxt[MAXP];
  double p_den[MAXP];
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
};

template <typename T>
__device__ __forceinline__ const T *veff_of(const NodeArgs &a);
template <>
__device__ __forceinline__ const double *veff_of<double>(const NodeArgs &a) { return a.veff64; }
template <>
__device__ __forceinline__ const float *veff_of<float>(const NodeArgs &a) { return a.veff32; }
template <typename T>
__device__ __forceinline__ const T *tab_of(const NodeArgs &a);
template <>
__device__ __forceinline__ const double *tab_of<double>(const NodeArgs &a) { return a.at.tab64; }
template <>
__device__ __forceinline__ const float *tab_of<float>(const NodeArgs &a) { return a.at.tab32; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
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

// Accumulate chi_J,q . plane into p_nxt for every projector box crossing plane zz.
template <typename T>
__device__ void dot_phase(NodeShared &S, const T *plane, int zz, int n, const T *tab) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int e = warp; e < S.n_ent; e += nw) {
    if (zz < S.e_z0[e] || zz > S.e_z1[e]) continue;
    const int x0 = S.e_x0[e], y0 = S.e_y0[e];
    const int bx = S.e_x1[e] - x0 + 1, cnt = bx * (S.e_y1[e] - y0 + 1);
    const int Sd = S.e_S[e];
    const T *U = tab + S.e_tab[e] + S.e_base[e] + zz * Sd * Sd;
    for (int q = 0; q < S.e_np[e]; q++) {
      double acc = 0.0;
      for (int i = lane; i < cnt; i += 32) {
        const int y = y0 + i / bx, x = x0 + i % bx;
        acc += (double)plane[y * n + x] * (double)U[(long long)q * S.e_nb[e] + y * Sd + x];
      }
      acc = warp_sum(acc);
      if (lane == 0) S.p_nxt[S.e_pb[e] + q] += acc;
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

// One sweep over the window's z-planes.
template <typename T, int C, int PK>
__device__ void pass(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const PassIO<T> &io,
                     const uint32_t (&mask)[C][4], double &acc0, double &acc1) {
  constexpr bool STENCIL = (PK == PK_HV || PK == PK_CH1 || PK == PK_CH || PK == PK_FD || PK == PK_APPLY);
  constexpr bool DOTS = (PK == PK_ONES || PK == PK_DELTA || PK == PK_DOTS || PK == PK_LZB || PK == PK_CH1 ||
                         PK == PK_CH || PK == PK_FD);
  const int n = a.n, n2 = n * n, P = n + 2 * FDN, P2 = P * P;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int centre_col = a.nloc * n + a.nloc;
  T *sm_in = reinterpret_cast<T *>(dyn);
  T *sm_out = sm_in + 2 * P2;
  const T *veff = veff_of<T>(a);
  const T *tab = tab_of<T>(a);
  const size_t vplane = (size_t)a.ex * a.ey;

  if (STENCIL) {
    for (int i = tid; i < 2 * P2; i += nt) sm_in[i] = T(0);
  }
  __syncthreads();

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
  T q_ve[C], q_p1[C], q_p2[C];
  double q_d[C];
  auto ld_point = [&](int c, int z) {
    if (!ok[c] || z >= n) return;
    const size_t g = (size_t)z * n2 + col[c];
    if constexpr (STENCIL) q_ve[c] = veff[vb[c] + (size_t)z * vplane];
    if constexpr (PK == PK_LZB || PK == PK_CH || PK == PK_FD || PK == PK_FD01) q_p1[c] = io.p1[g] * (T)io.s1;
    if constexpr (PK == PK_LZB || PK == PK_FD01) q_p2[c] = io.p2[g] * (T)io.s2;
    if constexpr (PK == PK_LZB || PK == PK_DOTS) pf[c] = ld_in(c, z);
    if constexpr (PK == PK_FD) q_d[c] = io.dacc[g];
  };
#pragma unroll
  for (int c = 0; c < C; c++) {
    if constexpr (STENCIL) {
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

  for (int z = 0; z <= n; z++) {
    T *smz = sm_in + (z & 1) * P2;
    T *smo = sm_out + (z & 1) * n2;
    if (STENCIL && z < n) {
#pragma unroll
      for (int c = 0; c < C; c++)
        if (ok[c]) smz[(cy[c] + FDN) * P + cx[c] + FDN] = win[c][FDN];
    }
    __syncthreads();
    if (DOTS && z >= 1 && S.n_ent > 0) dot_phase<T>(S, sm_out + ((z - 1) & 1) * n2, z - 1, n, tab);
    if (z == n) break;
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
        double vnl = 0.0;
#pragma unroll
        for (int w = 0; w < 4; w++) {
          uint32_t m = mask[c][w];
          while (m) {
            const int e = w * 32 + __ffs(m) - 1;
            m &= m - 1;
            if (z < S.e_z0[e] || z > S.e_z1[e]) continue;
            const int Sd = S.e_S[e];
            const T *U = tab + S.e_tab[e] + S.e_base[e] + (z * Sd + cy[c]) * Sd + cx[c];
            const int pb = S.e_pb[e], np = S.e_np[e], nb = S.e_nb[e];
            for (int q = 0; q < np; q++) vnl += S.p_cur[pb + q] * (double)U[(long long)q * nb];
          }
        }
        hv = -0.5 * temp + (double)q_ve[c] * v + vnl;
      }
      T o = T(0);
      if constexpr (PK == PK_ONES) {
        o = T(1);
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
      }
      if constexpr (DOTS) smo[col[c]] = o;
      if (col[c] == centre_col && z == a.nloc) S.center_val = (double)o;
      if (!isfinite((double)o)) atomicOr(a.status, ST_NONFINITE);
    }
    // advance the register windows and prefetch the next plane's operands
#pragma unroll
    for (int c = 0; c < C; c++) {
      if constexpr (STENCIL) {
#pragma unroll
        for (int s = 0; s < 2 * FDN; s++) win[c][s] = win[c][s + 1];
        win[c][2 * FDN] = pf[c];
        pf[c] = ld_in(c, z + FDN + 2);
      }
      ld_point(c, z + 1);
    }
  }
  __syncthreads();
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
        S.e_nb[pos] = Sd * Sd * Sd;
        S.e_base[pos] = (oz - knn + nlocc) * Sd * Sd + (oy - jnn + nlocc) * Sd + (ox - inn + nlocc);
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
  __syncthreads();
}

template <int C>
__device__ void column_masks(const NodeArgs &a, NodeShared &S, uint32_t (&mask)[C][4]) {
  const int n = a.n, n2 = n * n;
#pragma unroll
  for (int c = 0; c < C; c++) {
    const int col = threadIdx.x + c * blockDim.x;
    const int x = col % n, y = col / n;
#pragma unroll
    for (int w = 0; w < 4; w++) mask[c][w] = 0u;
    if (col >= n2) continue;
    for (int e = 0; e < S.n_ent; e++)
      if (x >= S.e_x0[e] && x <= S.e_x1[e] && y >= S.e_y0[e] && y <= S.e_y1[e]) mask[c][e >> 5] |= 1u << (e & 31);
  }
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

// Lanczos bounds (FP64), sq.cpp:965-1092.
template <int C>
__device__ void lanczos(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const uint32_t (&mask)[C][4],
                        double &lmin_out, double &lmax_out, int &iters) {
  const double nw = (double)a.n * a.n * a.n;
  double *B[3] = {slot<double>(a, 0), slot<double>(a, 1), slot<double>(a, 2)};
  double s[3] = {1.0, 1.0, 1.0};
  double d0 = 0.0, d1 = 0.0;
  // v0 = 1/||1|| (sq.cpp:538-546, 993-1004)
  {
    PassIO<double> io;
    io.out = B[0];
    pass<double, C, PK_ONES>(a, S, dyn, io, mask, d0, d1);
    s[0] = 1.0 / sqrt(nw);
    rotate_proj(S, s[0]);
  }
  {
    PassIO<double> io;
    io.vin = B[0];
    io.sin = s[0];
    io.out = B[1];
    d0 = 0.0;
    pass<double, C, PK_HV>(a, S, dyn, io, mask, d0, d1);
    block_sum3(S, d0, 0.0, 0.0);
    if (threadIdx.x == 0) S.aa[0] = S.scal[0];
    __syncthreads();
  }
  {
    PassIO<double> io;
    io.vin = B[0];
    io.sin = s[0];
    io.p1 = B[1];
    io.p2 = B[0];
    io.s2 = 0.0;
    io.out = B[1];
    io.ca = S.aa[0];
    io.cb = 0.0;
    d0 = 0.0;
    pass<double, C, PK_LZB>(a, S, dyn, io, mask, d0, d1);
    block_sum3(S, d0, 0.0, 0.0);
    if (threadIdx.x == 0) S.bb[0] = sqrt(S.scal[0]);
    __syncthreads();
    s[1] = 1.0 / S.bb[0];
    rotate_proj(S, s[1]);
  }
  int P = 0, Q = 1, R = 2;
  double lmin_prev = 0.0, lmax_prev = 0.0;
  if (threadIdx.x == 0) {
    S.count = 0;
    S.stop = 0;
  }
  __syncthreads();
  int passes = 3;
  while (true) {
    const int cnt = S.count;
    {
      PassIO<double> io;
      io.vin = B[Q];
      io.sin = s[Q];
      io.out = B[R];
      d0 = 0.0;
      pass<double, C, PK_HV>(a, S, dyn, io, mask, d0, d1);
      block_sum3(S, d0, 0.0, 0.0);
      if (threadIdx.x == 0) S.aa[cnt + 1] = S.scal[0];
      __syncthreads();
    }
    {
      PassIO<double> io;
      io.vin = B[Q];
      io.sin = s[Q];
      io.p1 = B[R];
      io.p2 = B[P];
      io.s2 = s[P];
      io.out = B[R];
      io.ca = S.aa[cnt + 1];
      io.cb = S.bb[cnt];
      d0 = 0.0;
      pass<double, C, PK_LZB>(a, S, dyn, io, mask, d0, d1);
      block_sum3(S, d0, 0.0, 0.0);
      if (threadIdx.x == 0) S.bb[cnt + 1] = sqrt(S.scal[0]);
      __syncthreads();
      s[R] = 1.0 / S.bb[cnt + 1];
      rotate_proj(S, s[R]);
    }
    passes += 2;
    const int t = P;
    P = Q;
    Q = R;
    R = t;
    tridiag_extremes(S, cnt + 2);
    __syncthreads();
    if (threadIdx.x == 0) {
      const double lmin = S.eig[0], lmax = S.eig[1];
      const double dl = fabs(lmin - lmin_prev), dm = fabs(lmax - lmax_prev);
      lmin_prev = lmin;
      lmax_prev = lmax;
      S.count = cnt + 1;
      S.stop = !(S.count < LANCZOS_MAX_ITER && (dl > a.lanczos_tol || dm > a.lanczos_tol));
      if (S.count >= LANCZOS_MAX_ITER) atomicOr(a.status, ST_LANCZOS_MAXITER);
      S.scal[3] = lmin;
      S.eig[0] = lmin;
      S.eig[1] = lmax;
    }
    __syncthreads();
    if (S.stop) break;
  }
  lmin_out = S.eig[0] - a.lanczos_tol;
  lmax_out = S.eig[1] + a.lanczos_tol;
  iters = S.count;
  count_proj_points(a, S, S.count + 1, 0);  // Lanczos: iterations + the first matvec
}

// Chebyshev moments (sq.cpp:564-655) in precision T.
template <typename T, int C>
__device__ void moments(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const uint32_t (&mask)[C][4],
                        double chi, double zee, double *mu) {
  T *B0 = slot<T>(a, 0), *B1 = slot<T>(a, 1);
  double d0 = 0.0, d1 = 0.0;
  {
    PassIO<T> io;
    io.out = B0;
    pass<T, C, PK_DELTA>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
  }
  {
    PassIO<T> io;
    io.vin = B0;
    io.out = B1;
    io.ca = chi;
    io.cb = zee;
    pass<T, C, PK_CH1>(a, S, dyn, io, mask, d0, d1);
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
    pass<T, C, PK_CH>(a, S, dyn, io, mask, d0, d1);
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
__device__ void node_forces(const NodeArgs &a, NodeShared &S, unsigned char *dyn, const uint32_t (&mask)[C][4],
                            double chi, double zee, const double *ci, double *fslot) {
  T *B0 = slot<T>(a, 0), *B1 = slot<T>(a, 1);
  double *D = slot<double>(a, 3);
  double d0 = 0.0, d1 = 0.0;
  {
    PassIO<T> io;
    io.out = B0;
    pass<T, C, PK_DELTA>(a, S, dyn, io, mask, d0, d1);
    rotate_proj(S, 1.0);
  }
  {
    PassIO<T> io;
    io.vin = B0;
    io.out = B1;
    io.ca = chi;
    io.cb = zee;
    pass<T, C, PK_CH1>(a, S, dyn, io, mask, d0, d1);
  }
  {
    PassIO<T> io;
    io.p1 = B0;
    io.p2 = B1;
    io.dacc = D;
    io.cd = ci[0];
    io.ce = ci[1];
    pass<T, C, PK_FD01>(a, S, dyn, io, mask, d0, d1);
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
    pass<T, C, PK_FD>(a, S, dyn, io, mask, d0, d1);
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
    const int Sd = S.e_S[e], vol = bx * by * bz;
    const double *U = a.at.tab64 + S.e_tab[e] + S.e_base[e];
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
        const double u = U[(long long)q * S.e_nb[e] + (z * Sd + y) * Sd + x];
        ax += u * gx;
        ay += u * gy;
        az += u * gz;
      }
      block_sum3(S, ax, ay, az);
      const double uc = U[(long long)q * S.e_nb[e] + (nl * Sd + nl) * Sd + nl];
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

template <int C>
__global__ void __launch_bounds__(C == 1 ? 1024 : 576, 1) node_kernel(NodeArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  NodeShared &S = *reinterpret_cast<NodeShared *>(smem);
  unsigned char *dyn = smem + kSharedFixed;
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
    uint32_t mask[C][4];
    column_masks<C>(a, S, mask);
    if (a.mode == MODE_SQ) {
      double lmin, lmax;
      int iters;
      lanczos<C>(a, S, dyn, mask, lmin, lmax, iters);
      const double chi = (lmax + lmin) / 2, zee = (lmax - lmin) / 2;  // sq.cpp:564-565
      double *mu = a.rho_pj + (size_t)node * (a.npl + 1);
      if (a.mixed) moments<float, C>(a, S, dyn, mask, chi, zee, mu);
      else moments<double, C>(a, S, dyn, mask, chi, zee, mu);
      if (threadIdx.x == 0) {
        a.chi[node] = chi;
        a.zee[node] = zee;
        if (a.lmin) a.lmin[node] = lmin;
        if (a.lmax) a.lmax[node] = lmax;
        if (a.lanczos_iters) a.lanczos_iters[node] = iters;
      }
    } else if (a.mode == MODE_FORCES) {
      double *fs = a.fslots + (size_t)S.qidx * FSLOTS * 4;
      for (int i = threadIdx.x; i < FSLOTS * 4; i += blockDim.x) fs[i] = (i % 4 == 0) ? -1.0 : 0.0;
      __syncthreads();
      const double *ci = a.ci + (size_t)node * (a.npl + 1);
      if (a.mixed) node_forces<float, C>(a, S, dyn, mask, a.chi_in[node], a.zee_in[node], ci, fs);
      else node_forces<double, C>(a, S, dyn, mask, a.chi_in[node], a.zee_in[node], ci, fs);
    } else {
      const size_t nw = (size_t)a.n * a.n * a.n;
      double d0 = 0.0, d1 = 0.0;
      PassIO<double> io;
      io.din = a.apply_in + (size_t)S.qidx * nw;
      pass<double, C, PK_DOTS>(a, S, dyn, io, mask, d0, d1);
      rotate_proj(S, 1.0);
      io.dout = a.apply_out + (size_t)S.qidx * nw;
      pass<double, C, PK_APPLY>(a, S, dyn, io, mask, d0, d1);
    }
    __syncthreads();
  }
}

}  // namespace

int node_kernel_threads(int n, int cols) {
  const int per = (n * n + cols - 1) / cols;
  return ((per + 31) / 32) * 32;
}

size_t node_kernel_smem(int n, int cols) {
  (void)cols;
  const int P = n + 2 * FDN;
  return kSharedFixed + sizeof(double) * (size_t)(2 * P * P + 2 * n * n);
}

cudaError_t node_kernel_setup(int n) {
  cudaError_t e1 = cudaFuncSetAttribute(node_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)node_kernel_smem(n, 1));
  cudaError_t e2 = cudaFuncSetAttribute(node_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)node_kernel_smem(n, 2));
  return e1 != cudaSuccess ? e1 : e2;
}

cudaError_t launch_node_kernel(const NodeArgs &a, int grid, int cols, cudaStream_t s) {
  const int threads = node_kernel_threads(a.n, cols);
  const size_t smem = node_kernel_smem(a.n, cols);
  if (threads > 1024 || threads < 64) return cudaErrorInvalidConfiguration;
  if (cols == 1) node_kernel<1><<<grid, threads, smem, s>>>(a);
  else if (cols == 2) node_kernel<2><<<grid, threads, smem, s>>>(a);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

}  // namespace sqb
