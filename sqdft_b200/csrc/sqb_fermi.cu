// Per-node Chebyshev-coefficient kernels (Fermi-level constraint and density /
// energy assembly), the nonlocal-force reduction and the projector tables.
#include <cmath>

#include "sqb_internal.cuh"

namespace sqb {

namespace {

constexpr int FW = 32;         // warps per block: one node per warp
constexpr int FTHREADS = FW * 32;
constexpr double TEMP_TOL = 1e-12;

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order block sum of two values; result valid in thread 0.
__device__ void bsum2(double &a, double &b, double (*red)[2]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = wsum(a);
  b = wsum(b);
  if (lane == 0) {
    red[w][0] = a;
    red[w][1] = b;
  }
  __syncthreads();
  if (w == 0) {
    a = lane < (int)(blockDim.x >> 5) ? red[lane][0] : 0.0;
    b = lane < (int)(blockDim.x >> 5) ? red[lane][1] : 0.0;
    a = wsum(a);
    b = wsum(b);
  }
  __syncthreads();
}

// The cos table (npl+1)^2 is staged in shared memory when it fits.
__device__ __forceinline__ const double *stage_table(const double *g, double *s, int K, bool fits) {
  if (!fits) return g;
  for (int i = threadIdx.x; i < K * K; i += blockDim.x) s[i] = g[i];
  __syncthreads();
  return s;
}

// ChebyshevCoeff (sq.cpp:1230-1259) for one node on one warp: c_j =
// 2/(npl+1) sum_k d_k cos(pi j (k+1/2)/(npl+1)), c_0 halved; d_k in dk.
__device__ __forceinline__ double cheb_coeff(const double *dk, const double *ctab, int K, int j) {
  double sum = 0.0;
  const double *row = ctab + (size_t)j * K;
  for (int k = 0; k < K; k++) sum = sum + dk[k] * row[k];
  double c = (2.0 / K) * sum;
  if (j == 0) c = c / 2.0;
  return c;
}

// NeConstraint (sq.cpp:1183-1228) and, with deriv, NeConstraint_derv
// (sq.cpp:1407-1449): per-block partial sums of 2 rho_pj . c.
__global__ void __launch_bounds__(FTHREADS) ne_kernel(FermiArgs a, double lambda_arg, int deriv, int fits) {
  const double lambda = a.lam_dev ? *a.lam_dev : lambda_arg;
  extern __shared__ __align__(16) double fsm[];
  __shared__ double red[FW][2];
  const int K = a.npl + 1;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *dk = fsm + (fits ? K * K : 0) + (size_t)w * 2 * K;
  const double *ctab = stage_table(a.ctab, fsm, K, fits);
  double g = 0.0, dg = 0.0;
  for (int node = blockIdx.x * FW + w; node < a.n_nodes; node += gridDim.x * FW) {
    const double zee = a.zee[node];
    const double lambda_fp = (lambda - a.chi[node]) / zee;
    const double bet = a.bet0 * zee;
    for (int k = lane; k < K; k += 32) {
      const double f = 1 / (1 + exp(bet * (a.xk[k] - lambda_fp)));  // FermiDirac, sq.cpp:1261
      dk[k] = f;
      dk[K + k] = f * (1 - f);  // FermiDirac_derv, sq.cpp:1451
    }
    __syncwarp();
    const double *mu = a.rho_pj + (size_t)node * K;
    for (int j = lane; j < K; j += 32) {
      g = g + 2 * mu[j] * cheb_coeff(dk, ctab, K, j);
      if (deriv) dg = dg + 2 * mu[j] * cheb_coeff(dk + K, ctab, K, j);
    }
    __syncwarp();
  }
  bsum2(g, dg, red);
  if (threadIdx.x == 0) {
    a.partial[2 * blockIdx.x] = g;
    a.partial[2 * blockIdx.x + 1] = dg;
  }
}

// Density of a node at bounds (chi', zee') from its moments at (chi, zee).
// T_j((H - chi')/zee') = T_j(al Ht + be) with Ht = (H - chi)/zee, al = zee/zee',
// be = (chi - chi')/zee', is a degree-j polynomial in Ht: its coefficients P_j
// in the T_m(Ht) follow from P_j+1 = 2 (al X + be) P_j - P_j-1, X the product
// by x in the Chebyshev basis (x T_0 = T_1, x T_m = (T_m+1 + T_m-1)/2), so the
// moments at the new bounds are P_j . mu, exactly, with no new matvec.  The
// density is then |2 sum_j c'_j mu'_j| with the coefficients of sq.cpp:1230-1259
// on the new interval (sq.cpp:743-797).  One warp; buffers in w: 4K doubles.
__device__ double rho_at_bounds(const FermiArgs &a, const double *mu, double chi, double zee, double chi2,
                                double zee2, double lambda, const double *ctab, double *w) {
  const int K = a.npl + 1, lane = threadIdx.x & 31;
  double *pm = w, *pc = w + K, *pn = w + 2 * K, *mu2 = w + 3 * K;
  const double al = zee / zee2, be = (chi - chi2) / zee2;
  for (int m = lane; m < K; m += 32) {
    pm[m] = m == 0 ? 1.0 : 0.0;
    pc[m] = m == 0 ? be : (m == 1 ? al : 0.0);
  }
  __syncwarp();
  if (lane == 0) {
    mu2[0] = mu[0];
    mu2[1] = al * mu[1] + be * mu[0];
  }
  for (int j = 1; j < a.npl; j++) {
    double acc = 0.0;
    for (int m = lane; m < K; m += 32) {
      const double up = m + 1 < K ? pc[m + 1] : 0.0;
      const double xp = m == 0 ? 0.5 * up : (m == 1 ? pc[0] + 0.5 * up : 0.5 * (pc[m - 1] + up));
      const double v = 2.0 * (al * xp + be * pc[m]) - pm[m];
      pn[m] = v;
      acc += v * mu[m];
    }
    acc = wsum(acc);
    __syncwarp();
    if (lane == 0) mu2[j + 1] = acc;
    double *t = pm;
    pm = pc;
    pc = pn;
    pn = t;
    __syncwarp();
  }
  // Fermi-Dirac values on the new interval (pn is free), then 2 c' . mu'
  const double lambda_fp = (lambda - chi2) / zee2, bet = a.bet0 * zee2;
  for (int k = lane; k < K; k += 32) pn[k] = 1 / (1 + exp(bet * (a.xk[k] - lambda_fp)));
  __syncwarp();
  double r = 0.0;
  for (int j = lane; j < K; j += 32) r += 2 * mu2[j] * cheb_coeff(pn, ctab, K, j);
  r = wsum(r);
  __syncwarp();
  return fabs(r);
}

// Sensitivity of every node's density to its bounds: rho at bounds with the
// lower end moved down by delta and, separately, the upper end moved up by
// delta, against rho at the node's bounds; sens = the sum of the two changes.
__global__ void __launch_bounds__(256) bound_sens_kernel(FermiArgs a, double lambda, double delta, double *sens,
                                                         double *rho0) {
  extern __shared__ __align__(16) double bsm[];
  const int K = a.npl + 1;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double *buf = bsm + (size_t)w * 4 * K;
  for (int node = blockIdx.x * nw + w; node < a.n_nodes; node += gridDim.x * nw) {
    const double chi = a.chi[node], zee = a.zee[node];
    const double *mu = a.rho_pj + (size_t)node * K;
    const double r0 = rho_at_bounds(a, mu, chi, zee, chi, zee, lambda, a.ctab, buf);
    const double rlo = rho_at_bounds(a, mu, chi, zee, chi - 0.5 * delta, zee + 0.5 * delta, lambda, a.ctab, buf);
    const double rhi = rho_at_bounds(a, mu, chi, zee, chi + 0.5 * delta, zee + 0.5 * delta, lambda, a.ctab, buf);
    if (lane == 0) {
      sens[node] = fabs(rlo - r0) + fabs(rhi - r0);
      rho0[node] = r0;
    }
  }
}

// Adjoint of a density loss L = sum_p w_p rho_p, rho_p = |2 c(lambda) . mu_p|
// (sq.cpp:743-797), the bounds held fixed: per node the sign s_p of 2 c . mu_p
// into sgn and, with a fixed electron count, the density's derivative with
// respect to the Fermi level, drho_p/dlambda = 2 s_p dc/dlambda . mu_p, where
// dc/dlambda are the Chebyshev coefficients (ChebyshevCoeff, sq.cpp:1230-1259)
// of d f/d lambda = beta f (1 - f) on the node's interval; block partials of
// sum_p w_p drho_p/dlambda and sum_p drho_p/dlambda.  One warp per node.
__global__ void __launch_bounds__(FTHREADS) loss_lambda_kernel(FermiArgs a, double lambda, const double *w,
                                                               int fixed, double *sgn, int fits) {
  extern __shared__ __align__(16) double fsm[];
  __shared__ double red[FW][2];
  const int K = a.npl + 1;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  double *dk = fsm + (fits ? K * K : 0) + (size_t)wp * K;
  const double *ctab = stage_table(a.ctab, fsm, K, fits);
  double pw = 0.0, pn = 0.0;
  for (int node = blockIdx.x * FW + wp; node < a.n_nodes; node += gridDim.x * FW) {
    const double *mu = a.rho_pj + (size_t)node * K;
    const double *ci = a.ci + (size_t)node * K;
    double r = 0.0;
    for (int j = lane; j < K; j += 32) r = r + 2 * mu[j] * ci[j];
    r = wsum(r);
    const double sg = (double)((r > 0.0) - (r < 0.0));
    if (fixed) {
      const double zee = a.zee[node], chi = a.chi[node];
      const double lambda_fp = (lambda - chi) / zee, bet = a.bet0 * zee;
      for (int k = lane; k < K; k += 32) {
        const double f = 1 / (1 + exp(bet * (a.xk[k] - lambda_fp)));
        dk[k] = a.bet0 * f * (1 - f);
      }
      __syncwarp();
      double d = 0.0;
      for (int j = lane; j < K; j += 32) d = d + 2 * mu[j] * cheb_coeff(dk, ctab, K, j);
      d = wsum(d) * sg;
      if (lane == 0) {
        pw += w[node] * d;
        pn += d;
      }
      __syncwarp();
    }
    if (lane == 0) sgn[node] = sg;
  }
  bsum2(pw, pn, red);
  if (threadIdx.x == 0) {
    a.partial[2 * blockIdx.x] = pw;
    a.partial[2 * blockIdx.x + 1] = pn;
  }
}

// Moment weights of the loss: g[p][j] = scale (w_p - off) s_p Ci[p][j].
__global__ void loss_gmu_kernel(int n, int K, const double *ci, const double *w, const double *sgn, double scale,
                                double off, double *g) {
  const long long total = (long long)n * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(i / K);
    g[i] = scale * (w[p] - off) * sgn[p] * ci[i];
  }
}

__global__ void sum_partials(const double *partial, int nblocks, int width, double *out) {
  __shared__ double red[32][2];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  // Each thread sums a contiguous run so the order does not depend on timing.
  const int per = (nblocks + blockDim.x - 1) / blockDim.x;
  for (int b = threadIdx.x * per; b < min(nblocks, (int)(threadIdx.x + 1) * per); b++) {
    s0 += partial[(size_t)width * b];
    if (width > 1) s1 += partial[(size_t)width * b + 1];
    if (width > 2) s2 += partial[(size_t)width * b + 2];
  }
  bsum2(s0, s1, red);
  double z = 0.0;
  bsum2(s2, z, red);
  if (threadIdx.x == 0) {
    out[0] = s0;
    if (width > 1) out[1] = s1;
    if (width > 2) out[2] = s2;
  }
}

// Density and energies (sq.cpp:733-797): Ci (FermiDirac), rho = |2 mu.c|,
// Ebs and Eent partial sums.
__global__ void __launch_bounds__(FTHREADS) density_kernel(FermiArgs a, double lambda_arg, int fits) {
  const double lambda = a.lam_dev ? *a.lam_dev : lambda_arg;
  extern __shared__ __align__(16) double fsm[];
  __shared__ double red[FW][2];
  const int K = a.npl + 1;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *dk = fsm + (fits ? K * K : 0) + (size_t)w * 3 * K;
  const double *ctab = stage_table(a.ctab, fsm, K, fits);
  double ebs_sum = 0.0, ent_sum = 0.0;
  for (int node = blockIdx.x * FW + w; node < a.n_nodes; node += gridDim.x * FW) {
    const double zee = a.zee[node], chi = a.chi[node];
    const double lambda_fp = (lambda - chi) / zee;
    const double bet = a.bet0 * zee;
    for (int k = lane; k < K; k += 32) {
      const double t = a.xk[k];
      const double focc = (1 / (1 + exp(bet * (t - lambda_fp))));
      dk[k] = focc;                                                    // FermiDirac
      dk[K + k] = t * (1 / (1 + exp(bet * (t - lambda_fp))));          // UbandFunc, sq.cpp:1268
      double v;                                                        // EentFunc, sq.cpp:1275
      if (fabs(focc) < 0.01 * TEMP_TOL || fabs(focc - 1.0) < 0.01 * TEMP_TOL) v = 0.0;
      else v = (focc * log(focc) + (1 - focc) * log(1 - focc));
      dk[2 * K + k] = v;
    }
    __syncwarp();
    const double *mu = a.rho_pj + (size_t)node * K;
    double r = 0.0, e = 0.0, s = 0.0;
    for (int j = lane; j < K; j += 32) {
      const double c = cheb_coeff(dk, ctab, K, j);
      a.ci[(size_t)node * K + j] = c;
      r = r + 2 * mu[j] * c;
      e = e + 2 * mu[j] * cheb_coeff(dk + K, ctab, K, j);
      s = s + 2 * mu[j] * cheb_coeff(dk + 2 * K, ctab, K, j);
    }
    r = wsum(r);
    e = wsum(e);
    s = wsum(s);
    if (lane == 0) {
      a.rho[node] = fabs(r);
      if (r < 0 && fabs(r) > 1e-6) atomicOr(a.status, 1);
      if (!isfinite(r)) atomicOr(a.status, 2);
      ebs_sum += (zee * e + chi * r) * a.h3;
      ent_sum += (1 / a.bet0) * s * a.h3;
    }
    __syncwarp();
  }
  bsum2(ebs_sum, ent_sum, red);
  if (threadIdx.x == 0) {
    a.partial[2 * blockIdx.x] = ebs_sum;
    a.partial[2 * blockIdx.x + 1] = ent_sum;
  }
}

// Nonlocal forces: sum the per-node contributions of each atom in node order.
__global__ void force_reduce_kernel(const double *fslots, int n_list, int n_atm, double *f) {
  __shared__ double red[32][2];
  const int atom = blockIdx.x;
  if (atom >= n_atm) return;
  const long long total = (long long)n_list * FSLOTS;
  const long long per = (total + blockDim.x - 1) / blockDim.x;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (long long i = threadIdx.x * per; i < min(total, (threadIdx.x + 1) * per); i++) {
    const double *s = fslots + 4 * i;
    if ((int)s[0] == atom) {
      fx += s[1];
      fy += s[2];
      fz += s[3];
    }
  }
  bsum2(fx, fy, red);
  double z = 0.0;
  bsum2(fz, z, red);
  if (threadIdx.x == 0) {
    f[3 * atom] = fx;
    f[3 * atom + 1] = fy;
    f[3 * atom + 2] = fz;
  }
}

// Cubic spline of spline.cpp:11-55 at one radius (interval found by binary
// search: the first grid point >= r, stepped back unless equal).
__device__ bool spline_eval(const double *X, const double *Y, const double *YD, int len, double x, double &out) {
  if (!(x >= X[0] && x <= X[len - 1])) return false;
  int lo = 0, hi = len - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (X[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  int j = lo;
  if (x < X[j]) j--;
  if (j > len - 2) j = len - 2;
  if (j < 0) j = 0;
  const double p1 = X[j];
  const double dx = 1.0 / (X[j + 1] - X[j]);
  const double dy = (Y[j + 1] - Y[j]) * dx;
  const double A0 = Y[j], A1 = YD[j];
  const double A2 = dx * (3.0 * dy - 2.0 * YD[j] - YD[j + 1]);
  const double A3 = dx * dx * (-2.0 * dy + YD[j] + YD[j + 1]);
  const double t = x - p1;
  out = ((A3 * t + A2) * t + A1) * t + A0;
  return true;
}

// Real spherical harmonics of nonlocal.cpp:218-314 (same normalisation constants).
__device__ double real_sh(double x, double y, double z, double r, int l, int m) {
  const double C00 = 0.282094791773878, C1 = 0.488602511902920;
  const double C2m2 = 1.092548430592079, C20 = 0.315391565252520, C2p2 = 0.546274215296040;
  const double C3m3 = 0.590043589926644, C3m2 = 2.890611442640554, C3m1 = 0.457045799464466;
  const double C30 = 0.373176332590115, C3p2 = 1.445305721320277;
  double SH = 0.0;
  if (l == 0) SH = C00;
  if (fabs(r) > TEMP_TOL) {
    if (l == 0) SH = C00;
    else if (l == 1) SH = m == -1 ? C1 * (y / r) : m == 0 ? C1 * (z / r) : C1 * (x / r);
    else if (l == 2) {
      if (m == -2) SH = C2m2 * (x * y) / (r * r);
      else if (m == -1) SH = C2m2 * (y * z) / (r * r);
      else if (m == 0) SH = C20 * (-x * x - y * y + 2 * z * z) / (r * r);
      else if (m == 1) SH = C2m2 * (z * x) / (r * r);
      else SH = C2p2 * (x * x - y * y) / (r * r);
    } else {
      if (m == -3) SH = C3m3 * (3 * x * x - y * y) * y / (r * r * r);
      else if (m == -2) SH = C3m2 * (x * y * z) / (r * r * r);
      else if (m == -1) SH = C3m1 * y * (4 * z * z - x * x - y * y) / (r * r * r);
      else if (m == 0) SH = C30 * z * (2 * z * z - 3 * x * x - 3 * y * y) / (r * r * r);
      else if (m == 1) SH = C3m1 * x * (4 * z * z - x * x - y * y) / (r * r * r);
      else if (m == 2) SH = C3p2 * z * (x * x - y * y) / (r * r * r);
      else SH = C3m3 * x * (x * x - 3 * y * y) / (r * r * r);
    }
  }
  return SH;
}

// NonlocalProjectors (nonlocal.cpp:317-518): blockIdx.y = replica,
// blockIdx.z = projector (l,m), threads over the ball points.
__global__ void proj_kernel(ProjArgs a) {
  const int r = blockIdx.y, q = blockIdx.z;
  const int t = a.rep_nn[4 * r + 3];
  const int nlocc = a.typ_nlocc[t], lmax = a.typ_lmax[t], lloc = a.typ_lloc[t], len = a.typ_size[t];
  int l = -1, m = 0, cnt = 0;
  for (int ll = 0; ll <= lmax && l < 0; ll++) {
    if (ll == lloc) continue;
    if (q < cnt + 2 * ll + 1) {
      l = ll;
      m = q - cnt - ll;
    }
    cnt += 2 * ll + 1;
  }
  if (l < 0) return;
  const int Sd = 2 * nlocc + 1, nnd = Sd * Sd * Sd;
  const double *G = a.tables + a.typ_tab[t];
  const double *rVloc = G + len, *DVloc = G + 10 * (size_t)len;
  const double *rV = G + (size_t)(2 + l) * len, *rU = G + (size_t)(6 + l) * len;
  const double *DV = G + (size_t)(11 + l) * len, *DU = G + (size_t)(15 + l) * len;
  const int inn = a.rep_nn[4 * r], jnn = a.rep_nn[4 * r + 1], knn = a.rep_nn[4 * r + 2];
  const double ax = a.rep_xyz[3 * r], ay = a.rep_xyz[3 * r + 1], az = a.rep_xyz[3 * r + 2];
  for (int ctr = blockIdx.x * blockDim.x + threadIdx.x; ctr < nnd; ctr += gridDim.x * blockDim.x) {
    const int ii = ctr % Sd - nlocc, jj = (ctr / Sd) % Sd - nlocc, kk = ctr / (Sd * Sd) - nlocc;
    const double xr = (inn + ii) * a.delta - ax, yr = (jnn + jj) * a.delta - ay, zr = (knn + kk) * a.delta - az;
    const double rad = sqrt(xr * xr + yr * yr + zr * zr);
    double VlocJ, VlJ, UlJ;
    if (!spline_eval(G, rVloc, DVloc, len, rad, VlocJ) || !spline_eval(G, rV, DV, len, rad, VlJ) ||
        !spline_eval(G, rU, DU, len, rad, UlJ)) {
      atomicOr(a.status, ST_SPLINE_RANGE);
      continue;
    }
    if (fabs(rad - 0.0) < TEMP_TOL) {
      VlocJ = rVloc[1] / G[1];
      VlJ = rV[1] / G[1];
      UlJ = rU[1] / G[1];
    } else {
      VlocJ = VlocJ / rad;
      VlJ = VlJ / rad;
      UlJ = UlJ / rad;
    }
    const double u = UlJ * real_sh(xr, yr, zr, rad, l, m) * (VlJ - VlocJ);
    const long long o = a.rep_off[r] + ((long long)q * Sd + ctr / (Sd * Sd)) * plane_stride(Sd) + ctr % (Sd * Sd);
    a.out64[o] = u;
  }
}

// Global Lanczos extremes of the block (the min/max over nodes taken before
// the Allgather of sq.cpp:676-713).
__global__ void minmax_kernel(const double *lmin, const double *lmax, int n, double *out) {
  __shared__ double smin[32], smax[32];
  double a = 1e300, b = -1e300;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    a = fmin(a, lmin[i]);
    b = fmax(b, lmax[i]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    smin[w] = a;
    smax[w] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
      a = fmin(a, smin[k]);
      b = fmax(b, smax[k]);
    }
    out[0] = fmin(a, smin[0]);
    out[1] = fmax(b, smax[0]);
  }
}

// Tables between the reference's UdVtm layout [rep][q][Sd^3] and the padded
// device layout (blockIdx.y = replica).
__global__ void repack_kernel(const int *rep_nn, const int *typ_nlocc, const int *typ_nproj, const long long *off_ref,
                              const long long *off_pad, const double *in, double *out, int to_pad) {
  const int r = blockIdx.y, t = rep_nn[4 * r + 3];
  const int Sd = 2 * typ_nlocc[t] + 1, sp2 = plane_stride(Sd), S2 = Sd * Sd;
  const long long cnt = (long long)typ_nproj[t] * Sd * S2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    const long long ir = off_ref[r] + i, ip = off_pad[r] + (i / S2) * sp2 + i % S2;
    if (to_pad) out[ip] = in[ir];
    else out[ir] = in[ip];
  }
}

// (plus - minus) * scale, element-wise (central differences of tables).
__global__ void fd_combine_kernel(const double *plus, const double *minus, double *out, long long n, double scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (plus[i] - minus[i]) * scale;
}

size_t fermi_smem(int K, int per_warp, bool &fits) {
  const size_t base = (size_t)FW * per_warp * K * sizeof(double);
  const size_t tab = (size_t)K * K * sizeof(double);
  fits = base + tab <= 200 * 1024;
  return base + (fits ? tab : 0);
}

}  // namespace

int fermi_blocks(int n_nodes) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int need = (n_nodes + FW - 1) / FW;
  return need < sms ? need : sms;
}

cudaError_t launch_ne_constraint(const FermiArgs &a, double lambda, int with_derivative, cudaStream_t s) {
  bool fits;
  const size_t smem = fermi_smem(a.npl + 1, 2, fits);
  cudaFuncSetAttribute(ne_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int nb = fermi_blocks(a.n_nodes);
  ne_kernel<<<nb, FTHREADS, smem, s>>>(a, lambda, with_derivative, fits ? 1 : 0);
  sum_partials<<<1, 1024, 0, s>>>(a.partial, nb, 2, a.result);
  return cudaGetLastError();
}

cudaError_t launch_density_energy(const FermiArgs &a, double lambda, cudaStream_t s) {
  bool fits;
  const size_t smem = fermi_smem(a.npl + 1, 3, fits);
  cudaFuncSetAttribute(density_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int nb = fermi_blocks(a.n_nodes);
  density_kernel<<<nb, FTHREADS, smem, s>>>(a, lambda, fits ? 1 : 0);
  sum_partials<<<1, 1024, 0, s>>>(a.partial, nb, 2, a.result);
  return cudaGetLastError();
}

cudaError_t launch_loss_lambda(const FermiArgs &a, double lambda, const double *w, int fixed, double *sgn,
                               cudaStream_t s) {
  bool fits;
  const size_t smem = fermi_smem(a.npl + 1, 1, fits);
  cudaFuncSetAttribute(loss_lambda_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int nb = fermi_blocks(a.n_nodes);
  loss_lambda_kernel<<<nb, FTHREADS, smem, s>>>(a, lambda, w, fixed, sgn, fits ? 1 : 0);
  sum_partials<<<1, 1024, 0, s>>>(a.partial, nb, 2, a.result);
  return cudaGetLastError();
}

cudaError_t launch_loss_gmu(int n, int K, const double *ci, const double *w, const double *sgn, double scale,
                            double off, double *g, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  loss_gmu_kernel<<<592, 256, 0, s>>>(n, K, ci, w, sgn, scale, off, g);
  return cudaGetLastError();
}

cudaError_t launch_bound_sens(const FermiArgs &a, double lambda, double delta, double *sens, double *rho0,
                              cudaStream_t s) {
  if (a.n_nodes <= 0) return cudaSuccess;
  const size_t per_warp = (size_t)4 * (a.npl + 1) * sizeof(double);
  int warps = 8;
  while (warps > 1 && per_warp * warps > 48 * 1024) warps--;
  if (per_warp * warps > 48 * 1024) return cudaErrorInvalidValue;
  int blocks = (a.n_nodes + warps - 1) / warps;
  if (blocks > 4096) blocks = 4096;
  bound_sens_kernel<<<blocks, 32 * warps, per_warp * warps, s>>>(a, lambda, delta, sens, rho0);
  return cudaGetLastError();
}

cudaError_t launch_force_reduce(const double *fslots, int n_list, int n_atm, double *f, cudaStream_t s) {
  if (n_atm <= 0) return cudaSuccess;
  force_reduce_kernel<<<n_atm, 256, 0, s>>>(fslots, n_list, n_atm, f);
  return cudaGetLastError();
}

cudaError_t launch_projectors(const ProjArgs &a, cudaStream_t s) {
  if (a.n_rep <= 0) return cudaSuccess;
  dim3 grid(8, a.n_rep, MAXPROJ_TYPE);
  proj_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_minmax(const double *lmin, const double *lmax, int n, double *out, cudaStream_t s) {
  minmax_kernel<<<1, 1024, 0, s>>>(lmin, lmax, n, out);
  return cudaGetLastError();
}

cudaError_t launch_fd_combine(const double *plus, const double *minus, double *out, long long n, double scale,
                              cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  fd_combine_kernel<<<296, 256, 0, s>>>(plus, minus, out, n, scale);
  return cudaGetLastError();
}

cudaError_t launch_repack(int n_rep, const int *rep_nn, const int *typ_nlocc, const int *typ_nproj,
                          const long long *off_ref, const long long *off_pad, const double *in, double *out,
                          int to_pad, cudaStream_t s) {
  if (n_rep <= 0) return cudaSuccess;
  dim3 grid(4, n_rep);
  repack_kernel<<<grid, 256, 0, s>>>(rep_nn, typ_nlocc, typ_nproj, off_ref, off_pad, in, out, to_pad);
  return cudaGetLastError();
}

}  // namespace sqb
