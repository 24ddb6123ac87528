// Pseudocharge density and local forces on the device: the per-atom loops of
// ChargeDensity (initialize.cpp:470-784) and ForcesLocal (forces.cpp:20-315).
//
// Every atom replica J whose rb-box meets the block contributes, on its
// intersection box, b_J = -(1/4 pi) Lap_h V_J and the same of the smooth
// reference potential V~_J, with V_J the spline of r Vloc over r.
//
// Charge density: one CTA per 8^3 tile of the block, one thread per node.
// The CTA lists the replicas that meet its tile, in the reference's loop
// order, and for each one puts V_J and V~_J on the tile and its FDN halo
// into shared memory. Each thread then adds the replica's terms to its own
// node. A node therefore sums its replicas in the reference's order, and its
// b and rho_at equal the reference's bit for bit. This translation unit is
// compiled without multiply-add contraction, as the reference's x86 build
// runs.
//
// Local forces: each replica's V_J, V~_J (box + 2 FDN) and b_J, b~_J
// (box + FDN) go into a scratch box in global memory. The contraction over
// the box is spread over LOC_FORCE_CTAS CTAs per replica, with a fixed
// reduction order.
#include "sqb_internal.cuh"

namespace sqb {

namespace {

constexpr int LT = LOC_TILE;
constexpr int LH = LT + 2 * FDN;  // halo'd tile edge
constexpr int LH3 = LH * LH * LH;
constexpr int LLIST = 512;        // replicas tested per list pass (one per thread)
constexpr double PI = 3.14159265358979323846;  // M_PI
constexpr double TOL = 1e-12;                  // TEMP_TOL of the reference

// ispline_gen (spline.cpp:11-55) at one point: the first grid point >= x,
// stepped back unless equal; false out of the table's range.
__device__ bool spline_at(const double *X, const double *Y, const double *YD, int len, double x, double &out) {
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

// Distance of global node (gi, gj, gk) from a replica (initialize.cpp:571).
__device__ __forceinline__ double node_radius(const LocalArgs &a, const double *c, int gi, int gj, int gk) {
  const double dx = gi * a.delta - c[0], dy = gj * a.delta - c[1], dz = gk * a.delta - c[2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

// VlocJ and VlocJ_tilda of a replica of type t at distance r
// (initialize.cpp:573-597, forces.cpp:126-143).
__device__ bool vloc_pair(const LocalArgs &a, int t, double r, double &v, double &vt) {
  const double *G = a.tab + a.typ_off[t];
  const int len = a.typ_size[t];
  const double *rV = G + len, *DV = G + 2 * (size_t)len;
  double s;
  if (!spline_at(G, rV, DV, len, r, s)) return false;
  v = fabs(r - 0.0) < TOL ? rV[1] / G[1] : s / r;
  const double rc = a.rc_tilda, Z = a.Z[t];
  if (r < rc)
    vt = -Z * (9 * pow(r, 7) - 30 * rc * pow(r, 6) + 28 * rc * rc * pow(r, 5) - 14 * pow(rc, 5) * pow(r, 2) +
               12 * pow(rc, 7)) /
         (5 * pow(rc, 8));
  else
    vt = -Z / r;
  return true;
}

// -(1/4 pi) Lap_h f at index q of a box with x stride 1, y stride sy and z
// stride sz (the expression of initialize.cpp:604-614, forces.cpp:154-170).
__device__ __forceinline__ double neg_lap(const LocalArgs &a, const double *f, long long q, long long sy, long long sz) {
  double s = f[q] * 3 * a.coeff_lap[0] * (-1 / (4 * PI));
#pragma unroll
  for (int k = 1; k <= FDN; k++)
    s += (f[q - k] + f[q + k] + f[q - k * sy] + f[q + k * sy] + f[q - k * sz] + f[q + k * sz]) * a.coeff_lap[k] *
         (-1 / (4 * PI));
  return s;
}

__device__ __forceinline__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
  return s;  // valid in thread 0
}

__global__ void __launch_bounds__(LT *LT *LT) charge_density_kernel(LocalArgs a) {
  extern __shared__ double sm[];
  double *sV = sm, *sVt = sm + LH3;
  __shared__ int list[LLIST];
  __shared__ int wcount[LT * LT * LT / 32 + 1];
  __shared__ int nlist;
  __shared__ double red[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const int NX = a.np[0], NY = a.np[1], NZ = a.np[2];
  const int x0 = blockIdx.x * LT, y0 = blockIdx.y * LT, z0 = blockIdx.z * LT;  // tile origin (block nodes)
  const int li = tid % LT, lj = (tid / LT) % LT, lk = tid / (LT * LT);
  const int x = x0 + li, y = y0 + lj, z = z0 + lk;
  const bool in = x < NX && y < NY && z < NZ;
  const int gx = x + a.pnode_s[0], gy = y + a.pnode_s[1], gz = z + a.pnode_s[2];
  // the tile's global node range (clipped to the block)
  const int tx0 = x0 + a.pnode_s[0], ty0 = y0 + a.pnode_s[1], tz0 = z0 + a.pnode_s[2];
  const int tx1 = min(x0 + LT, NX) - 1 + a.pnode_s[0], ty1 = min(y0 + LT, NY) - 1 + a.pnode_s[1],
            tz1 = min(z0 + LT, NZ) - 1 + a.pnode_s[2];
  const double h = a.delta;
  double b = 0.0, bt = 0.0, vc = 0.0, ra = 0.0;
  double eS = 0.0, nC = 0.0, nE = 0.0, nCt = 0.0, eSt = 0.0;
  for (int base = 0; base < a.n_rep; base += LLIST) {
    // the replicas of [base, base + LLIST) whose box meets the tile, in order
    const int r = base + tid;
    bool hit = false;
    if (tid < LLIST && r < a.n_rep) {
      const int *bx = a.rep_box + 6 * r;
      hit = bx[0] <= tx1 && bx[1] >= tx0 && bx[2] <= ty1 && bx[3] >= ty0 && bx[4] <= tz1 && bx[5] >= tz0;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) wcount[warp] = __popc(bal);
    __syncthreads();
    if (tid == 0) {
      int s = 0;
      for (int w = 0; w < nwarp; w++) {
        const int c = wcount[w];
        wcount[w] = s;
        s += c;
      }
      nlist = s;
    }
    __syncthreads();
    if (hit) list[wcount[warp] + __popc(bal & ((1u << lane) - 1u))] = r;
    __syncthreads();
    const int nl = nlist;
    for (int q = 0; q < nl; q++) {
      const int rr = list[q], t = a.rep_type[rr];
      const int *bx = a.rep_box + 6 * rr;
      const double *c = a.rep_xyz + 3 * rr;
      // V and V~ on the halo'd tile where the replica's box + FDN covers it
      for (int p = tid; p < LH3; p += blockDim.x) {
        const int Gx = tx0 - FDN + p % LH, Gy = ty0 - FDN + (p / LH) % LH, Gz = tz0 - FDN + p / (LH * LH);
        if (Gx >= bx[0] - FDN && Gx <= bx[1] + FDN && Gy >= bx[2] - FDN && Gy <= bx[3] + FDN && Gz >= bx[4] - FDN &&
            Gz <= bx[5] + FDN) {
          double v, vt;
          if (!vloc_pair(a, t, node_radius(a, c, Gx, Gy, Gz), v, vt)) {
            atomicOr(a.status, ST_SPLINE_RANGE);
            v = vt = 0.0;
          }
          sV[p] = v;
          sVt[p] = vt;
        }
      }
      __syncthreads();
      if (in && gx >= bx[0] && gx <= bx[1] && gy >= bx[2] && gy <= bx[3] && gz >= bx[4] && gz <= bx[5]) {
        const long long hc = ((long long)(lk + FDN) * LH + (lj + FDN)) * LH + (li + FDN);
        // initialize.cpp:583-588: the atomic density at the node
        const double *G = a.tab + a.typ_off[t];
        const int len = a.typ_size[t];
        double rho_temp;
        if (!spline_at(G, G + 3 * (size_t)len, G + 4 * (size_t)len, len, node_radius(a, c, gx, gy, gz), rho_temp)) {
          atomicOr(a.status, ST_SPLINE_RANGE);
          rho_temp = 0.0;
        }
        ra += rho_temp;
        nE += rho_temp * h * h * h;
        // initialize.cpp:600-626
        const double bJ = neg_lap(a, sV, hc, LH, LH * LH), bJt = neg_lap(a, sVt, hc, LH, LH * LH);
        b += bJ;
        eS += 0.5 * bJ * sV[hc] * h * h * h;
        nC += bJ * h * h * h;
        bt += bJt;
        eSt += 0.5 * bJt * sVt[hc] * h * h * h;
        nCt += bJt * h * h * h;
        vc += sVt[hc] - sV[hc];
      }
      __syncthreads();
    }
  }
  if (in) {
    const long long g = ((long long)z * NY + y) * NX + x;
    a.b[g] = b;
    a.b_tilda[g] = bt;
    a.vc[g] = vc;
    a.rho_at[g] = ra;
  }
  const int nb = gridDim.x * gridDim.y * gridDim.z, blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const double sums[5] = {eS, nC, nE, nCt, eSt};
  for (int k = 0; k < 5; k++) {
    const double s = block_sum(sums[k], red);
    if (tid == 0) a.partial[k * nb + blk] = s;
  }
}

__global__ void charge_finish_kernel(LocalArgs a, double scale, double shift) {
  __shared__ double red[32];
  const long long n = (long long)a.np[0] * a.np[1] * a.np[2];
  double e = 0.0;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const double bt = scale * a.b_tilda[g];
    a.b_tilda[g] = bt;
    const double v = a.vc[g] + shift;
    a.vc[g] = v;
    e += 0.5 * (bt + a.b[g]) * v * a.h3;
  }
  const double s = block_sum(e, red);
  if (threadIdx.x == 0) a.partial[blockIdx.x] = s;
}

// Scratch box of replica r: extent box + 2 FDN per side.
struct SBox {
  int nx, ny, nz, i0, j0, k0;
};
__device__ __forceinline__ SBox sbox(const LocalArgs &a, int r) {
  const int *bx = a.rep_box + 6 * r;
  SBox s;
  s.nx = bx[1] - bx[0] + 1 + 4 * FDN;
  s.ny = bx[3] - bx[2] + 1 + 4 * FDN;
  s.nz = bx[5] - bx[4] + 1 + 4 * FDN;
  s.i0 = bx[0] - 2 * FDN;
  s.j0 = bx[2] - 2 * FDN;
  s.k0 = bx[4] - 2 * FDN;
  return s;
}

// forces.cpp:116-143: VlocJ, VlocJ_tilda on the box + 2 FDN.
__global__ void local_v_kernel(LocalArgs a, int r0) {
  const int r = r0 + blockIdx.y, t = a.rep_type[r];
  const SBox s = sbox(a, r);
  const long long nb = (long long)s.nx * s.ny * s.nz;
  double *V = a.scr + a.scr_off[r], *Vt = V + nb;
  const double *c = a.rep_xyz + 3 * r;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < nb; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % s.nx), j = (int)((p / s.nx) % s.ny), k = (int)(p / ((long long)s.nx * s.ny));
    double v, vt;
    if (!vloc_pair(a, t, node_radius(a, c, s.i0 + i, s.j0 + j, s.k0 + k), v, vt)) {
      atomicOr(a.status, ST_SPLINE_RANGE);
      v = vt = 0.0;
    }
    V[p] = v;
    Vt[p] = vt;
  }
}

// forces.cpp:149-173: bJ, bJ_tilda on the box + FDN.
__global__ void local_b_kernel(LocalArgs a, int r0) {
  const int r = r0 + blockIdx.y;
  const SBox s = sbox(a, r);
  const long long nb = (long long)s.nx * s.ny * s.nz, sy = s.nx, sz = (long long)s.nx * s.ny;
  double *V = a.scr + a.scr_off[r], *Vt = V + nb, *bJ = Vt + nb, *bJt = bJ + nb;
  const int mx = s.nx - 2 * FDN, my = s.ny - 2 * FDN, mz = s.nz - 2 * FDN;
  const long long m = (long long)mx * my * mz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < m; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % mx) + FDN, j = (int)((p / mx) % my) + FDN, k = (int)(p / ((long long)mx * my)) + FDN;
    const long long q = ((long long)k * s.ny + j) * s.nx + i;
    bJ[q] = neg_lap(a, V, q, sy, sz);
    bJt[q] = neg_lap(a, Vt, q, sy, sz);
  }
}

// forces.cpp:178-277: the gradients along x, y, z of bJ, bJ_tilda, VlocJ and
// VlocJ_tilda on the intersection box and the local and correction force
// terms; per-CTA sums into fpart.
__global__ void local_force_kernel(LocalArgs a, int r0) {
  __shared__ double red[32];
  const int r = r0 + blockIdx.y;
  const SBox s = sbox(a, r);
  const long long nb = (long long)s.nx * s.ny * s.nz;
  const long long st[3] = {1, s.nx, (long long)s.nx * s.ny};
  const double *V = a.scr + a.scr_off[r], *Vt = V + nb, *bJ = Vt + nb, *bJt = bJ + nb;
  const int NX = a.np[0], NY = a.np[1], PX = NX + 2 * FDN, PY = NY + 2 * FDN;
  const int mx = s.nx - 4 * FDN, my = s.ny - 4 * FDN, mz = s.nz - 4 * FDN;
  const long long m = (long long)mx * my * mz;
  double fl[3] = {0, 0, 0}, fc[3] = {0, 0, 0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < m; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % mx) + 2 * FDN, j = (int)((p / mx) % my) + 2 * FDN,
              k = (int)(p / ((long long)mx * my)) + 2 * FDN;
    const long long q = ((long long)k * s.ny + j) * s.nx + i;
    const int li = i + s.i0 - a.pnode_s[0], lj = j + s.j0 - a.pnode_s[1], lk = k + s.k0 - a.pnode_s[2];
    const double ph = a.phi[((long long)(lk + FDN) * PY + (lj + FDN)) * PX + (li + FDN)];
    const long long g = ((long long)lk * NY + lj) * NX + li;
    const double vcg = a.vcf[g], bsum = a.btf[g] + a.bf[g];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const long long sd = st[d];
      double Db = 0, Dbt = 0, DV = 0, DVt = 0;
#pragma unroll
      for (int k2 = 1; k2 <= FDN; k2++) Db += (-bJ[q - k2 * sd] + bJ[q + k2 * sd]) * a.coeff_grad[k2];
      fl[d] += Db * (ph - V[q]) * a.h3;
#pragma unroll
      for (int k2 = 1; k2 <= FDN; k2++) Dbt += (-bJt[q - k2 * sd] + bJt[q + k2 * sd]) * a.coeff_grad[k2];
#pragma unroll
      for (int k2 = 1; k2 <= FDN; k2++) DV += (-V[q - k2 * sd] + V[q + k2 * sd]) * a.coeff_grad[k2];
#pragma unroll
      for (int k2 = 1; k2 <= FDN; k2++) DVt += (-Vt[q - k2 * sd] + Vt[q + k2 * sd]) * a.coeff_grad[k2];
      fc[d] += 0.5 * (Dbt * (vcg - Vt[q]) + Db * (vcg + V[q]) + (DVt - DV) * bsum + bJ[q] * DV - bJt[q] * DVt) * a.h3;
    }
  }
  double *out = a.fpart + ((long long)blockIdx.y * gridDim.x + blockIdx.x) * 6;
  for (int d = 0; d < 3; d++) {
    const double s1 = block_sum(fl[d], red);
    if (threadIdx.x == 0) out[d] = s1;
    const double s2 = block_sum(fc[d], red);
    if (threadIdx.x == 0) out[3 + d] = s2;
  }
}

}  // namespace

int charge_density_ctas(const int np[3]) {
  return ((np[0] + LT - 1) / LT) * ((np[1] + LT - 1) / LT) * ((np[2] + LT - 1) / LT);
}

cudaError_t launch_charge_density(const LocalArgs &a, cudaStream_t s) {
  const size_t smem = 2 * (size_t)LH3 * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(charge_density_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((a.np[0] + LT - 1) / LT, (a.np[1] + LT - 1) / LT, (a.np[2] + LT - 1) / LT);
  charge_density_kernel<<<grid, LT * LT * LT, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_charge_finish(const LocalArgs &a, double scale, double shift, cudaStream_t s) {
  charge_finish_kernel<<<charge_density_ctas(a.np), 256, 0, s>>>(a, scale, shift);
  return cudaGetLastError();
}

cudaError_t launch_forces_local(const LocalArgs &a, int r0, int r1, cudaStream_t s) {
  if (r1 <= r0) return cudaSuccess;
  const dim3 grid(LOC_FORCE_CTAS, r1 - r0);
  local_v_kernel<<<grid, 256, 0, s>>>(a, r0);
  local_b_kernel<<<grid, 256, 0, s>>>(a, r0);
  local_force_kernel<<<grid, 256, 0, s>>>(a, r0);
  return cudaGetLastError();
}

}  // namespace sqb
