// Device-side Fermi-level solver of the whole-step CUDA graph (FermiDev in
// sqb_internal.cuh): Brent's and Newton's methods with the host solvers'
// statements (sqb_api.cu).  Compiled without multiply-add contraction
// (-fmad=false, see build.py) so that every operation rounds as the host's
// separate multiply and add do and the sequence of trial Fermi levels is the
// host path's bit for bit.
#include <cmath>

#include "sqb_internal.cuh"

namespace sqb {

namespace {

#define SQB_SIGN(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))

// The Brent iteration of sq.cpp:1322-1399 up to the next evaluation: the
// bracket update, the convergence test (root found: status 1) and the next
// trial level b.  The host solver (sqb_api.cu) runs the same statements.
__device__ void brent_advance(FermiDev &s) {
  const double EPS = 2.5e-16, tol = s.tol;
  double tol1q, eq, min1, min2, p, q, r, sv, tol1, xm;
  if ((s.fb > 0.0 && s.fc > 0.0) || (s.fb < 0.0 && s.fc < 0.0)) {
    s.cc = s.a;
    s.fc = s.fa;
    s.e = s.d = s.b - s.a;
  }
  if (fabs(s.fc) < fabs(s.fb)) {
    s.a = s.b;
    s.b = s.cc;
    s.cc = s.a;
    s.fa = s.fb;
    s.fb = s.fc;
    s.fc = s.fa;
  }
  tol1 = 2.0 * EPS * fabs(s.b) + 0.5 * tol;
  xm = 0.5 * (s.cc - s.b);
  if (fabs(xm) <= tol1 || s.fb == 0.0) {
    s.root = s.b;
    s.iters = s.iter;
    s.status = 1;
    return;
  }
  if (fabs(s.e) >= tol1 && fabs(s.fa) > fabs(s.fb)) {
    sv = s.fb / s.fa;
    if (s.a == s.cc) {
      p = 2.0 * xm * sv;
      q = 1.0 - sv;
    } else {
      q = s.fa / s.fc;
      r = s.fb / s.fc;
      p = sv * (2.0 * xm * q * (q - r) - (s.b - s.a) * (r - 1.0));
      q = (q - 1.0) * (r - 1.0) * (sv - 1.0);
    }
    if (p > 0.0) q = -q;
    p = fabs(p);
    tol1q = tol1 * q;
    min1 = 3.0 * xm * q - fabs(tol1q);
    eq = s.e * q;
    min2 = fabs(eq);
    if (2.0 * p < (min1 < min2 ? min1 : min2)) {
      s.e = s.d;
      s.d = p / q;
    } else {
      s.d = xm;
      s.e = s.d;
    }
  } else {
    s.d = xm;
    s.e = s.d;
  }
  s.a = s.b;
  s.fa = s.fb;
  if (fabs(s.d) > tol1) s.b += s.d;
  else s.b += SQB_SIGN(tol1, xm);
  s.x = s.b;
}

__global__ void fermi_init_kernel(FermiDev *st, const double *minmax) {
  FermiDev &s = *st;
  s.steps = 0;
  s.status = 0;
  s.dstat = 0;
  s.lmin_all = minmax[0];
  s.lmax_all = minmax[1];
  s.iters = 0;
  s.root = 0.0;
  if (s.alg == 1) {  // sq.cpp:1289-1311 with the bracket of sq.cpp:669-713
    s.a = minmax[0] - 1;
    s.b = minmax[1] + 1;
    s.cc = s.b;
    s.d = s.e = 0.0;
    if (s.scf_iter > 1) {
      s.a = s.lambda_warm - 2;
      s.b = s.lambda_warm + 2;
    }
    s.phase = 0;
    s.iter = 0;
    s.x = s.a;
  } else {  // sq.cpp:721-730, 1459-1490
    s.lnew = 0.0;
    s.lold = s.scf_iter <= 1 ? 0.2 : s.lambda_warm;
    s.err = 1.0;
    s.count = 0;
    s.x = s.lold;
    if (!(s.err > s.tol)) {
      s.root = s.lnew;
      s.status = 1;
    }
  }
}

// One NeConstraint result (sums[0], and sums[1] for Newton) into the solver;
// sets the loop condition.  The loop ends after at most 512 evaluations
// whatever the inputs (the solvers' own limits are 102 and 200).
__global__ void fermi_step_kernel(FermiDev *st, const double *sums, cudaGraphConditionalHandle h) {
  FermiDev &s = *st;
  if (s.status == 0) {
    s.steps++;
    if (s.alg == 1) {
      const double f = sums[0] * s.h3 - (-s.ncharge);  // sq.cpp:1214-1226
      if (!isfinite(f)) {
        s.status = -3;
      } else if (s.phase == 0) {
        s.fa = f;
        s.phase = 1;
        s.x = s.b;
      } else {
        s.fb = f;
        if (s.phase == 1) {
          if ((s.fa > 0.0 && s.fb > 0.0) || (s.fa < 0.0 && s.fb < 0)) s.status = -1;
          s.fc = s.fb;
          s.phase = 2;
        }
        if (s.status == 0) {
          s.iter++;
          if (s.iter > 100) s.status = -2;
          else brent_advance(s);
        }
      }
    } else {
      double g = sums[0], dg = sums[1];
      dg = dg * s.bet;
      dg = dg * s.h3;
      g = g * s.h3;
      const double fa = g - (-s.ncharge), dfa = dg;
      s.lnew = s.lold - (fa / dfa);
      s.err = fabs(s.lnew - s.lold);
      s.lold = s.lnew;
      s.count += 1;
      s.x = s.lold;
      if (!(s.err > s.tol && s.count < 200)) {
        s.root = s.lnew;
        s.iters = s.count;
        s.status = isfinite(s.lnew) ? 1 : -3;
      }
    }
    if (s.status == 0 && s.steps >= 512) s.status = -2;
  }
  cudaGraphSetConditional(h, s.status == 0 ? 1u : 0u);
}

}  // namespace

cudaError_t launch_fermi_init(FermiDev *st, const double *minmax, cudaStream_t s) {
  fermi_init_kernel<<<1, 1, 0, s>>>(st, minmax);
  return cudaGetLastError();
}

cudaError_t launch_fermi_step(FermiDev *st, const double *sums, cudaGraphConditionalHandle h, cudaStream_t s) {
  fermi_step_kernel<<<1, 1, 0, s>>>(st, sums, h);
  return cudaGetLastError();
}

}  // namespace sqb
