/* CPU restatement of SQDFT's SQ step -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Every routine restates the cited reference function with its arithmetic
 * order kept (sums in the same sequence, divisions where the reference
 * divides), so that, compiled without FMA contraction, it agrees with the
 * reference build to rounding level.  See sq_oracle.h for layouts.
 */
#include "sq_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define TEMP_TOL 1e-12
#define SIGN(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))

/* ---------------------------------------------------------------------- */
/* Nonlocal geometry                                                       */
/* ---------------------------------------------------------------------- */

/* Nearest node of a replica coordinate with the midpoint rule of
 * nonlocal.cpp:49-64 (round, but an atom on a midpoint goes left). */
static int nearest_node(double c, double h) {
  int n = (int)round(c / h);
  if (fabs(fabs(n * h - c) - h * 0.5) < TEMP_TOL) n = (int)floor((c / h) - 10 * TEMP_TOL);
  return n;
}

typedef struct {
  int rep;           /* replica index */
  int x0, x1, y0, y1, z0, z1; /* intersection in global node indices */
  int inn, jnn, knn, nlocc, nproj, type;
} nl_entry;

/* Replicas whose rc-ball meets the Rcut window of global node (gx,gy,gz), in
 * the reference's loop order (types, main atoms, replicas; nonlocal.cpp:41-44).
 * The interval logic of nonlocal.cpp:80-108 is a plain intersection. */
static int node_entries(const sqo_problem *p, int gx, int gy, int gz, nl_entry *out) {
  int cnt = 0;
  for (int r = 0; r < p->n_rep; r++) {
    int t = p->rep_type[r];
    int nlocc = p->typ_nlocc[t];
    int inn = nearest_node(p->rep_xyz[3 * r], p->delta);
    int jnn = nearest_node(p->rep_xyz[3 * r + 1], p->delta);
    int knn = nearest_node(p->rep_xyz[3 * r + 2], p->delta);
    int x0 = inn - nlocc > gx - p->nloc ? inn - nlocc : gx - p->nloc;
    int x1 = inn + nlocc < gx + p->nloc ? inn + nlocc : gx + p->nloc;
    int y0 = jnn - nlocc > gy - p->nloc ? jnn - nlocc : gy - p->nloc;
    int y1 = jnn + nlocc < gy + p->nloc ? jnn + nlocc : gy + p->nloc;
    int z0 = knn - nlocc > gz - p->nloc ? knn - nlocc : gz - p->nloc;
    int z1 = knn + nlocc < gz + p->nloc ? knn + nlocc : gz + p->nloc;
    if (x0 > x1 || y0 > y1 || z0 > z1) continue;
    if (p->typ_nproj[t] == 0) continue;
    nl_entry e = {r, x0, x1, y0, y1, z0, z1, inn, jnn, knn, nlocc, p->typ_nproj[t], t};
    out[cnt++] = e;
  }
  return cnt;
}

/* Denominator of projector c of type t (the l of the c-th (l,m) pair). */
static double proj_denom(const sqo_problem *p, int t, int c) {
  int cnt = 0;
  for (int l = 0; l <= p->typ_lmax[t]; l++) {
    if (l == p->typ_lloc[t]) continue;
    if (c < cnt + 2 * l + 1) return p->typ_denom[4 * t + l];
    cnt += 2 * l + 1;
  }
  return 0.0;
}

typedef struct {
  const sqo_problem *p;
  int nd, i, j, k, gx, gy, gz, n, nent;
  nl_entry *ent;
  double *vv;
} node_ctx;

static void node_begin(const sqo_problem *p, int nd, node_ctx *c) {
  c->p = p;
  c->nd = nd;
  c->i = nd % p->np[0];
  c->j = (nd / p->np[0]) % p->np[1];
  c->k = nd / (p->np[0] * p->np[1]);
  c->gx = p->pnode_s[0] + c->i;
  c->gy = p->pnode_s[1] + c->j;
  c->gz = p->pnode_s[2] + c->k;
  c->n = 2 * p->nloc + 1;
  c->ent = (nl_entry *)malloc(sizeof(nl_entry) * (size_t)(p->n_rep > 0 ? p->n_rep : 1));
  c->nent = node_entries(p, c->gx, c->gy, c->gz, c->ent);
  c->vv = (double *)malloc(sizeof(double) * (size_t)c->n * c->n * c->n);
}

static void node_end(node_ctx *c) {
  free(c->ent);
  free(c->vv);
}

/* VnlocsubTimesVec (nonlocal.cpp:20-215): vv += sum over replicas and (l,m) of
 * chi (chi^T v / Denom).  vv must be zeroed by the caller (sq.cpp:872-881). */
static void vnloc_times_vec(const node_ctx *c, const double *v, double *vv, int only_rep_atom) {
  const sqo_problem *p = c->p;
  const int n = c->n, nl = p->nloc;
  for (int e = 0; e < c->nent; e++) {
    const nl_entry *E = &c->ent[e];
    if (only_rep_atom >= 0 && p->rep_atom[E->rep] != only_rep_atom) continue;
    const int S = 2 * E->nlocc + 1;
    for (int q = 0; q < E->nproj; q++) {
      const double denom = proj_denom(p, E->type, q);
      const double *U = p->udvtm + p->rep_off[E->rep] + (long long)q * S * S * S;
      double temp = 0.0;
      for (int z = E->z0; z <= E->z1; z++)
        for (int y = E->y0; y <= E->y1; y++)
          for (int x = E->x0; x <= E->x1; x++) {
            int w = ((z - c->gz + nl) * n + (y - c->gy + nl)) * n + (x - c->gx + nl);
            int b = ((z - E->knn) + E->nlocc) * S * S + ((y - E->jnn) + E->nlocc) * S + ((x - E->inn) + E->nlocc);
            temp = temp + v[w] * U[b] / denom;
          }
      for (int z = E->z0; z <= E->z1; z++)
        for (int y = E->y0; y <= E->y1; y++)
          for (int x = E->x0; x <= E->x1; x++) {
            int w = ((z - c->gz + nl) * n + (y - c->gy + nl)) * n + (x - c->gx + nl);
            int b = ((z - E->knn) + E->nlocc) * S * S + ((y - E->jnn) + E->nlocc) * S + ((x - E->inn) + E->nlocc);
            vv[w] = vv[w] + temp * U[b];
          }
    }
  }
}

/* HsubTimesVec (sq.cpp:838-929): -1/2 Lap v + Veff v + Vnl v on the window,
 * with v zero outside it. */
static void hsub(const node_ctx *c, const double *v, double *hv) {
  const sqo_problem *p = c->p;
  const int n = c->n, nl = p->nloc, F = p->fdn;
  const int ex = p->np[0] + 2 * nl, ey = p->np[1] + 2 * nl;
  memset(c->vv, 0, sizeof(double) * (size_t)n * n * n);
  vnloc_times_vec(c, v, c->vv, -1);
  for (int z = 0; z < n; z++)
    for (int y = 0; y < n; y++)
      for (int x = 0; x < n; x++) {
        const int w = (z * n + y) * n + x;
        double temp = v[w] * 3 * p->coeff_lap[0];
        for (int a = 1; a <= F; a++) {
          double xm = x - a >= 0 ? v[w - a] : 0.0, xp = x + a < n ? v[w + a] : 0.0;
          double ym = y - a >= 0 ? v[w - a * n] : 0.0, yp = y + a < n ? v[w + a * n] : 0.0;
          double zm = z - a >= 0 ? v[w - a * n * n] : 0.0, zp = z + a < n ? v[w + a * n * n] : 0.0;
          temp += (xm + xp + ym + yp + zm + zp) * p->coeff_lap[a];
        }
        /* Veff[k+kk][j+jj][i+ii] with k = node + nloc and kk = z - nloc */
        const double ve = p->veff[((size_t)(c->k + z) * ey + (c->j + y)) * ex + (c->i + x)];
        hv[w] = -0.5 * temp + ve * v[w] + c->vv[w];
      }
}

void sqo_hsub_times_vec(const sqo_problem *p, int nd, const double *v, double *hv) {
  node_ctx c;
  node_begin(p, nd, &c);
  hsub(&c, v, hv);
  node_end(&c);
}

/* ---------------------------------------------------------------------- */
/* Lanczos                                                                 */
/* ---------------------------------------------------------------------- */

/* TridiagEigenSolve (sq.cpp:1094-1180): implicit QL, then extreme diagonal. */
int sqo_tridiag_eigen(const double *diag, const double *subdiag, int n, double *lambda_min, double *lambda_max) {
  int m, l, iter, i;
  double s, r, p, g, f, dd, c, b;
  double *d = (double *)malloc(sizeof(double) * (size_t)n), *e = (double *)malloc(sizeof(double) * (size_t)n);
  for (i = 0; i < n; i++) {
    d[i] = diag[i];
    e[i] = subdiag[i];
  }
  e[n - 1] = 0.0;
  for (l = 0; l <= n - 1; l++) {
    iter = 0;
    do {
      for (m = l; m <= n - 2; m++) {
        dd = fabs(d[m]) + fabs(d[m + 1]);
        if ((double)(fabs(e[m]) + dd) == dd) break;
      }
      if (m != l) {
        if (iter++ == 200) {
          free(d);
          free(e);
          return -1;
        }
        g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        r = sqrt(g * g + 1.0);
        g = d[m] - d[l] + e[l] / (g + SIGN(r, g));
        s = c = 1.0;
        p = 0.0;
        for (i = m - 1; i >= l; i--) {
          f = s * e[i];
          b = c * e[i];
          e[i + 1] = (r = sqrt(g * g + f * f));
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          d[i + 1] = g + (p = s * r);
          g = c * r - b;
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  *lambda_min = d[0];
  *lambda_max = d[0];
  for (i = 1; i < n; i++) {
    if (d[i] > *lambda_max) *lambda_max = d[i];
    else if (d[i] < *lambda_min) *lambda_min = d[i];
  }
  free(d);
  free(e);
  return 0;
}

static double dot(const double *a, const double *b, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; i++) s = s + a[i] * b[i];
  return s;
}

/* LanczosAlgorithm (sq.cpp:965-1092) with the start vector of sq.cpp:538-546
 * (all ones).  Returns the iteration count; lambda_min/max include the
 * +-lanczos_tol widening (sq.cpp:1067-1068). */
static int lanczos(const node_ctx *c, double *lambda_min, double *lambda_max) {
  const sqo_problem *p = c->p;
  const size_t nw = (size_t)c->n * c->n * c->n;
  const int max_iter = 500;
  double *vkm1 = malloc(sizeof(double) * nw), *vk = malloc(sizeof(double) * nw), *vkp1 = malloc(sizeof(double) * nw);
  double *aa = calloc(nw, sizeof(double)), *bb = calloc(nw, sizeof(double));
  for (size_t w = 0; w < nw; w++) vkm1[w] = 1.0;
  double val = sqrt(dot(vkm1, vkm1, nw));
  for (size_t w = 0; w < nw; w++) vkm1[w] = vkm1[w] / val;
  hsub(c, vkm1, vk);
  aa[0] = dot(vkm1, vk, nw);
  for (size_t w = 0; w < nw; w++) vk[w] = vk[w] - aa[0] * vkm1[w];
  bb[0] = sqrt(dot(vk, vk, nw));
  for (size_t w = 0; w < nw; w++) vk[w] = vk[w] / bb[0];
  int count = 0;
  double lmin_prev = 0.0, lmax_prev = 0.0, dl = 1.0, dm = 1.0;
  while (count < max_iter && (dl > p->lanczos_tol || dm > p->lanczos_tol)) {
    hsub(c, vk, vkp1);
    aa[count + 1] = dot(vk, vkp1, nw);
    for (size_t w = 0; w < nw; w++) vkp1[w] = vkp1[w] - aa[count + 1] * vk[w] - bb[count] * vkm1[w];
    bb[count + 1] = sqrt(dot(vkp1, vkp1, nw));
    for (size_t w = 0; w < nw; w++) {
      vkm1[w] = vk[w];
      vk[w] = vkp1[w] / bb[count + 1];
    }
    sqo_tridiag_eigen(aa, bb, count + 2, lambda_min, lambda_max);
    dl = fabs((*lambda_min) - lmin_prev);
    dm = fabs((*lambda_max) - lmax_prev);
    lmin_prev = *lambda_min;
    lmax_prev = *lambda_max;
    count = count + 1;
  }
  *lambda_min -= p->lanczos_tol;
  *lambda_max += p->lanczos_tol;
  free(vkm1);
  free(vk);
  free(vkp1);
  free(aa);
  free(bb);
  return count;
}

int sqo_lanczos(const sqo_problem *p, int nd, double *lambda_min, double *lambda_max) {
  node_ctx c;
  node_begin(p, nd, &c);
  int it = lanczos(&c, lambda_min, lambda_max);
  node_end(&c);
  return it;
}

/* Chebyshev moments (sq.cpp:564-655): direct for nq <= npl/4, then the
 * doubling identities T_2n = 2 T_n^2 - 1, T_2n-1 = 2 T_n T_n-1 - T_1. */
static void moments(const node_ctx *c, double chi, double zee, double *rho_pj) {
  const sqo_problem *p = c->p;
  const size_t nw = (size_t)c->n * c->n * c->n;
  const size_t ctr = nw / 2;
  const double h3 = pow(p->delta, 3);
  double *t0 = malloc(sizeof(double) * nw), *t1 = malloc(sizeof(double) * nw), *t2 = malloc(sizeof(double) * nw);
  double *hv = malloc(sizeof(double) * nw);
  for (size_t w = 0; w < nw; w++) t0[w] = 0.0;
  t0[ctr] = 1.0;
  hsub(c, t0, hv);
  for (size_t w = 0; w < nw; w++) t1[w] = (hv[w] - chi * t0[w]) / zee;
  const double htemp = t1[ctr];
  const int q1 = (int)round(0.25 * p->npl), q2 = (int)round(0.5 * p->npl);
  for (int nq = 0; nq <= q1; nq++) {
    if (nq == 0) rho_pj[nq] = (double)(t0[ctr] / h3);
    else if (nq == 1) rho_pj[nq] = (double)(t1[ctr] / h3);
    else {
      hsub(c, t1, hv);
      for (size_t w = 0; w < nw; w++) {
        t2[w] = (2 * (hv[w] - chi * t1[w]) / zee) - t0[w];
        t0[w] = t1[w];
        t1[w] = t2[w];
      }
      rho_pj[nq] = (double)(t2[ctr] / h3);
    }
  }
  for (int nq = q1 + 1; nq <= q2; nq++) {
    double d1 = 0.0, d2 = 0.0;
    hsub(c, t1, hv);
    for (size_t w = 0; w < nw; w++) {
      t2[w] = (2 * (hv[w] - chi * t1[w]) / zee) - t0[w];
      d1 += t2[w] * t2[w];
      d2 += t2[w] * t1[w];
      t0[w] = t1[w];
      t1[w] = t2[w];
    }
    rho_pj[nq] = (double)(t2[ctr] / h3);
    rho_pj[2 * nq] = (double)((2 * d1 - 1) / h3);
    rho_pj[2 * nq - 1] = (double)((2 * d2 - htemp) / h3);
  }
  free(t0);
  free(t1);
  free(t2);
  free(hv);
}

void sqo_moments(const sqo_problem *p, int nd, double chi, double zee, double *rho_pj) {
  node_ctx c;
  node_begin(p, nd, &c);
  moments(&c, chi, zee, rho_pj);
  node_end(&c);
}

static int g_threads = 1;
void sqo_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

typedef struct {
  const sqo_problem *p;
  const int *nodes;
  int count;
  double *chi, *zee, *rho_pj, *lmin, *lmax;
  int *iters;
  int next;
  pthread_mutex_t mu;
} lm_job;

static void lm_one(lm_job *J, int q) {
  const sqo_problem *p = J->p;
  const int nd = J->nodes[q];
  node_ctx c;
  node_begin(p, nd, &c);
  double lmin, lmax;
  int it = lanczos(&c, &lmin, &lmax);
  if (J->iters) J->iters[nd] = it;
  if (J->lmin) J->lmin[nd] = lmin;
  if (J->lmax) J->lmax[nd] = lmax;
  J->chi[nd] = (lmax + lmin) / 2; /* sq.cpp:564-565 */
  J->zee[nd] = (lmax - lmin) / 2;
  moments(&c, J->chi[nd], J->zee[nd], J->rho_pj + (size_t)nd * (p->npl + 1));
  node_end(&c);
}

static void *lm_worker(void *arg) {
  lm_job *J = (lm_job *)arg;
  for (;;) {
    pthread_mutex_lock(&J->mu);
    int q = J->next++;
    pthread_mutex_unlock(&J->mu);
    if (q >= J->count) return NULL;
    lm_one(J, q);
  }
}

int sqo_lanczos_moments(const sqo_problem *p, const int *nodes, int count, double *chi, double *zee,
                        double *rho_pj, int *lanczos_iters, double *lmin_out, double *lmax_out) {
  lm_job J = {p, nodes, count, chi, zee, rho_pj, lmin_out, lmax_out, lanczos_iters, 0, PTHREAD_MUTEX_INITIALIZER};
  int nt = g_threads < count ? g_threads : count;
  if (nt <= 1) {
    for (int q = 0; q < count; q++) lm_one(&J, q);
    return 0;
  }
  pthread_t th[256];
  if (nt > 256) nt = 256;
  for (int t = 0; t < nt; t++) pthread_create(&th[t], NULL, lm_worker, &J);
  for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Fermi level, density and energies                                      */
/* ---------------------------------------------------------------------- */

static double fermi_dirac(double t, double lf, double bet) { return 1 / (1 + exp(bet * (t - lf))); } /* sq.cpp:1261 */
static double uband(double t, double lf, double bet) { return t * (1 / (1 + exp(bet * (t - lf)))); } /* sq.cpp:1268 */
static double eent(double t, double lf, double bet) {                                                /* sq.cpp:1275 */
  double focc = (1 / (1 + exp(bet * (t - lf))));
  if (fabs(focc) < 0.01 * TEMP_TOL || fabs(focc - 1.0) < 0.01 * TEMP_TOL) return 0.0;
  return (focc * log(focc) + (1 - focc) * log(1 - focc));
}
static double fermi_derv(double t, double lf, double bet) { /* sq.cpp:1451 */
  double v = 1 / (1 + exp(bet * (t - lf)));
  return v * (1 - v);
}

void sqo_chebyshev_coeff(int npl, double lambda_fp, double bet, double *ci, int kind) {
  double *d = malloc(sizeof(double) * (size_t)(npl + 1));
  for (int k = 0; k < npl + 1; k++) {
    double y = cos(M_PI * ((double)((k - 0.5 + 1) / (npl + 1))));
    d[k] = kind == 0 ? fermi_dirac(y, lambda_fp, bet)
         : kind == 1 ? uband(y, lambda_fp, bet)
         : kind == 2 ? eent(y, lambda_fp, bet)
                     : fermi_derv(y, lambda_fp, bet);
  }
  double fac = 2.0 / (npl + 1);
  for (int j = 0; j < npl + 1; j++) {
    double sum = 0.0;
    for (int k = 0; k < npl + 1; k++) sum = sum + d[k] * cos((M_PI * (j - 1 + 1)) * ((double)((k - 0.5 + 1) / (npl + 1))));
    ci[j] = fac * sum;
  }
  ci[0] = ci[0] / 2.0;
  free(d);
}

double sqo_ne_constraint(const sqo_problem *p, const double *chi, const double *zee, const double *rho_pj,
                         double lambda_f) {
  const int nn = p->np[0] * p->np[1] * p->np[2];
  double *ci = malloc(sizeof(double) * (size_t)(p->npl + 1));
  double g = 0.0;
  for (int k = 0; k < nn; k++) {
    double lambda_fp = (lambda_f - chi[k]) / zee[k];
    double bet = p->bet * zee[k];
    sqo_chebyshev_coeff(p->npl, lambda_fp, bet, ci, 0);
    for (int j = 0; j < p->npl + 1; j++) g = g + 2 * rho_pj[(size_t)k * (p->npl + 1) + j] * ci[j];
  }
  g = g * pow(p->delta, 3);
  free(ci);
  return g - (-p->ncharge);
}

static void ne_constraint_derv(const sqo_problem *p, const double *chi, const double *zee, const double *rho_pj,
                               double lambda_f, double *fa, double *dfa) { /* sq.cpp:1407-1449 */
  const int nn = p->np[0] * p->np[1] * p->np[2];
  double *ci = malloc(sizeof(double) * (size_t)(p->npl + 1));
  double g = 0.0, dg = 0.0;
  for (int k = 0; k < nn; k++) {
    double lambda_fp = (lambda_f - chi[k]) / zee[k];
    double bet = p->bet * zee[k];
    sqo_chebyshev_coeff(p->npl, lambda_fp, bet, ci, 0);
    for (int j = 0; j < p->npl + 1; j++) g = g + 2 * rho_pj[(size_t)k * (p->npl + 1) + j] * ci[j];
    sqo_chebyshev_coeff(p->npl, lambda_fp, bet, ci, 3);
    for (int j = 0; j < p->npl + 1; j++) dg = dg + 2 * rho_pj[(size_t)k * (p->npl + 1) + j] * ci[j];
  }
  dg = dg * p->bet;
  dg = dg * pow(p->delta, 3);
  g = g * pow(p->delta, 3);
  *fa = g - (-p->ncharge);
  *dfa = dg;
  free(ci);
}

int sqo_fermi_level(const sqo_problem *p, const double *chi, const double *zee, const double *rho_pj, int scf_iter,
                    double lambda_warm, double lmin, double lmax, double *lambda_out, int *iters_out) {
  if (p->fermi_alg == 2) { /* NewtonRaphson, sq.cpp:1459-1490, started as sq.cpp:721-730 */
    double lam = scf_iter <= 1 ? 0.2 : lambda_warm;
    double tol = p->fermi_tol, lnew = 0.0, fa, dfa, err = 1.0;
    int count = 0;
    while (err > tol && count < 200) {
      ne_constraint_derv(p, chi, zee, rho_pj, lam, &fa, &dfa);
      lnew = lam - (fa / dfa);
      err = fabs(lnew - lam);
      lam = lnew;
      count += 1;
    }
    *lambda_out = lnew;
    if (iters_out) *iters_out = count;
    return 0;
  }
  /* BrentsAlgorithm (sq.cpp:1289-1404) on (lmin-1, lmax+1), sq.cpp:720 */
  const double EPS = 2.5e-16, tol = p->fermi_tol;
  double tol1q, eq, a = lmin - 1, b = lmax + 1, c = lmax + 1, d = 0.0, e = 0.0, min1, min2;
  if (scf_iter > 1) {
    a = lambda_warm - 2;
    b = lambda_warm + 2;
  }
  double fa = sqo_ne_constraint(p, chi, zee, rho_pj, a), fb = sqo_ne_constraint(p, chi, zee, rho_pj, b);
  double fc, pp, q, r, s, tol1, xm;
  if ((fa > 0.0 && fb > 0.0) || (fa < 0.0 && fb < 0)) return -2;
  fc = fb;
  for (int iter = 1; iter <= 100; iter++) {
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) {
      c = a;
      fc = fa;
      e = d = b - a;
    }
    if (fabs(fc) < fabs(fb)) {
      a = b;
      b = c;
      c = a;
      fa = fb;
      fb = fc;
      fc = fa;
    }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * tol;
    xm = 0.5 * (c - b);
    if (fabs(xm) <= tol1 || fb == 0.0) {
      *lambda_out = b;
      if (iters_out) *iters_out = iter;
      return 0;
    }
    if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
      s = fb / fa;
      if (a == c) {
        pp = 2.0 * xm * s;
        q = 1.0 - s;
      } else {
        q = fa / fc;
        r = fb / fc;
        pp = s * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (pp > 0.0) q = -q;
      pp = fabs(pp);
      tol1q = tol1 * q;
      min1 = 3.0 * xm * q - fabs(tol1q);
      eq = e * q;
      min2 = fabs(eq);
      if (2.0 * pp < (min1 < min2 ? min1 : min2)) {
        e = d;
        d = pp / q;
      } else {
        d = xm;
        e = d;
      }
    } else {
      d = xm;
      e = d;
    }
    a = b;
    fa = fb;
    if (fabs(d) > tol1) b += d;
    else b += SIGN(tol1, xm);
    fb = sqo_ne_constraint(p, chi, zee, rho_pj, b);
  }
  return -3;
}

int sqo_density_energy(const sqo_problem *p, const double *chi, const double *zee, const double *rho_pj,
                       double lambda_f, double *rho, double *ci_all, double *ebs_out, double *eent_out) {
  const int nn = p->np[0] * p->np[1] * p->np[2], K = p->npl + 1;
  const double bet0 = p->bet, h3 = pow(p->delta, 3);
  double *ci = malloc(sizeof(double) * (size_t)K);
  double Ebs = 0.0, Eent = 0.0;
  int status = 0;
  for (int nd = 0; nd < nn; nd++) {
    const double *mu = rho_pj + (size_t)nd * K;
    double *cf = ci_all + (size_t)nd * K;
    double bet = bet0 * zee[nd];
    double lambda_fp = (lambda_f - chi[nd]) / zee[nd];
    sqo_chebyshev_coeff(p->npl, lambda_fp, bet, cf, 0);
    double rho_pc = 0.0;
    for (int j = 0; j < K; j++) rho_pc = rho_pc + 2 * mu[j] * cf[j];
    rho[nd] = fabs(rho_pc);
    if (rho_pc < 0 && fabs(rho_pc) > 1e-6) status = -4;
    sqo_chebyshev_coeff(p->npl, lambda_fp, bet, ci, 1);
    double ebs = 0.0;
    for (int j = 0; j < K; j++) ebs = ebs + 2 * mu[j] * ci[j];
    Ebs = Ebs + (zee[nd] * ebs + chi[nd] * rho_pc) * h3;
    sqo_chebyshev_coeff(p->npl, lambda_fp, bet, ci, 2);
    double ent = 0.0;
    for (int j = 0; j < K; j++) ent = ent + 2 * mu[j] * ci[j];
    Eent = Eent + (1 / bet0) * ent * h3;
  }
  *ebs_out = Ebs;
  *eent_out = Eent;
  free(ci);
  return status;
}

/* ---------------------------------------------------------------------- */
/* Nonlocal forces                                                         */
/* ---------------------------------------------------------------------- */

int sqo_forces_nonlocal(const sqo_problem *p, const int *nodes, int count, const double *chi, const double *zee,
                        const double *ci_all, double *f) {
  const int nl = p->nloc, F = p->fdn, n = 2 * nl + 1, m = n + 2 * F;
  const size_t nw = (size_t)n * n * n;
  const double h3 = pow(p->delta, 3);
  double *t0 = malloc(sizeof(double) * nw), *t1 = malloc(sizeof(double) * nw), *t2 = malloc(sizeof(double) * nw);
  double *hv = malloc(sizeof(double) * nw), *dm = calloc((size_t)m * m * m, sizeof(double));
  double *grad[3] = {malloc(sizeof(double) * nw), malloc(sizeof(double) * nw), malloc(sizeof(double) * nw)};
  for (int qn = 0; qn < count; qn++) {
    const int nd = nodes[qn];
    node_ctx c;
    node_begin(p, nd, &c);
    const double *cf = ci_all + (size_t)nd * (p->npl + 1);
    for (size_t w = 0; w < nw; w++) t0[w] = 0.0;
    t0[nw / 2] = 1.0;
    hsub(&c, t0, hv);
    for (size_t w = 0; w < nw; w++) t1[w] = (hv[w] - chi[nd] * t0[w]) / zee[nd];
    for (int z = 0; z < n; z++)
      for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) dm[((size_t)(z + F) * m + (y + F)) * m + (x + F)] = 0.0;
    for (int nq = 0; nq <= p->npl; nq++) { /* forces.cpp:410-460 */
      if (nq >= 2) hsub(&c, t1, hv);
      for (int z = 0; z < n; z++)
        for (int y = 0; y < n; y++)
          for (int x = 0; x < n; x++) {
            size_t w = ((size_t)z * n + y) * n + x, d = ((size_t)(z + F) * m + (y + F)) * m + (x + F);
            if (nq == 0) dm[d] += (double)(t0[w] * cf[nq] / h3);
            else if (nq == 1) dm[d] += (double)(t1[w] * cf[nq] / h3);
            else {
              t2[w] = (2 * (hv[w] - chi[nd] * t1[w]) / zee[nd]) - t0[w];
              dm[d] += (double)(t2[w] * cf[nq] / h3);
              t0[w] = t1[w];
              t1[w] = t2[w];
            }
          }
    }
    /* 12th-order gradient of the density-matrix column (forces.cpp:464-501) */
    for (int z = 0; z < n; z++)
      for (int y = 0; y < n; y++)
        for (int x = 0; x < n; x++) {
          size_t w = ((size_t)z * n + y) * n + x, d = ((size_t)(z + F) * m + (y + F)) * m + (x + F);
          double gx = 0.0, gy = 0.0, gz = 0.0;
          for (int a = 1; a <= F; a++) gx += (-dm[d - a] + dm[d + a]) * p->coeff_grad[a];
          for (int a = 1; a <= F; a++) gy += (-dm[d - (size_t)a * m] + dm[d + (size_t)a * m]) * p->coeff_grad[a];
          for (int a = 1; a <= F; a++) gz += (-dm[d - (size_t)a * m * m] + dm[d + (size_t)a * m * m]) * p->coeff_grad[a];
          grad[0][w] = gx;
          grad[1][w] = gy;
          grad[2][w] = gz;
        }
    /* per atom: centre value of VnlocsubTimesVec_J (nonlocal.cpp:522-724) */
    for (int atom = 0; atom < p->n_atm; atom++) {
      int has = 0;
      for (int r = 0; r < p->n_rep && !has; r++) has = p->rep_atom[r] == atom;
      if (!has) continue;
      for (int dir = 0; dir < 3; dir++) {
        memset(hv, 0, sizeof(double) * nw);
        vnloc_times_vec(&c, grad[dir], hv, atom);
        f[3 * atom + dir] += -4 * hv[nw / 2] * h3;
      }
    }
    node_end(&c);
  }
  free(t0);
  free(t1);
  free(t2);
  free(hv);
  free(dm);
  for (int d = 0; d < 3; d++) free(grad[d]);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Projectors                                                              */
/* ---------------------------------------------------------------------- */

/* ispline_gen (spline.cpp:11-55) at one point; returns -1 out of range. */
static int spline_at(const double *X, const double *Y, const double *YD, int len, double x, double *out) {
  if (x < X[0] || x > X[len - 1]) return -1;
  int j = 0;
  for (; j < len && x > X[j]; j++) {
  }
  if (x < X[j]) j--;
  double p1 = X[j];
  double dx = 1.0 / (X[j + 1] - X[j]);
  double dy = (Y[j + 1] - Y[j]) * dx;
  double A0 = Y[j], A1 = YD[j];
  double A2 = dx * (3.0 * dy - 2.0 * YD[j] - YD[j + 1]);
  double A3 = dx * dx * (-2.0 * dy + YD[j] + YD[j + 1]);
  double t = x - p1;
  *out = ((A3 * t + A2) * t + A1) * t + A0;
  return 0;
}

/* SphericalHarmonics (nonlocal.cpp:218-314): real harmonics with the same
 * 15-digit normalisation constants. */
static double real_sh(double x, double y, double z, double r, int l, int m) {
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

int sqo_projectors(const sqo_problem *p, const sqo_psd *psd, double *udvtm) {
  for (int r = 0; r < p->n_rep; r++) {
    const int t = p->rep_type[r];
    const sqo_psd *P = &psd[t];
    const int nlocc = P->nlocc, S = 2 * nlocc + 1, nnd = S * S * S, len = P->size;
    const double *G = P->tables, *rVloc = G + len, *DVloc = G + 10 * len;
    const double ax = p->rep_xyz[3 * r], ay = p->rep_xyz[3 * r + 1], az = p->rep_xyz[3 * r + 2];
    const int inn = nearest_node(ax, p->delta), jnn = nearest_node(ay, p->delta), knn = nearest_node(az, p->delta);
    double *out = udvtm + p->rep_off[r];
    int cnt = 0;
    for (int l = 0; l <= P->lmax; l++) {
      if (l == P->lloc) continue;
      const double *rV = G + (2 + l) * len, *rU = G + (6 + l) * len;
      const double *DV = G + (11 + l) * len, *DU = G + (15 + l) * len;
      for (int m = -l; m <= l; m++, cnt++) {
        int ctr = 0;
        for (int kk = -nlocc; kk <= nlocc; kk++)
          for (int jj = -nlocc; jj <= nlocc; jj++)
            for (int ii = -nlocc; ii <= nlocc; ii++, ctr++) {
              double xr = (inn + ii) * p->delta - ax, yr = (jnn + jj) * p->delta - ay, zr = (knn + kk) * p->delta - az;
              double rad = sqrt(xr * xr + yr * yr + zr * zr);
              double VlocJ, VlJ, UlJ;
              if (spline_at(G, rVloc, DVloc, len, rad, &VlocJ) || spline_at(G, rV, DV, len, rad, &VlJ) ||
                  spline_at(G, rU, DU, len, rad, &UlJ))
                return -5;
              if (fabs(rad - 0.0) < TEMP_TOL) {
                VlocJ = rVloc[1] / G[1];
                VlJ = rV[1] / G[1];
                UlJ = rU[1] / G[1];
              } else {
                VlocJ = VlocJ / rad;
                VlJ = VlJ / rad;
                UlJ = UlJ / rad;
              }
              out[(size_t)cnt * nnd + ctr] = UlJ * real_sh(xr, yr, zr, rad, l, m) * (VlJ - VlocJ);
            }
      }
    }
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Pseudocharge density and local forces                                  */
/* ---------------------------------------------------------------------- */

/* VlocJ and VlocJ_tilda of one replica at a grid node (initialize.cpp:565-597,
 * forces.cpp:116-143): the spline of r Vloc divided by r (the first table
 * point's ratio at the nucleus) and the smooth reference potential of
 * radius rc_tilda.  *rad receives r. */
static int vloc_at(const sqo_local *L, int t, const double *c, double h, int gi, int gj, int gk, double *v,
                   double *vt, double *rad) {
  const double *G = L->typ_tab[t], *rV = G + L->typ_size[t], *DV = G + 2 * (size_t)L->typ_size[t];
  const double dx = gi * h - c[0], dy = gj * h - c[1], dz = gk * h - c[2];
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  double s;
  if (spline_at(G, rV, DV, L->typ_size[t], r, &s)) return -1;
  *v = fabs(r - 0.0) < TEMP_TOL ? rV[1] / G[1] : s / r;
  const double rc = L->rc_tilda, Z = L->Z[t];
  if (r < rc)
    *vt = -Z * (9 * pow(r, 7) - 30 * rc * pow(r, 6) + 28 * rc * rc * pow(r, 5) - 14 * pow(rc, 5) * pow(r, 2) +
                12 * pow(rc, 7)) /
          (5 * pow(rc, 8));
  else
    *vt = -Z / r;
  *rad = r;
  return 0;
}

/* -(1/4 pi) Lap_h of a box field at box index (i, j, k) (the stencil of
 * initialize.cpp:604-614 and forces.cpp:154-170). */
static double neg_lap(const sqo_problem *p, const double *f, int nx, int ny, int i, int j, int k) {
  const double *cl = p->coeff_lap;
#define F(ii, jj, kk) f[((size_t)(kk) * ny + (jj)) * nx + (ii)]
  double s = F(i, j, k) * 3 * cl[0] * (-1 / (4 * M_PI));
  for (int a = 1; a <= p->fdn; a++)
    s += (F(i - a, j, k) + F(i + a, j, k) + F(i, j - a, k) + F(i, j + a, k) + F(i, j, k - a) + F(i, j, k + a)) * cl[a] *
         (-1 / (4 * M_PI));
#undef F
  return s;
}

int sqo_charge_density(const sqo_problem *p, const sqo_local *L, double *b, double *b_tilda, double *vc,
                       double *rho_at, double *scal) {
  const int NX = p->np[0], NY = p->np[1], NZ = p->np[2], fdn = p->fdn;
  const size_t N = (size_t)NX * NY * NZ;
  const double h = p->delta;
  memset(b, 0, N * sizeof(double));
  memset(b_tilda, 0, N * sizeof(double));
  memset(vc, 0, N * sizeof(double));
  memset(rho_at, 0, N * sizeof(double));
  double Eself = 0.0, Ncharge = 0.0, Nel = 0.0, Eself_t = 0.0, Ncharge_t = 0.0, Vcon = 0.0;
  for (int r = 0; r < L->n_rep; r++) {
    const int t = L->rep_type[r];
    const int *bx = L->rep_box + 6 * r;
    const double *c = L->rep_xyz + 3 * r;
    const double *G = L->typ_tab[t], *U = G + 3 * (size_t)L->typ_size[t], *DU = G + 4 * (size_t)L->typ_size[t];
    const int nx = bx[1] - bx[0] + 1 + 2 * fdn, ny = bx[3] - bx[2] + 1 + 2 * fdn, nz = bx[5] - bx[4] + 1 + 2 * fdn;
    const int i0 = bx[0] - fdn, j0 = bx[2] - fdn, k0 = bx[4] - fdn;
    double *V = malloc(sizeof(double) * nx * ny * nz), *Vt = malloc(sizeof(double) * nx * ny * nz);
    /* initialize.cpp:565-597 */
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          const size_t q = ((size_t)k * ny + j) * nx + i;
          double rad;
          if (vloc_at(L, t, c, h, i0 + i, j0 + j, k0 + k, &V[q], &Vt[q], &rad)) {
            free(V);
            free(Vt);
            return -1;
          }
          if (i >= fdn && i < nx - fdn && j >= fdn && j < ny - fdn && k >= fdn && k < nz - fdn) {
            double rho_temp;
            if (spline_at(G, U, DU, L->typ_size[t], rad, &rho_temp)) {
              free(V);
              free(Vt);
              return -1;
            }
            rho_at[((size_t)(k + k0 - p->pnode_s[2]) * NY + (j + j0 - p->pnode_s[1])) * NX + (i + i0 - p->pnode_s[0])] +=
                rho_temp;
            Nel += rho_temp * h * h * h;
          }
        }
    /* initialize.cpp:600-628 */
    for (int k = bx[4]; k <= bx[5]; k++)
      for (int j = bx[2]; j <= bx[3]; j++)
        for (int i = bx[0]; i <= bx[1]; i++) {
          const int ii = i - i0, jj = j - j0, kk = k - k0;
          const size_t q = ((size_t)kk * ny + jj) * nx + ii;
          const double bt = neg_lap(p, V, nx, ny, ii, jj, kk), btt = neg_lap(p, Vt, nx, ny, ii, jj, kk);
          const size_t g = ((size_t)(k - p->pnode_s[2]) * NY + (j - p->pnode_s[1])) * NX + (i - p->pnode_s[0]);
          b[g] += bt;
          Eself += 0.5 * bt * V[q] * h * h * h;
          Ncharge += bt * h * h * h;
          b_tilda[g] += btt;
          Eself_t += 0.5 * btt * Vt[q] * h * h * h;
          Ncharge_t += btt * h * h * h;
          vc[g] += Vt[q] - V[q];
        }
    /* initialize.cpp:631-635: Vcon at the main domain's first node */
    if (bx[0] <= 0 && bx[1] >= 0 && bx[2] <= 0 && bx[3] >= 0 && bx[4] <= 0 && bx[5] >= 0) {
      const size_t q = ((size_t)(0 - k0) * ny + (0 - j0)) * nx + (0 - i0);
      Vcon += Vt[q] - V[q];
    }
    free(V);
    free(Vt);
  }
  /* initialize.cpp:729-780 (one rank: the reductions are the local sums,
   * V000 and Vcon the block's own) */
  const double s = fabs(Ncharge / Ncharge_t), V000 = vc[0], h3 = pow(h, 3);
  double Ecorr = 0.0;
  for (size_t g = 0; g < N; g++) b_tilda[g] = s * b_tilda[g];
  for (size_t g = 0; g < N; g++) {
    vc[g] += -V000 + Vcon;
    Ecorr += 0.5 * (b_tilda[g] + b[g]) * vc[g] * h3;
  }
  scal[0] = Eself;
  scal[1] = Ncharge;
  scal[2] = Nel;
  scal[3] = Ncharge_t;
  scal[4] = Eself_t;
  scal[5] = Vcon;
  scal[6] = Ecorr + Eself - Eself_t;
  return 0;
}

int sqo_forces_local(const sqo_problem *p, const sqo_local *L, const double *phi, const double *vc, const double *b,
                     const double *b_tilda, double *floc, double *fcorr) {
  const int NX = p->np[0], NY = p->np[1], fdn = p->fdn;
  const int PX = NX + 2 * fdn, PY = NY + 2 * fdn;
  const double h = p->delta, h3 = pow(h, 3);
  const double *cg = p->coeff_grad;
  memset(floc, 0, sizeof(double) * 3 * p->n_atm);
  memset(fcorr, 0, sizeof(double) * 3 * p->n_atm);
  for (int r = 0; r < L->n_rep; r++) {
    const int t = L->rep_type[r], atom = L->rep_atom[r];
    const int *bx = L->rep_box + 6 * r;
    const double *c = L->rep_xyz + 3 * r;
    const int nx = bx[1] - bx[0] + 1 + 4 * fdn, ny = bx[3] - bx[2] + 1 + 4 * fdn, nz = bx[5] - bx[4] + 1 + 4 * fdn;
    const int i0 = bx[0] - 2 * fdn, j0 = bx[2] - 2 * fdn, k0 = bx[4] - 2 * fdn;
    const size_t nb = (size_t)nx * ny * nz;
    double *V = malloc(sizeof(double) * nb), *Vt = malloc(sizeof(double) * nb);
    double *bJ = calloc(nb, sizeof(double)), *bJt = calloc(nb, sizeof(double));
    /* forces.cpp:116-143 */
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          const size_t q = ((size_t)k * ny + j) * nx + i;
          double rad;
          if (vloc_at(L, t, c, h, i0 + i, j0 + j, k0 + k, &V[q], &Vt[q], &rad)) {
            free(V);
            free(Vt);
            free(bJ);
            free(bJt);
            return -1;
          }
        }
    /* forces.cpp:149-173 */
    for (int k = fdn; k < nz - fdn; k++)
      for (int j = fdn; j < ny - fdn; j++)
        for (int i = fdn; i < nx - fdn; i++) {
          const size_t q = ((size_t)k * ny + j) * nx + i;
          bJ[q] = neg_lap(p, V, nx, ny, i, j, k);
          bJt[q] = neg_lap(p, Vt, nx, ny, i, j, k);
        }
    /* forces.cpp:178-277: per direction the gradients of bJ, bJ_tilda, VlocJ,
     * VlocJ_tilda and the two force terms */
    for (int k = 2 * fdn; k < nz - 2 * fdn; k++)
      for (int j = 2 * fdn; j < ny - 2 * fdn; j++)
        for (int i = 2 * fdn; i < nx - 2 * fdn; i++) {
          const size_t q = ((size_t)k * ny + j) * nx + i;
          const int gi = i + i0 - p->pnode_s[0], gj = j + j0 - p->pnode_s[1], gk = k + k0 - p->pnode_s[2];
          const double ph = phi[((size_t)(gk + fdn) * PY + (gj + fdn)) * PX + (gi + fdn)];
          const size_t g = ((size_t)gk * NY + gj) * NX + gi;
          const size_t stride[3] = {1, (size_t)nx, (size_t)nx * ny};
          for (int d = 0; d < 3; d++) {
            const size_t s = stride[d];
            double Db = 0, Dbt = 0, DV = 0, DVt = 0;
            for (int a = 1; a <= fdn; a++) Db += (-bJ[q - a * s] + bJ[q + a * s]) * cg[a];
            floc[3 * atom + d] += Db * (ph - V[q]) * h3;
            for (int a = 1; a <= fdn; a++) Dbt += (-bJt[q - a * s] + bJt[q + a * s]) * cg[a];
            for (int a = 1; a <= fdn; a++) DV += (-V[q - a * s] + V[q + a * s]) * cg[a];
            for (int a = 1; a <= fdn; a++) DVt += (-Vt[q - a * s] + Vt[q + a * s]) * cg[a];
            fcorr[3 * atom + d] += 0.5 *
                                   (Dbt * (vc[g] - Vt[q]) + Db * (vc[g] + V[q]) + (DVt - DV) * (b_tilda[g] + b[g]) +
                                    bJ[q] * DV - bJt[q] * DVt) *
                                   h3;
          }
        }
    free(V);
    free(Vt);
    free(bJ);
    free(bJt);
  }
  return 0;
}
