/* CPU restatement of SQDFT's spectral-quadrature (SQ) step.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker that the CUDA path is compared
 * with; nothing in the shipped library calls it.  Each function restates one
 * reference function with the same arithmetic order (file:line cited at the
 * definition), so that on the same inputs it agrees with the reference
 * compiled from source to rounding level.  Parity is pinned: the tests compare
 * it with outputs of the reference build (oracle/_ref/sqref_driver) and with
 * the reference's shipped regression log values.
 *
 * Layouts: a node is (i, j, k) in the processor block with nd = (k*ny + j)*nx + i
 * (x fastest, as the loops of sq.cpp:530-535); a window vector is
 * (2nloc+1)^3 values, z-major with x fastest; Veff is the block with its
 * Rcut halo, [nz+2nloc][ny+2nloc][nx+2nloc] (initialize.cpp:940-967).
 */
#ifndef SQB_ORACLE_H
#define SQB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sqo_problem {
  int np[3];       /* np_x, np_y, np_z */
  int pnode_s[3];  /* global index of the block's first node */
  int nloc, fdn, npl, fermi_alg;
  double delta, bet, lanczos_tol, fermi_tol, ncharge;
  const double *coeff_lap;  /* fdn+1 */
  const double *coeff_grad; /* fdn+1 */
  const double *veff;       /* block + halo */
  int n_typ;
  const int *typ_nlocc, *typ_nproj, *typ_lmax, *typ_lloc;
  const double *typ_denom; /* [n_typ][4]: Denom_s, _p, _d, _f */
  int n_rep;
  const int *rep_type, *rep_atom; /* replica -> type, global (type-major) atom index */
  const double *rep_xyz;          /* [n_rep][3] */
  const double *udvtm;            /* concatenated [nproj][ball^3] tables, replica order */
  const long long *rep_off;       /* start of each replica's table in udvtm */
  int n_atm;
} sqo_problem;

/* Radial tables of one type: rows grid, rVloc, rV_{s,p,d,f}, rU_{s,p,d,f},
 * DVloc, DV_{s,p,d,f}, DU_{s,p,d,f} (19 x size), as DS_Psd holds them. */
typedef struct sqo_psd {
  int size, lmax, lloc, nlocc;
  const double *tables;
} sqo_psd;

/* Worker threads for sqo_lanczos_moments (nodes are independent). */
void sqo_set_threads(int n);
/* NonlocalProjectors (nonlocal.cpp:317-518) for every replica. */
int sqo_projectors(const sqo_problem *p, const sqo_psd *psd, double *udvtm_out);
/* HsubTimesVec (sq.cpp:838-929) at block node nd. */
void sqo_hsub_times_vec(const sqo_problem *p, int nd, const double *v, double *hv);
/* LanczosAlgorithm (sq.cpp:965-1092); returns the iteration count. */
int sqo_lanczos(const sqo_problem *p, int nd, double *lambda_min, double *lambda_max);
/* TridiagEigenSolve (sq.cpp:1094-1180); returns 0, or -1 after 200 sweeps. */
int sqo_tridiag_eigen(const double *diag, const double *subdiag, int n, double *lmin, double *lmax);
/* Chebyshev moments of one node (sq.cpp:564-655): rho_pj[0..npl]. */
void sqo_moments(const sqo_problem *p, int nd, double chi, double zee, double *rho_pj);
/* Lanczos + moments for nodes[0..count): chi, zee, rho_pj rows and
 * Lanczos counts written at each node's slot (indexed by node id). */
int sqo_lanczos_moments(const sqo_problem *p, const int *nodes, int count, double *chi, double *zee,
                        double *rho_pj, int *lanczos_iters, double *lmin_out, double *lmax_out);
/* ChebyshevCoeff (sq.cpp:1230-1259); kind 0 FermiDirac, 1 UbandFunc,
 * 2 EentFunc, 3 FermiDirac_derv. */
void sqo_chebyshev_coeff(int npl, double lambda_fp, double bet, double *ci, int kind);
/* NeConstraint (sq.cpp:1183-1228) over all block nodes. */
double sqo_ne_constraint(const sqo_problem *p, const double *chi, const double *zee, const double *rho_pj,
                         double lambda_f);
/* Fermi level as ClenshawCurtisSpectralQuadrature finds it (sq.cpp:669-731):
 * Brent (sq.cpp:1289-1404) or Newton (sq.cpp:1459-1490).  lmin/lmax are the
 * global Lanczos extremes (used when scf_iter <= 1).  Returns 0 or a
 * negative error (-2 not bracketed, -3 iteration limit). */
int sqo_fermi_level(const sqo_problem *p, const double *chi, const double *zee, const double *rho_pj,
                    int scf_iter, double lambda_warm, double lmin, double lmax, double *lambda_f,
                    int *iters);
/* Density, Ci, Ebs, Eent (sq.cpp:733-797); returns 0 or -4 (negative rho). */
int sqo_density_energy(const sqo_problem *p, const double *chi, const double *zee, const double *rho_pj,
                       double lambda_f, double *rho, double *ci, double *ebs, double *eent);
/* ForcesNonLocal (forces.cpp:318-578) for nodes[0..count): adds into f[n_atm][3]. */
int sqo_forces_nonlocal(const sqo_problem *p, const int *nodes, int count, const double *chi, const double *zee,
                        const double *ci, double *f);

/* Pseudocharge replicas of ChargeDensity and ForcesLocal: the atoms whose
 * rb-box meets the block (Replica_atoms, initialize.cpp:21-160), in the
 * functions' loop order (type, main atom, replica). */
typedef struct sqo_local {
  int n_typ;
  const int *typ_size;            /* radial grid length per type */
  const double *const *typ_tab;   /* per type [5][size]: grid, rVloc, DVloc, uu, Duu */
  const double *Z;                /* valence charge per type */
  int n_rep;
  const int *rep_type, *rep_atom; /* replica -> type, global (type-major) atom index */
  const double *rep_xyz;          /* [n_rep][3] */
  const int *rep_box;             /* [n_rep][6]: xstart, xend, ystart, yend, zstart, zend (global nodes) */
  double rc_tilda;
} sqo_local;

/* The pseudocharge part of ChargeDensity (initialize.cpp:470-784) on one
 * block: b, b_tilda (scaled), Vc (shifted), rho_at (accumulated from zero),
 * and scal[7] = Eself, Ncharge, Nelectron of rho_at, Ncharge_tilda,
 * Eself_tilda, Vcon, Ecorr.  Returns 0 or -1 (spline out of range). */
int sqo_charge_density(const sqo_problem *p, const sqo_local *L, double *b, double *b_tilda, double *vc,
                       double *rho_at, double *scal);
/* ForcesLocal (forces.cpp:20-315): floc and fcorr [n_atm][3] from phi (block
 * with its FDn halo), Vc, b and b_tilda.  Returns 0 or -1. */
int sqo_forces_local(const sqo_problem *p, const sqo_local *L, const double *phi, const double *vc, const double *b,
                     const double *b_tilda, double *floc, double *fcorr);

#ifdef __cplusplus
}
#endif
#endif
