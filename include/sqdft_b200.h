/* sqdft_b200: B200 (sm_100a) implementation of SQDFT's spectral-quadrature
 * density / energy / nonlocal-force step, behind a C ABI.
 *
 * One context (sqb_ctx) holds one processor block of the SQDFT grid -- the
 * whole periodic domain on a single GPU -- with its Veff, atoms and projector
 * tables resident in HBM.  Every entry point replaces one reference function
 * (cited as file:line of the SQDFT sources) and keeps its argument meaning;
 * arrays are plain host pointers in the reference's own layouts:
 *   node nd = (k*np_y + j)*np_x + i            (sq.cpp:530-535)
 *   rho      [np_z][np_y][np_x]                 (DS_SQ::rho)
 *   rho_pj, Ci [nnode][npl+1]                   (DS_SQ::rho_pj, DS_SQ::Ci)
 *   chi, zee [nnode]                            (DS_SQ::chi, DS_SQ::zee)
 *   veff     [np_z+2nloc][np_y+2nloc][np_x+2nloc], halo filled
 *                                               (DS_SQ::Veff, initialize.cpp:940)
 *   forces   [n_atm][3], atoms type-major       (fnlocx/y/z, forces.cpp:504-527)
 * All functions return SQB_OK (0) or one of the SQB_ERR_* codes; none of them
 * exits the process.  A context is used by one host thread at a time.
 */
#ifndef SQDFT_B200_H
#define SQDFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference prints and exit(1)s in the cases marked. */
#define SQB_OK 0
#define SQB_ERR_ARG 1              /* bad argument or size */
#define SQB_ERR_CUDA 2             /* CUDA runtime error or no device */
#define SQB_ERR_UNSUPPORTED 3      /* configuration outside what the kernels cover */
#define SQB_ERR_NOT_BRACKETED 4    /* sq.cpp:1307-1311, Brent root not bracketed */
#define SQB_ERR_FERMI_MAXITER 5    /* sq.cpp:1400-1401, Brent iteration limit */
#define SQB_ERR_NEGATIVE_RHO 6     /* sq.cpp:764-765, rho < -1e-6 */
#define SQB_ERR_LANCZOS_MAXITER 7  /* not returned: a node whose Lanczos hits 500
                                      iterations keeps its last Ritz values and is
                                      counted in sqb_stats.lanczos_maxiter_nodes, as
                                      the reference prints and carries on
                                      (sq.cpp:1073-1074) */
#define SQB_ERR_DENOM_ZERO 8       /* nonlocal.cpp:163, zero KB denominator */
#define SQB_ERR_SPLINE_RANGE 9     /* spline.cpp:17-22, radius outside the radial grid */
#define SQB_ERR_CAPACITY 10        /* more projector atoms in one window than supported */
#define SQB_ERR_NONFINITE 11       /* NaN or Inf met in inputs or in a result */
#define SQB_ERR_STATE 12           /* entry point called before its inputs were set */
#define SQB_ERR_BOUNDS 13          /* a device index check failed (the bounds-check build,
                                      libsqdft_b200_bc.so, only) */

/* Precision of the recursion vectors (Chebyshev and Lanczos). */
#define SQB_FP64 0        /* everything in FP64: parity path */
#define SQB_FP32_MIXED 1  /* Lanczos vectors (and the nonlocal-force recursion
                             vectors) stored in FP32, stencil arms summed in FP32;
                             Veff, projector tables, the rest of the arithmetic,
                             the Chebyshev moments, coefficients, Fermi solve and
                             assembly in FP64.  Lanczos stops at
                             max(lanczos_tol, sqb_set_mixed_lanczos tol). */
#define SQB_FP64_LANCZOS_QUAD 2 /* FP64; bounds and Chebyshev moments of each node
                             from one Lanczos run started at the node's unit
                             vector: its tridiagonal T_m gives mu_j = e_1^T
                             T_j((T_m - chi)/zee) e_1 exactly for j <= 2m - 1
                             (m >= npl/2 + 1 steps), its extreme Ritz values
                             the bounds (stop and margin as for SQB_FP32_MIXED).
                             Same moments as the reference at slightly
                             different bounds; no counterpart in the reference. */

typedef struct sqb_ctx sqb_ctx;

/* Grid and SQ parameters: the DS_SQ fields of ds_sq.h:133-161. */
typedef struct sqb_grid {
  int np[3];      /* np_x, np_y, np_z: nodes of this block */
  int pnode_s[3]; /* global index of the block's first node */
  int n_int[3];   /* global grid intervals (periodic) */
  int nloc;       /* ceil(Rcut/delta), readfiles.cpp:306 */
  int fdn;        /* half FD order; the kernels support 6 (12th order) */
  int npl;        /* Chebyshev degree, multiple of 4 (sq.cpp:523) */
  int fermi_alg;  /* 1 Brent, 2 Newton-Raphson */
  double delta, bet, lanczos_tol, fermi_tol, ncharge;
  double coeff_lap[8];  /* coeff_lap[0..fdn], readfiles.cpp:371-381 */
  double coeff_grad[8]; /* coeff_grad[0..fdn], readfiles.cpp:384-389 */
} sqb_grid;

/* One atom type: DS_Psd (ds_sq.h:76-102) + DS_Atm fields. */
typedef struct sqb_species {
  int natm, lmax, lloc;
  int nlocc;       /* ceil(rc/delta), nonlocal.cpp:43 */
  int size;        /* radial grid length */
  double rc;
  double denom[4]; /* Denom_s, Denom_p, Denom_d, Denom_f */
  /* 19 x size rows: RadialGrid, rVloc, rVs, rVp, rVd, rVf, rUs, rUp, rUd, rUf,
   * DVloc, DVsJ, DVpJ, DVdJ, DVfJ, DUsJ, DUpJ, DUdJ, DUfJ; may be NULL when the
   * projector tables are supplied by sqb_set_projectors. */
  const double *tables;
} sqb_species;

/* Reduction operators of the allreduce hook. */
#define SQB_SUM 0
#define SQB_MIN 1
#define SQB_MAX 2

/* Reduce `count` doubles across ranks in place: MPI_Allreduce with MPI_SUM
 * in the reference (sq.cpp:1219, 1442, 792; forces.cpp:623) and the
 * MPI_Allgather + min/max of the Lanczos bounds (sq.cpp:676-713).  Return 0
 * on success.  Unset means a single rank. */
typedef int (*sqb_allreduce_fn)(double *values, int count, int op, void *user);

/* Timings and counters of the last calls (CUDA events on the context's
 * stream, milliseconds). */
typedef struct sqb_stats {
  double ms_lanczos_moments; /* node kernel of the last SQ call */
  double ms_fermi;           /* Fermi-level solve */
  double ms_density;         /* density / energy assembly */
  double ms_forces;          /* nonlocal-force kernel + reduction */
  double ms_projectors;      /* projector tables */
  long long matvecs;         /* window matvecs in the last node kernel */
  long long lanczos_iters;   /* sum of Lanczos iterations over nodes */
  long long window_points;   /* (2nloc+1)^3 */
  long long proj_points;     /* sum over nodes and matvec steps of the projector-ball points of the
                                atoms meeting the window (n_proj * n_b per atom, algorithmic) */
  long long proj_points_cheb; /* the same over the Chebyshev steps only */
  int fermi_iters;
  int max_lanczos_iters;
  int kernel_launches;       /* kernels launched by the last SQ or forces call */
  double ms_vjp;             /* adjoint node kernel of the last sqb_moments_vjp */
  double ms_defect;          /* defect check of a fast form in the last SQ step (its
                                sensitivity kernel, FP64 redo and superseded Fermi solve) */
  long long defect_nodes;    /* nodes the last SQ step's defect check redid in FP64 */
  long long lanczos_maxiter_nodes; /* nodes of the last node kernel whose Lanczos stopped at
                                      the 500-iteration cap (sq.cpp:1073-1074 prints them) */
  long long proj_points_window; /* as proj_points, with each ball clipped to the window (the
                                   projector values a matvec reads) */
  int node_kernel;           /* kernel of the last Lanczos + moments work: SQB_KERNEL_PLANE or
                                SQB_KERNEL_SWEEP */
  double ms_charge_density;  /* kernels of the last sqb_charge_density */
  double ms_forces_local;    /* kernels of the last sqb_forces_local */
} sqb_stats;

/* Create a context on CUDA device `device` (cudaSetDevice).  Mirrors the
 * per-call allocations of sq.cpp:496-517 with resident device buffers. */
int sqb_create(const sqb_grid *grid, int device, sqb_ctx **out);
int sqb_destroy(sqb_ctx *ctx);
int sqb_set_precision(sqb_ctx *ctx, int precision);
/* Lanczos of the FP32-mixed and Lanczos-quadrature forms.  tol: stopping
 * tolerance (Ha), also the margin put around the Ritz values (sq.cpp:1050-1092
 * with this tolerance); default 0, i.e. sqb_grid.lanczos_tol.  The density's
 * sensitivity to the bounds falls with npl: a looser stop suits high-order
 * expansions only.  checkerboard in [0, 1] (FP32-mixed form): start vector
 * 1 + c (-1)^(x+y+z), normalised, in place of the reference's constant vector
 * (sq.cpp:538-546); its overlap with the top of the spectrum speeds the
 * convergence of lambda_max; default 0.5.  The FP64 path always uses the
 * reference's start vector and sqb_grid.lanczos_tol.  No counterpart in the
 * reference. */
int sqb_set_mixed_lanczos(sqb_ctx *ctx, double tol, double checkerboard);
/* Density budget of the fast forms' defect check (relative to max rho, e.g.
 * 1e-6; default 0, the check off).  When a fast form's Lanczos stop is
 * looser than sqb_grid.lanczos_tol, sqb_spectral_quadrature evaluates every
 * node's density at bounds moved by 4x the stop at either end, from the
 * node's own moments (exact re-expansion of the Chebyshev polynomials, no
 * matvec); nodes that move by more than half the budget are redone by the
 * FP64 parity path and the Fermi level is solved again (the count is in
 * sqb_stats.defect_nodes).  The 4x widening is conservative: where the
 * looser stop already meets the budget it still redoes a share of the nodes
 * (17% at npl 96, 40% of the step's time), hence opt-in.  No counterpart in
 * the reference. */
int sqb_set_defect_check(sqb_ctx *ctx, double budget);
int sqb_set_allreduce(sqb_ctx *ctx, sqb_allreduce_fn fn, void *user);
/* Launch shape of the node kernel: persistent CTAs per SM, and the layout of
 * its plane loop: window columns per thread (1 or 2; 0 = automatic, one
 * column per thread when the window has at most 1024 columns), or -2 for the
 * row layout (a warp per two window rows, windows up to 32 wide). */
int sqb_set_launch(sqb_ctx *ctx, int ctas_per_sm, int cols_per_thread);

/* Kernel of the per-node Lanczos bounds and Chebyshev moments (the node loop
 * of sq.cpp:530-661).  SQB_KERNEL_SWEEP: one plane sweep per matvec with the
 * nonlocal term read from layered projector fields (per grid point, the
 * projector of at most one ball in each of four layers of non-touching
 * balls), the dot products accumulated along z; it covers systems whose
 * balls split into four such layers (the FCC sublattices) with at most three
 * projectors per type.  SQB_KERNEL_PLANE: the plane-streaming kernel with
 * per-window box lists, any system.  SQB_KERNEL_AUTO (default): the sweep
 * kernel where it covers the system.  Results agree to rounding.  The nonlocal
 * forces, the adjoint, sqb_moments_at, sqb_hsub_times_vec and
 * sqb_lanczos_moments_noalloc run the plane-streaming kernel.  No counterpart
 * in the reference. */
#define SQB_KERNEL_AUTO 0
#define SQB_KERNEL_PLANE 1
#define SQB_KERNEL_SWEEP 2
int sqb_set_node_kernel(sqb_ctx *ctx, int kernel);
/* Window rows per thread of the sweep kernel: 2 (one column and two rows per
 * thread, the default), 3 (fewer threads, more registers each; windows up to
 * 33 wide), or 0 for the default.  Results agree to rounding (the block
 * reductions sum in another order). */
int sqb_set_sweep_rows(sqb_ctx *ctx, int rows);
/* Times the SQ node work on the sweep kernel with two and with three rows
 * per thread on `sample` evenly spaced nodes (0: two per SM), keeps the
 * faster for the context; *rows the choice, ms[2] the times (-1 where a
 * variant does not apply).  SQB_ERR_UNSUPPORTED when the sweep kernel does
 * not cover the context. */
int sqb_autotune_sweep(sqb_ctx *ctx, int sample, int *rows, double *ms);

/* Test hook of the plane-streaming kernel's bounded waits (its projector
 * table planes arrive by bulk copies whose completion each plane waits for,
 * bounded in time).  extra_bytes (a multiple of 16, at most 4096) is added
 * to every stage's expected byte count, so no stage completes; wait_ms
 * replaces the 2 s wait limit (0 restores it).  A launch then ends with
 * SQB_ERR_CUDA after about wait_ms plus a 1 ms grace for the copies already
 * issued, with no copy in flight, and the context stays usable.  (0, 0)
 * turns the hook off.  No counterpart in the reference. */
int sqb_test_stage_wait(sqb_ctx *ctx, unsigned extra_bytes, double wait_ms);

/* CUDA-graph replay.  on = 1: the node-kernel sequence of
 * sqb_lanczos_moments (work-queue and status resets, the persistent Lanczos +
 * Chebyshev launch and the bound min/max), captured on the first call after
 * a plain run has allocated their buffers and replayed afterwards; the
 * Fermi-level solve stays host-driven (one launch per Brent or Newton trial).
 * on = 2: in addition sqb_spectral_quadrature runs the whole step as one
 * graph -- node kernel, min/max, the Fermi solve as a conditional while node
 * (NeConstraint, then a one-thread step of Brent's or Newton's method, the
 * host solvers' control flow and arithmetic, which sets the loop condition;
 * at most 512 evaluations) and the density assembly -- with one launch and
 * one synchronisation per step; single rank (no allreduce hook), sweep kernel
 * and no active defect check, else the plain path runs.  In graph mode 2 the
 * step's whole device time is reported in sqb_stats.ms_lanczos_moments.
 * Graphs are dropped when atoms, launch layout or precision change.
 * 0 = plain launches (default). */
int sqb_set_graph(sqb_ctx *ctx, int on);

/* Autotuner of the node kernel's plane-loop layout: times the Lanczos +
 * moments kernel on `sample` evenly spaced nodes (0 = two per SM) with every
 * layout the window allows -- one or two window columns per thread, and the
 * row layout for windows up to 32 wide -- and keeps the fastest for the
 * context, as sqb_set_launch(ctx, 0, layout) would.  *chosen receives the
 * layout; ms_out (3 doubles, or NULL) the sample times for 1, 2 and -2
 * (negative where a layout does not apply).  The sample runs overwrite part
 * of the per-node outputs, so run sqb_lanczos_moments (or the SQ step)
 * afterwards.  Results do not depend on the layout.  No counterpart in the
 * reference. */
int sqb_autotune(sqb_ctx *ctx, int sample, int *chosen, double *ms_out);

/* Veff on the block with its Rcut halo: the state of DS_SQ::Veff after the
 * halo exchange of sq.cpp:400-492. */
int sqb_set_veff(sqb_ctx *ctx, const double *veff_ext);
/* sqb_set_veff from device memory of the context's device (the same layout),
 * for callers that hold Veff on the GPU, e.g. after a broadcast of the
 * whole-grid potential to every rank's GPU.  Ordered after the work queued on
 * the legacy default stream; the buffer may be reused when it returns.  The
 * values are not checked on the host: a non-finite Veff surfaces as
 * SQB_ERR_NONFINITE from the next step. */
int sqb_set_veff_device(sqb_ctx *ctx, const double *veff_ext_device);

/* Atom types and the replica atoms whose rc-ball meets the block + Rcut
 * region (Replica_atoms_Rcut, initialize.cpp:1003-1196), type-major as
 * DS_Atm::R{x,y,z}[a].ProcAtmRcut[r] lists them.  rep_atom is the global
 * type-major atom index the force is accumulated into. */
int sqb_set_atoms(sqb_ctx *ctx, int n_typ, const sqb_species *types, int n_rep, const int *rep_type,
                  const int *rep_atom, const double *rep_xyz, int n_atm);

/* NonlocalProjectors (nonlocal.cpp:317-518): UdVtm on every replica's ball,
 * computed on the device from the radial tables.  If udvtm_out is not NULL
 * the tables are also copied out, concatenated in replica order, each
 * [nproj][(2nlocc+1)^3] as DS_ProcAtmRcut::UdVtm holds them. */
int sqb_nonlocal_projectors(sqb_ctx *ctx, double *udvtm_out);
/* Upload projector tables computed elsewhere (same layout as above). */
int sqb_set_projectors(sqb_ctx *ctx, const double *udvtm);

/* HsubTimesVec (sq.cpp:838-929) for `count` block nodes: vin and vout are
 * [count][(2nloc+1)^3] window vectors. */
int sqb_hsub_times_vec(sqb_ctx *ctx, int count, const int *nodes, const double *vin, double *vout);

/* Lanczos bounds (LanczosAlgorithm, sq.cpp:965-1092) and Chebyshev moments
 * (sq.cpp:530-661) of every block node.  Any output pointer may be NULL. */
int sqb_lanczos_moments(sqb_ctx *ctx, double *chi, double *zee, double *rho_pj, int *lanczos_iters,
                        double *lambda_min, double *lambda_max);

/* The per-node body of the node loop of ClenshawCurtisSpectralQuadrature
 * (sq.cpp:530-661: Lanczos bounds and Chebyshev moments) for the `count`
 * block nodes listed in `nodes` only.  Outputs are per listed node: chi, zee,
 * lanczos_iters [count], rho_pj [count][npl+1]; any may be NULL.  The
 * context's moments of the other nodes are left stale, so call
 * sqb_lanczos_moments before sqb_fermi_level / sqb_density_energy. */
int sqb_lanczos_moments_nodes(sqb_ctx *ctx, int count, const int *nodes, double *chi, double *zee, double *rho_pj,
                              int *lanczos_iters);

/* NeConstraint (sq.cpp:1183-1228) on the moments of the last
 * sqb_lanczos_moments call: 2 h^3 sum rho_pj.c(lambda) - N_e, reduced over
 * ranks through the allreduce hook. */
int sqb_ne_constraint(sqb_ctx *ctx, double lambda_f, double *fval);

/* Fermi level as sq.cpp:669-731 finds it: BrentsAlgorithm (sq.cpp:1289) or
 * NewtonRaphson (sq.cpp:1459) by grid->fermi_alg.  For scf_iter <= 1 the
 * bracket is the global Lanczos range +-1, else lambda_warm +-2. */
int sqb_fermi_level(sqb_ctx *ctx, int scf_iter, double lambda_warm, double *lambda_f, int *iters);

/* Density, Fermi coefficients, band and entropy energies (sq.cpp:733-797). */
int sqb_density_energy(sqb_ctx *ctx, double lambda_f, double *rho, double *ci, double *ebs, double *eent);

/* ClenshawCurtisSpectralQuadrature (sq.cpp:377-834) end to end: the three
 * calls above.  lambda_f is the warm start in and the Fermi level out. */
int sqb_spectral_quadrature(sqb_ctx *ctx, int scf_iter, double *lambda_f, double *rho, double *rho_pj, double *ci,
                            double *chi, double *zee, double *ebs, double *eent);

/* ForcesNonLocal (forces.cpp:318-578) with chi, zee, Ci of the last
 * sqb_spectral_quadrature call (or given ones when not NULL). */
int sqb_forces_nonlocal(sqb_ctx *ctx, const double *chi, const double *zee, const double *ci, double *forces);

/* Chebyshev moments (sq.cpp:564-655) with given spectral bounds: the node
 * loop of ClenshawCurtisSpectralQuadrature with chi, zee [nnode] supplied
 * instead of computed by LanczosAlgorithm.  The bounds become the context's
 * (sqb_density_energy and sqb_moments_vjp use them).  rho_pj may be NULL. */
int sqb_moments_at(sqb_ctx *ctx, const double *chi, const double *zee, double *rho_pj);

/* Adjoint of the moments: given g_mu [nnode][npl+1] = dL/d rho_pj for a
 * scalar L (rho_pj as sqb_lanczos_moments returns it, divided by h^3), writes
 * g_veff = dL/dVeff on the Veff block with its halo (the layout of
 * sqb_set_veff) and, when g_atoms is not NULL, g_atoms = dL/dR [n_atm][3]
 * (type-major, the layout of sqb_forces_nonlocal) through the projector
 * tables, with the spectral bounds chi, zee of the last moments held fixed.
 * Computed by the reverse Chebyshev (Clenshaw) recursion with checkpoints
 * every 8 recursion vectors; the projector derivatives dchi/dR are central
 * differences (step 1e-4 bohr) of the projector tables.  Contributions of
 * different nodes to one Veff point or atom are added with atomics, so the
 * outputs vary between runs at rounding level.  No counterpart in the
 * reference. */
int sqb_moments_vjp(sqb_ctx *ctx, const double *g_mu, double *g_veff, double *g_atoms);

/* Forward and backward of a density loss L = sum_p w[p] rho[p] (the density
 * of the last sqb_density_energy, w per node of the block, reduced over
 * ranks), the bounds held fixed.  sqb_density_loss gives L.
 * sqb_density_loss_vjp gives grad_l * dL/dVeff on the Veff block with its halo
 * (layout of sqb_set_veff) and, when g_atoms is not NULL, grad_l * dL/dR
 * [n_atm][3]: one moment adjoint (sqb_moments_vjp) with weights
 * 2 grad_l (w_p - kappa h^3) sign(rho_p) c_j(p), where with
 * fixed_electrons = 0 the Fermi level is held (kappa = 0) and otherwise the
 * electron count (the SCF's constraint): kappa = (dL/dlambda) / (dN_e/dlambda),
 * the lambda-derivatives from the Chebyshev coefficients of beta f (1 - f) on
 * each node's interval.  Needs a prior sqb_density_energy (its Fermi level and
 * coefficients).  This pair is the forward/backward of a
 * torch.autograd.Function.  No counterpart in the reference. */
int sqb_density_loss(sqb_ctx *ctx, const double *w, double *loss);
int sqb_density_loss_vjp(sqb_ctx *ctx, const double *w, int fixed_electrons, double grad_l, double *g_veff,
                         double *g_atoms);

/* Pseudocharge density and local forces: the per-atom loops of
 * ChargeDensity (initialize.cpp:470-784) and ForcesLocal (forces.cpp:20-315)
 * on the device.  They need the block grid of the context only (delta,
 * coeff_lap, coeff_grad, np, pnode_s; fdn 6), not Veff or the projectors. */

/* One atom type of the pseudocharge: the radial tables ChargeDensity and
 * ForcesLocal spline (DS_Psd::RadialGrid, rVloc, uu) with the derivatives
 * getYD_gen gives them (initialize.cpp:506-510), and the valence charge. */
typedef struct sqb_local_species {
  int size;             /* radial grid length */
  double Z;             /* DS_Atm::Z */
  const double *tables; /* 5 x size rows: RadialGrid, rVloc, DVloc, uu, Duu */
} sqb_local_species;

/* The pseudocharge replicas: every atom image whose rb-box meets the block
 * (Replica_atoms, initialize.cpp:21-160), in the reference's loop order
 * (type, main atom, replica) as DS_Atm::R{x,y,z}[a].ProcAtm[r] lists them.
 * rep_box[6r..6r+5] = the intersection box xstart, xend, ystart, yend, zstart,
 * zend in global nodes (DS_ProcAtm::start/end), inside the block; rep_atom the
 * global type-major atom index; rc_tilda the reference charge radius
 * (DS_SQ::rc_tilda, 0.5 in ChargeDensity).  SQB_ERR_ARG for boxes outside the
 * block, SQB_ERR_UNSUPPORTED for fdn != 6. */
int sqb_set_local_atoms(sqb_ctx *ctx, int n_typ, const sqb_local_species *types, int n_rep, const int *rep_type,
                        const int *rep_atom, const double *rep_xyz, const int *rep_box, double rc_tilda, int n_atm);

/* ChargeDensity's pseudocharge part (initialize.cpp:470-784) on the block:
 * b, b_tilda (scaled by |Ncharge / Ncharge_tilda|), Vc (shifted by
 * -V000 + Vcon) and rho_at (the superposed atomic densities, from zero), each
 * np_z x np_y x np_x z-major host arrays (any may be NULL); scal[7] =
 * Eself, Ncharge, the integral of rho_at, Ncharge_tilda, Eself_tilda, Vcon,
 * Ecorr.  The sums go through the allreduce hook as the reference's
 * MPI_Allreduce (initialize.cpp:717-723, 770); V000 and Vcon come from the
 * block that holds the main domain's first node (the reference broadcasts
 * rank 0's).  b and rho_at equal the reference's bit for bit (each node sums
 * its replicas in the reference's order); b_tilda and Vc to rounding (pow).
 * The initial-guess handling of rho (MD step, restart, charge extrapolation)
 * stays with the caller. */
int sqb_charge_density(sqb_ctx *ctx, double *b, double *b_tilda, double *vc, double *rho_at, double *scal);

/* ForcesLocal (forces.cpp:20-315): the block's local forces floc and the
 * overlap-correction forces fcorr, [n_atm][3] host arrays, from phi (the
 * block with its fdn halo, (np_z+2fdn) x (np_y+2fdn) x (np_x+2fdn)), Vc, b and
 * b_tilda (block arrays).  Like the reference the result is this block's
 * part (no reduction across ranks). */
int sqb_forces_local(sqb_ctx *ctx, const double *phi, const double *vc, const double *b, const double *b_tilda,
                     double *floc, double *fcorr);

/* Size of the fixed device scratch array used by sqb_lanczos_moments_noalloc
 * (held on every GPU that loads the library, until the process exits). */
#define SQB_NOALLOC_SCRATCH_BYTES (64u << 20)

/* sqb_lanczos_moments without any GPU allocation during the call, for callers
 * that may not allocate device memory while they run: code inside an
 * allocator-managed framework that owns all device memory, or a host loop
 * that has to keep its memory footprint fixed.  No counterpart in the
 * reference.
 *
 * It runs the plane-streaming node kernel (SQB_KERNEL_PLANE) for the `count`
 * block nodes listed in host array `nodes`, but the kernel's per-CTA window
 * vectors, its work-queue counter and status word live in one fixed device
 * array of SQB_NOALLOC_SCRATCH_BYTES compiled into the library, not in
 * memory from cudaMalloc.  Inputs are the context's resident Veff, atoms and
 * projector tables; outputs go to caller-owned DEVICE arrays indexed by node
 * id (chi, zee: nnode doubles; rho_pj: nnode x (npl+1); lanczos_iters may be
 * NULL).  The call is synchronous and returns a status code; a window whose
 * scratch (plus the node list) does not fit the array is rejected with
 * SQB_ERR_CAPACITY.  The first call on a device looks up the array's device
 * address for that device, so make it before any stream capture.  All calls
 * in the process share the array: calls that overlap on the GPU (other
 * threads or streams) race and must be serialised by the caller.
 * Ordering: the kernel runs on the context's private non-blocking stream,
 * which first waits for the work queued so far on the legacy default stream
 * (stream 0, where torch and most callers queue by default), so writes the
 * caller queued there to the output arrays land before the kernel's.  Work
 * the caller queued on any other stream must have finished (or the caller
 * synchronises it) before the call. */
int sqb_lanczos_moments_noalloc(sqb_ctx *ctx, int count, const int *nodes, double *d_chi, double *d_zee,
                                double *d_rho_pj, int *d_lanczos_iters);

/* Counters and timings of the last calls.  out_size is sizeof(sqb_stats) as
 * the caller was compiled: the library writes min(out_size, its own size)
 * bytes, so a caller built against an older, shorter sqb_stats stays safe. */
int sqb_get_stats(const sqb_ctx *ctx, sqb_stats *out, size_t out_size);
const char *sqb_status_string(int status);
/* Library version string. */
const char *sqb_version(void);

#ifdef __cplusplus
}
#endif
#endif
