// Internal declarations shared by the sqdft_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sqb {

constexpr int FDN = 6;           // 12th-order stencil, the order the configurations use
constexpr int MAXE = 128;        // projector-bearing replicas per node window
constexpr int MAXP = 512;        // projector instances (replica x (l,m)) per node window
constexpr int MAXL = 504;        // tridiagonal capacity: 500 Lanczos iterations + 2 (sq.cpp:967)
constexpr int LANCZOS_MAX_ITER = 500;
constexpr int MAXPROJ_TYPE = 16; // (l,m) pairs of one type, l <= 3
constexpr int FSLOTS = 8;        // replicas whose ball holds one node (force contributions)
constexpr int MAXN = 64;         // window edge 2*nloc+1

// Projector tables on the device: replica r's table starts at rep_off[r]
// (a multiple of 4 values) and holds, for each projector q and ball plane z,
// the Sd x Sd values [y][x] padded to plane_stride(Sd) values, so every
// (q, z) plane starts 16-byte aligned in FP32 and FP64:
//   value(q, z, y, x) = tab[rep_off[r] + (q*Sd + z)*plane_stride(Sd) + y*Sd + x].
// The reference's UdVtm holds the same values without the padding.
__host__ __device__ __forceinline__ int plane_stride(int Sd) { return (Sd * Sd + 3) & ~3; }

// Device-side status bits (or-ed by the kernels, mapped to SQB_ERR_* on the host).
enum : int {
  ST_CAPACITY = 1,
  ST_LANCZOS_MAXITER = 2,
  ST_NONFINITE = 4,
  ST_SPLINE_RANGE = 8,
  ST_FSLOTS = 16,
  ST_WAIT_LIMIT = 32,  // a bounded wait on an asynchronous copy ran out
  ST_BOUNDS = 64,      // an index check of the bounds-check build failed
};

// Index checks of the bounds-check build (-DSQB_BOUNDS_CHECK; build.py makes
// it as a second library beside the normal one): a failed check sets
// ST_BOUNDS in the status word and redirects the access to element 0 (inside
// every buffer), so the kernel runs on and the host returns SQB_ERR_BOUNDS.
// In the normal build the checks compile to nothing.
#ifdef SQB_BOUNDS_CHECK
#define SQB_IDX(i, n, st) \
  (((unsigned long long)(long long)(i) < (unsigned long long)(n)) ? (i) : (atomicOr((st), ST_BOUNDS), 0))
#else
#define SQB_IDX(i, n, st) (i)
#endif

// Replica atoms and projector tables as the node kernels read them.
struct DevAtoms {
  int n_rep;
  const int *rep_nn;        // [n_rep][4]: nearest node x, y, z (global, reference tie rule), type
  const int *rep_atom;      // [n_rep] global atom index
  const long long *rep_off; // [n_rep] padded table offset (elements)
  const int *typ_nlocc;     // [n_typ]
  const int *typ_nproj;     // [n_typ]
  const double *proj_denom; // [n_typ][MAXPROJ_TYPE]
  const double *tab64;      // projector tables, padded planes, FP64
};

enum NodeMode : int { MODE_SQ = 0, MODE_FORCES = 1, MODE_APPLY = 2, MODE_MOMENTS = 3, MODE_VJP = 4 };
constexpr int VJP_K = 8;  // adjoint: checkpoint every VJP_K recursion vectors

struct NodeArgs {
  int mode;
  int mixed;     // 1: FP32-mixed path (FP32 Lanczos vectors, FP32 force recursion)
  int lq;        // 1: bounds and moments from one Lanczos run at the node (Gauss-quadrature identity)
  int n;         // window edge 2*nloc+1
  int nloc;
  int np[3];
  int pnode_s[3];
  int ex, ey;    // Veff block + halo dims (x, y)
  int npl;
  double h3;     // pow(delta, 3)
  double lanczos_tol;
  double lz_chk;      // checkerboard weight of the Lanczos start vector (0: the reference's ones)
  double coeff_lap[FDN + 1];
  double coeff_grad[FDN + 1];
  const double *veff64;
  DevAtoms at;
  const int *node_list; // nodes to process
  int n_list;
  int *counter;         // work-queue head (zeroed before launch)
  unsigned char *scratch;
  size_t scratch_stride; // bytes per CTA
  size_t stage_bytes;    // bytes of one projector-slice stage in shared memory (set by the launcher)
  int row_layout;        // plane-loop layout of the launch: 0 columns, 1 rows (set by the launcher)
  // MODE_SQ outputs, indexed by node id
  double *chi, *zee, *rho_pj, *lmin, *lmax;
  int *lanczos_iters;
  // MODE_FORCES inputs / outputs
  const double *chi_in, *zee_in, *ci;
  double *fslots; // [n_list][FSLOTS][4]: atom, fx, fy, fz
  // MODE_APPLY
  const double *apply_in;
  double *apply_out;
  // MODE_VJP: dL/dmu per node [nnode][npl+1], per-CTA scratch, dL/dVeff on the
  // Veff block with halo (accumulated with atomics)
  const double *gmu;
  double *vjp;
  size_t vjp_stride;  // doubles per CTA
  double *g_veff;
  // MODE_VJP with atom gradients: derivative tables dchi/dR_alpha (3 x the
  // padded tables, stride dtab_stride values), dL/dR per atom [n_atm][3]
  // (type-major, the layout of the forces), per-CTA scratch vjp_at
  const double *dtab;
  long long dtab_stride;
  double *g_atoms;
  double *vjp_at;
  size_t vjp_at_stride;  // doubles per CTA
  int *status;
  unsigned long long *proj_points; // algorithmic projector-ball points touched
  // test hook of the bounded stage waits (sqb_test_stage_wait): bytes added to
  // every stage's expected transaction count (which then never completes) and
  // the wait limit in ns (0: the default)
  unsigned test_extra_tx;
  unsigned long long wait_ns;
};

// Layered projector fields of the sweep kernel (sqb_sweep.cuh).  The replica
// balls are split into LAYERS layers in which no two balls overlap (in the
// periodic FCC systems the four simple-cubic sublattices), so every point of
// the extended grid (the block with its nloc halo, the domain of every node
// window) lies in at most one ball per layer.  Per point and layer the field
// holds the global index of that ball's first projector (16 bits, four layers
// in one 64-bit word; n_gproj where no ball covers the point) and the values
// of its projectors there (zero elsewhere).
constexpr int LAYERS = 4;
constexpr int LAY_PMAX = 3;  // projectors per replica the fields carry (l <= 1)

struct SweepArgs {
  int form;  // 0: FP64 (the reference's Lanczos + Chebyshev moments); 1: FP32-mixed
             // (FP32 Lanczos vectors, FP64 moments); 2: Lanczos quadrature
  int n, nloc, npl;
  int np[3];
  int ex, ey;
  long long evol;  // ex * ey * ez
  double h3, lanczos_tol, lz_chk;
  double coeff_lap[FDN + 1];
  const double *veff64;
  // layered projector fields
  int n_gproj;                       // projector instances of all replicas; the empty id
  int pmax;                          // projectors per layer slot (1 or 3)
  const unsigned long long *lay_id;  // [evol]: four 16-bit projector bases
  const double *lay_chi;             // [LAYERS][pmax][evol]
  // replicas with projectors, for each node's box list
  int n_rep;
  const int4 *rep_box;  // [n_rep] {x0 | x1 << 16, y0 | y1 << 16, z0 | z1 << 16, layer | nproj << 8 | type << 16},
                        // ball corners on the extended grid
  const int *rep_gpb;   // [n_rep] global index of the replica's first projector
  const int *typ_nlocc;
  const double *proj_denom;  // [n_typ][MAXPROJ_TYPE]
  // work queue and outputs (indexed by node id)
  const int *node_list;
  int n_list;
  int *counter;
  int *status;
  unsigned char *scratch;
  size_t scratch_stride;  // bytes per CTA: three window vectors (FP64), then the flush buffer
  int nsweep;             // threads of the block (a multiple of 32)
  int ry;                 // window rows per thread (2, or 3 up to 33-wide windows)
  double *chi, *zee, *rho_pj, *lmin, *lmax;
  int *lanczos_iters;
  // ForcesNonLocal (sweep_force_kernel): bounds in chi, zee (inputs), the
  // Chebyshev coefficients Ci [node][npl+1], the FD gradient coefficients,
  // the global atom of each replica of rep_box, force slots per listed node
  // [n_list][FSLOTS][4] (atom, fx, fy, fz; atom -1 unused)
  const double *ci;
  double coeff_grad[FDN + 1];
  const int *rep_atom;
  double *fslots;
  unsigned long long *proj_points;  // [3]: ball points x steps (all, Chebyshev only), ball-in-window points x steps
};

// Sweep kernel launchers (sqb_sweep.cu); ry: window rows per thread.
int sweep_threads(int n, int ry);
size_t sweep_smem(int n, int pmax, int n_gproj, int ry);
bool sweep_rows_supported(int n, int ry);
size_t sweep_scratch_bytes(int n, int pmax);  // scratch per CTA
cudaError_t sweep_setup(int n);
cudaError_t launch_sweep(const SweepArgs &a, int grid, cudaStream_t s);
// ForcesNonLocal on the sweep kernel (sqb_sweep_forces.cu); single: FP32
// storage of the Chebyshev vectors (the FP32-mixed form), else FP64.
cudaError_t sweep_forces_setup(int n);
cudaError_t launch_sweep_forces(const SweepArgs &a, int single, int grid, cudaStream_t s);
// Layered fields from the padded projector tables: ids and values of every
// replica's ball on the extended grid (fields zeroed / set empty first).
cudaError_t launch_fill_layers(int n_rep, const int4 *rep_box, const int *rep_gpb, const int *typ_nlocc,
                               const long long *rep_off, const double *tab64, int ex, int ey, int ez, int pmax,
                               int n_gproj, unsigned long long *lay_id, double *lay_chi, cudaStream_t s);

// Host-side launchers (sqb_node.cu).
int node_kernel_threads(int n, int cols);
cudaError_t launch_node_kernel(const NodeArgs &a, int grid, int cols, cudaStream_t s);
// Kernel groups compiled in their own translation units (sqb_node_forces.cu, sqb_node_vjp.cu).
cudaError_t setup_node_forces(int n);
cudaError_t launch_node_forces(const NodeArgs &a, int grid, int cols, cudaStream_t s);
cudaError_t setup_node_vjp(int n);
cudaError_t setup_node_sq32(int n);
cudaError_t setup_node_lq(int n);
cudaError_t launch_node_vjp(const NodeArgs &a, int grid, int cols, cudaStream_t s);
cudaError_t launch_node_sq32(const NodeArgs &a, int grid, int cols, cudaStream_t s);
cudaError_t launch_node_lq(const NodeArgs &a, int grid, int cols, cudaStream_t s);
cudaError_t node_kernel_setup(int n);
// Stage size wanted for a per-plane footprint of `elems` values (the launcher
// clamps it to what the launch's shared memory leaves).
size_t node_kernel_stage_bytes(int n, long long elems);
// Largest per-plane projector-slice footprint over the block's windows -> *d_out.
cudaError_t launch_plane_footprint(int n, int nloc, const int *np, const int *pnode_s, int n_rep, const int *rep_nn,
                                   const int *typ_nlocc, const int *typ_nproj, unsigned *d_out, cudaStream_t s);

// Fermi-level and assembly kernels (sqb_fermi.cu).
struct FermiArgs {
  int n_nodes, npl;
  double bet0, h3;
  const double *chi, *zee, *rho_pj;
  const double *xk;   // [npl+1] Chebyshev-Gauss nodes (sq.cpp:1241)
  const double *ctab; // [npl+1][npl+1] cos(pi j (k+1/2)/(npl+1)) (sq.cpp:1250)
  double *partial;    // per-block partial sums
  double *result;     // final sums
  double *rho, *ci;   // assembly outputs
  int *status;
  const double *lam_dev;  // when set, the kernels read the Fermi level here (graph replay)
};
cudaError_t launch_ne_constraint(const FermiArgs &a, double lambda, int with_derivative, cudaStream_t s);

// Fermi-level solve on the device (BrentsAlgorithm sq.cpp:1289-1404 or
// NewtonRaphson sq.cpp:1459-1490, the host solvers' control flow and
// arithmetic), one NeConstraint evaluation per step, for the whole SQ step
// replayed as one CUDA graph with a conditional while node: fermi_init sets
// the first trial level, each loop body runs NeConstraint at st->x and
// fermi_step, which takes the sums, advances the solver and sets the loop
// condition (0 once converged or failed).
struct FermiDev {
  int alg, scf_iter;          // 1 Brent, 2 Newton
  double lambda_warm, tol, h3, ncharge, bet;
  double a, b, cc, d, e, fa, fb, fc;  // Brent
  int phase, iter;
  double lold, lnew, err;     // Newton
  int count;
  double x;                   // the level the next NeConstraint evaluates
  int steps;                  // evaluations so far (bounded)
  int status;                 // 0 running, 1 converged, -1 not bracketed, -2 iteration limit, -3 non-finite
  double root;
  int iters;
  int dstat;                  // the density assembly's status bits (1 negative rho, 2 non-finite)
  double lmin_all, lmax_all;  // the spectral bracket of the step (min lmin, max lmax over nodes)
};
cudaError_t launch_fermi_init(FermiDev *st, const double *minmax, cudaStream_t s);
cudaError_t launch_fermi_step(FermiDev *st, const double *sums, cudaGraphConditionalHandle h, cudaStream_t s);
cudaError_t launch_density_energy(const FermiArgs &a, double lambda, cudaStream_t s);
int fermi_blocks(int n_nodes);
// Density-loss adjoint (sqb_density_loss_vjp): signs of the nodes' densities
// and the Fermi-level response sums into result[0..1]; then the moment weights.
cudaError_t launch_loss_lambda(const FermiArgs &a, double lambda, const double *w, int fixed, double *sgn,
                               cudaStream_t s);
cudaError_t launch_loss_gmu(int n, int K, const double *ci, const double *w, const double *sgn, double scale,
                            double off, double *g, cudaStream_t s);
cudaError_t launch_bound_sens(const FermiArgs &a, double lambda, double delta, double *sens, double *rho0,
                              cudaStream_t s);

// Force reduction and projector kernels.
cudaError_t launch_force_reduce(const double *fslots, int n_list, int n_atm, double *f, cudaStream_t s);
struct ProjArgs {
  int n_rep;
  double delta;
  const int *rep_nn;
  const double *rep_xyz;
  const long long *rep_off;
  const int *typ_nlocc, *typ_lmax, *typ_lloc, *typ_size;
  const long long *typ_tab; // offset of each type's 19 x size tables
  const double *tables;
  double *out64;
  long long total;
  int *status;
};
cudaError_t launch_projectors(const ProjArgs &a, cudaStream_t s);
// out = (plus - minus) * scale, element-wise.
cudaError_t launch_fd_combine(const double *plus, const double *minus, double *out, long long n, double scale,
                              cudaStream_t s);
// Copy tables between the reference's UdVtm layout and the padded device layout.
cudaError_t launch_repack(int n_rep, const int *rep_nn, const int *typ_nlocc, const int *typ_nproj,
                          const long long *off_ref, const long long *off_pad, const double *in, double *out,
                          int to_pad, cudaStream_t s);
cudaError_t launch_minmax(const double *lmin, const double *lmax, int n, double *out, cudaStream_t s);

// Pseudocharge density and local forces (sqb_local.cu): ChargeDensity
// (initialize.cpp:470-784) and ForcesLocal (forces.cpp:20-315) on the block.
struct LocalArgs {
  int np[3], pnode_s[3];
  double delta, h3;  // h3 = pow(delta, 3) formed on the host
  double coeff_lap[FDN + 1], coeff_grad[FDN + 1];
  int n_rep;
  const int *rep_type, *rep_atom;
  const double *rep_xyz;  // [n_rep][3]
  const int *rep_box;     // [n_rep][6]: xstart, xend, ystart, yend, zstart, zend (global nodes)
  const double *tab;      // per type [5][size]: grid, rVloc, DVloc, uu, Duu
  const long long *typ_off;
  const int *typ_size;
  const double *Z;
  double rc_tilda;
  int *status;
  // ChargeDensity: block fields (raw: b_tilda unscaled, Vc unshifted) and
  // per-CTA sums [5][n_cta] of Eself, Ncharge, the rho_at integral,
  // Ncharge_tilda, Eself_tilda
  double *b, *b_tilda, *vc, *rho_at, *partial;
  // ForcesLocal: the fields it reads (phi with its FDN halo), the per-replica
  // scratch boxes (VlocJ, VlocJ_tilda, bJ, bJ_tilda, each box + 2 FDN wide)
  // at scr + scr_off[r], and per-(replica, CTA) force sums [6]
  const double *phi, *vcf, *bf, *btf;
  double *scr;
  const long long *scr_off;
  double *fpart;
};
// Tile edge of the charge-density kernel and its CTA count for the block.
constexpr int LOC_TILE = 8;
int charge_density_ctas(const int np[3]);
cudaError_t launch_charge_density(const LocalArgs &a, cudaStream_t s);
// b_tilda *= scale, Vc += shift, and per-CTA sums of 0.5 (b_tilda + b) Vc h^3
// into partial[0..n_cta) (the Ecorr loop of initialize.cpp:759-768).
cudaError_t launch_charge_finish(const LocalArgs &a, double scale, double shift, cudaStream_t s);
constexpr int LOC_FORCE_CTAS = 64;  // CTAs per replica of the force contraction
// ForcesLocal for replicas [r0, r1): scratch boxes, then per-(replica, CTA)
// force sums into fpart[((r - r0) * LOC_FORCE_CTAS + cta) * 6].
cudaError_t launch_forces_local(const LocalArgs &a, int r0, int r1, cudaStream_t s);

}  // namespace sqb
