// C-ABI of sqdft_b200 (include/sqdft_b200.h): context management, uploads and
// the host-side control flow of the SQ step.
//
// The device does the per-node work (node kernel), the per-node Chebyshev
// coefficients and their reductions; the host keeps the reference's scalar
// control flow -- Brent / Newton for the Fermi level and the order of the
// phases of ClenshawCurtisSpectralQuadrature (sq.cpp:377-834) -- so the
// sequence of trial Fermi levels is the reference's.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sqdft_b200.h"
#include "sqb_internal.cuh"

using namespace sqb;

struct sqb_ctx {
  sqb_grid g{};
  int device = 0, sms = 148;
  cudaStream_t stream = nullptr;
  int precision = SQB_FP64;
  double mixed_lanczos_tol = 0.0;  // Ha: the mixed path's Lanczos stop and margin (0: the grid's)
  double defect_budget = 0.0;      // relative density budget of the fast forms' defect check (0: off)
  double mixed_lanczos_chk = 0.5;  // checkerboard weight of the mixed path's Lanczos start vector
  int cols = 0, ctas_per_sm = 1;
  int use_graph = 0;                       // replay the node-kernel sequence from a CUDA graph
  cudaGraphExec_t sq_graph = nullptr;      // captured Lanczos+moments sequence (node kernel, min/max)
  cudaGraphExec_t step_graph = nullptr;    // the whole SQ step (sqb_set_graph(ctx, 2))
  FermiDev *d_fermi = nullptr;             // its device-side Fermi solver state
  int sq_graph_warm = 0;                   // a plain run has allocated what the sequence uses
  int n = 0, nnode = 0, ex = 0, ey = 0, ez = 0;
  double h3 = 0.0;
  sqb_allreduce_fn allreduce = nullptr;
  void *allreduce_user = nullptr;

  double *d_veff64 = nullptr;
  bool have_veff = false;

  int n_typ = 0, n_rep = 0, n_atm = 0;
  std::vector<int> typ_nproj, typ_nlocc;
  int *d_rep_nn = nullptr, *d_rep_atom = nullptr;
  long long *d_rep_off = nullptr, *d_typ_tab = nullptr;
  int *d_typ_nlocc = nullptr, *d_typ_nproj = nullptr, *d_typ_lmax = nullptr, *d_typ_lloc = nullptr;
  int *d_typ_size = nullptr;
  double *d_proj_denom = nullptr, *d_tables = nullptr, *d_rep_xyz = nullptr;
  bool have_tables = false;
  double *d_tab64 = nullptr;
  long long tab_total = 0;      // values of the reference's UdVtm
  long long tab_pad_total = 0;  // values of the padded device tables
  long long *d_rep_off_ref = nullptr;
  double *d_vjp = nullptr;  // adjoint: per-CTA scratch, dL/dmu, dL/dVeff
  size_t vjp_bytes = 0;
  double *d_vjp_at = nullptr;  // adjoint with atom gradients: per-CTA scratch, dL/dR
  size_t vjp_at_bytes = 0;
  double *d_dtab = nullptr;    // dchi/dR_alpha tables, 3 x tab_pad_total
  bool have_dtab = false;
  std::vector<double> h_rep_xyz;  // replica positions (for the derivative tables)
  long long stage_elems = 0;  // largest per-plane projector-slice footprint (values)
  std::vector<int> h_rep_nn;  // [n_rep][4] nearest nodes and types (host copy)
  // Sweep kernel (sqb_sweep.cuh) and its layered projector fields, built on
  // first use after the projector tables are set.
  int node_kernel = SQB_KERNEL_AUTO;
  int sweep_ry = 0;  // window rows per sweep-kernel thread (0: automatic)
  int lay_state = 0;  // 0 not built, 1 built and usable, -1 the sweep kernel does not cover this context
  int n_gproj = 0, lay_pmax = 1, n_lrep = 0;
  unsigned long long *d_lay_id = nullptr;
  double *d_lay_chi = nullptr;
  int4 *d_rep_box = nullptr;
  int *d_rep_gpb = nullptr;
  int *d_rep_atom_l = nullptr;  // global atom of each replica of d_rep_box
  bool have_atoms = false, have_proj = false;

  unsigned char *d_scratch = nullptr;
  size_t scratch_stride = 0, scratch_bytes = 0;
  int *d_counter = nullptr, *d_nodes = nullptr, *d_status = nullptr, *d_iters = nullptr;
  unsigned long long *d_proj_points = nullptr;
  double *d_chi = nullptr, *d_zee = nullptr, *d_rho_pj = nullptr, *d_lmin = nullptr, *d_lmax = nullptr;
  bool have_moments = false;
  double lmin_all = 0.0, lmax_all = 0.0;

  double *d_xk = nullptr, *d_ctab = nullptr, *d_partial = nullptr, *d_result = nullptr;
  double *d_rho = nullptr, *d_ci = nullptr;
  double *d_sens = nullptr;  // per-node density sensitivity of the defect check
  double *d_loss = nullptr;  // density-loss adjoint: weights and signs [2][N]
  int loss_n = 0;
  double lambda_last = 0.0;  // Fermi level of the last sqb_density_energy
  bool have_ci = false;
  double *d_fslots = nullptr, *d_f = nullptr;
  double *d_tmp = nullptr;
  size_t tmp_bytes = 0;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_order = nullptr;  // orders the no-alloc call after the caller's queued work
  sqb_stats stats{};
  std::string metrics_path;  // SQDFT_B200_METRICS at creation: one JSON line per SQ step / force pass
  unsigned test_extra_tx = 0;           // sqb_test_stage_wait
  unsigned long long test_wait_ns = 0;

  // pseudocharge replicas (sqb_set_local_atoms) and the block fields of
  // sqb_charge_density / sqb_forces_local
  int loc_nrep = 0, loc_natm = 0;
  double loc_rc_tilda = 0.0;
  bool have_local = false;
  std::vector<int> h_loc_atom, h_loc_box;
  int *d_loc_type = nullptr, *d_loc_atom = nullptr, *d_loc_box = nullptr, *d_loc_size = nullptr;
  long long *d_loc_off = nullptr, *d_loc_scr_off = nullptr;
  double *d_loc_xyz = nullptr, *d_loc_tab = nullptr, *d_loc_Z = nullptr;
  double *d_loc_fields = nullptr;  // b, b_tilda, Vc, rho_at, phi (+halo), partial sums
  size_t loc_fields_bytes = 0;
  double *d_loc_scr = nullptr;     // ForcesLocal scratch boxes and per-CTA force sums
  size_t loc_scr_bytes = 0;
};

namespace {

#define CK(x)                                    \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) {                     \
      std::fprintf(stderr, "sqdft_b200: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
      return SQB_ERR_CUDA;                       \
    }                                            \
  } while (0)

// NVTX range over an entry point (visible in Nsight Systems / Compute; a
// no-op without a tool attached).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

// One JSON line per SQ step or force pass into the file named by
// SQDFT_B200_METRICS (read when the context is created): the phase times,
// iteration counts and status of the call.
void write_metrics(const sqb_ctx *c, const char *call, int rc, double lambda_f) {
  if (c->metrics_path.empty()) return;
  FILE *f = std::fopen(c->metrics_path.c_str(), "a");
  if (!f) return;
  const sqb_stats &s = c->stats;
  std::fprintf(f,
               "{\"call\": \"%s\", \"status\": %d, \"precision\": %d, \"node_kernel\": %d, \"nodes\": %d, "
               "\"window\": %d, \"npl\": %d, \"ms_lanczos_moments\": %.6f, \"ms_fermi\": %.6f, "
               "\"ms_density\": %.6f, \"ms_defect\": %.6f, \"ms_forces\": %.6f, \"lanczos_iters\": %lld, "
               "\"max_lanczos_iters\": %d, \"lanczos_maxiter_nodes\": %lld, \"fermi_iters\": %d, "
               "\"defect_nodes\": %lld, \"matvecs\": %lld, \"kernel_launches\": %d, \"lambda_f\": %.17g}\n",
               call, rc, c->precision, s.node_kernel, c->nnode, c->n, c->g.npl, s.ms_lanczos_moments, s.ms_fermi,
               s.ms_density, s.ms_defect, s.ms_forces, s.lanczos_iters, s.max_lanczos_iters, s.lanczos_maxiter_nodes,
               s.fermi_iters, s.defect_nodes, s.matvecs, s.kernel_launches, lambda_f);
  std::fclose(f);
}

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  return cudaMalloc((void **)p, count * sizeof(T) + 16);
}

// Nearest grid node of an atom coordinate with the midpoint rule of
// nonlocal.cpp:49-64 (Replica_atoms_Rcut uses the same rule).
int nearest_node(double c, double h) {
  int n = (int)round(c / h);
  if (fabs(fabs(n * h - c) - h * 0.5) < 1e-12) n = (int)floor((c / h) - 10 * 1e-12);
  return n;
}

int reduce(sqb_ctx *c, double *v, int count, int op) {
  if (!c->allreduce) return SQB_OK;
  return c->allreduce(v, count, op, c->allreduce_user) == 0 ? SQB_OK : SQB_ERR_ARG;
}

int status_to_err(int st) {
  if (st & ST_CAPACITY) return SQB_ERR_CAPACITY;
  if (st & ST_FSLOTS) return SQB_ERR_CAPACITY;
  if (st & ST_SPLINE_RANGE) return SQB_ERR_SPLINE_RANGE;
  if (st & ST_NONFINITE) return SQB_ERR_NONFINITE;
  // ST_LANCZOS_MAXITER is a warning: the reference prints and carries on with
  // the last Ritz values (sq.cpp:1073-1074); the nodes are counted in the stats.
  if (st & ST_WAIT_LIMIT) return SQB_ERR_CUDA;
  if (st & ST_BOUNDS) return SQB_ERR_BOUNDS;
  return SQB_OK;
}

int ensure_tmp(sqb_ctx *c, size_t bytes) {
  if (c->tmp_bytes >= bytes) return SQB_OK;
  if (c->d_tmp) cudaFree(c->d_tmp);
  c->d_tmp = nullptr;
  CK(cudaMalloc((void **)&c->d_tmp, bytes));
  c->tmp_bytes = bytes;
  return SQB_OK;
}

// Columns per thread of the node kernel: 0 lets the launcher pick its layout.
int choose_cols(const sqb_ctx *c) { return c->cols; }

void drop_graph(sqb_ctx *c);

int ensure_scratch(sqb_ctx *c, int grid) {
  const size_t nw = (size_t)c->n * c->n * c->n;
  c->scratch_stride = ((4 * nw * sizeof(double)) + 255) & ~size_t(255);
  const size_t need = c->scratch_stride * (size_t)grid;
  if (c->scratch_bytes < need) {
    drop_graph(c);  // captured launches hold the old buffer's address
    if (c->d_scratch) cudaFree(c->d_scratch);
    c->d_scratch = nullptr;
    CK(cudaMalloc((void **)&c->d_scratch, need));
    c->scratch_bytes = need;
  }
  return SQB_OK;
}

void fill_node_args(sqb_ctx *c, NodeArgs &a) {
  std::memset(&a, 0, sizeof(a));
  a.n = c->n;
  a.nloc = c->g.nloc;
  for (int d = 0; d < 3; d++) {
    a.np[d] = c->g.np[d];
    a.pnode_s[d] = c->g.pnode_s[d];
  }
  a.ex = c->ex;
  a.ey = c->ey;
  a.npl = c->g.npl;
  a.h3 = c->h3;
  a.mixed = c->precision == SQB_FP32_MIXED;
  a.lq = c->precision == SQB_FP64_LANCZOS_QUAD;
  a.lanczos_tol = (a.mixed || a.lq) ? std::max(c->g.lanczos_tol, c->mixed_lanczos_tol) : c->g.lanczos_tol;
  a.lz_chk = a.mixed ? c->mixed_lanczos_chk : 0.0;
  a.test_extra_tx = c->test_extra_tx;
  a.wait_ns = c->test_wait_ns;
  for (int k = 0; k <= FDN; k++) {
    a.coeff_lap[k] = c->g.coeff_lap[k];
    a.coeff_grad[k] = c->g.coeff_grad[k];
  }
  a.veff64 = c->d_veff64;
  a.at.n_rep = c->n_rep;
  a.at.rep_nn = c->d_rep_nn;
  a.at.rep_atom = c->d_rep_atom;
  a.at.rep_off = c->d_rep_off;
  a.at.typ_nlocc = c->d_typ_nlocc;
  a.at.typ_nproj = c->d_typ_nproj;
  a.at.proj_denom = c->d_proj_denom;
  a.at.tab64 = c->d_tab64;
  a.counter = c->d_counter;
  a.status = c->d_status;
  a.proj_points = c->d_proj_points;
  a.stage_bytes = node_kernel_stage_bytes(c->n, c->stage_elems);
}

// Launch the node kernel over `count` nodes of d_list; returns SQB status.
int run_nodes(sqb_ctx *c, NodeArgs &a, const int *d_list, int count) {
  const int cols = choose_cols(c);
  const int threads = node_kernel_threads(c->n, cols);
  if (threads > 1024) return SQB_ERR_UNSUPPORTED;
  int grid = c->sms * (c->ctas_per_sm > 0 ? c->ctas_per_sm : 1);
  if (grid > count) grid = count;
  if (grid < 1) grid = 1;
  int rc = ensure_scratch(c, grid);
  if (rc) return rc;
  a.scratch = c->d_scratch;
  a.scratch_stride = c->scratch_stride;
  a.node_list = d_list;
  a.n_list = count;
  CK(cudaMemsetAsync(c->d_counter, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->d_proj_points, 0, 3 * sizeof(unsigned long long), c->stream));
  CK(launch_node_kernel(a, grid, cols, c->stream));
  return SQB_OK;
}

// Layered projector fields of the sweep kernel: the replica balls with
// projectors, as boxes on the extended grid (the block with its nloc halo),
// split greedily in replica order into layers whose balls neither overlap nor
// touch along z (a gap of at least one plane where their x-y footprints
// overlap).  The sweep kernel covers the context when four layers suffice,
// every type has at most three projectors, the ids fit 16 bits and the
// block's shared memory holds the kernel's working set; otherwise the
// plane-streaming kernel runs.
int ensure_layers(sqb_ctx *c) {
  if (c->lay_state != 0) return SQB_OK;
  c->lay_state = -1;
  const int nl = c->g.nloc, E[3] = {c->ex, c->ey, c->ez};
  struct Box {
    int lo[3], hi[3], r, np, t;
  };
  std::vector<Box> boxes;
  int pmax = 0, ngp = 0;
  for (int r = 0; r < c->n_rep; r++) {
    const int t = c->h_rep_nn[4 * r + 3], np = c->typ_nproj[t], nlc = c->typ_nlocc[t];
    if (np == 0) continue;
    Box b{};
    bool in = true;
    for (int d = 0; d < 3; d++) {
      b.lo[d] = c->h_rep_nn[4 * r + d] - nlc - (c->g.pnode_s[d] - nl);
      b.hi[d] = b.lo[d] + 2 * nlc;
      in = in && b.hi[d] >= 0 && b.lo[d] < E[d];
    }
    if (!in) continue;
    b.r = r;
    b.np = np;
    b.t = t;
    boxes.push_back(b);
    pmax = std::max(pmax, np);
  }
  std::vector<std::vector<int>> layers;
  std::vector<int> layer_of(boxes.size());
  for (size_t i = 0; i < boxes.size(); i++) {
    const Box &b = boxes[i];
    int k = 0;
    for (; k < (int)layers.size(); k++) {
      bool clash = false;
      for (int j : layers[k]) {
        const Box &o = boxes[j];
        if (b.lo[0] <= o.hi[0] && o.lo[0] <= b.hi[0] && b.lo[1] <= o.hi[1] && o.lo[1] <= b.hi[1] &&
            b.lo[2] <= o.hi[2] + 1 && o.lo[2] <= b.hi[2] + 1) {
          clash = true;
          break;
        }
      }
      if (!clash) break;
    }
    if (k == (int)layers.size()) layers.emplace_back();
    layers[k].push_back((int)i);
    layer_of[i] = k;
  }
  std::vector<int4> box4(std::max<size_t>(boxes.size(), 1));
  std::vector<int> gpb(std::max<size_t>(boxes.size(), 1));
  for (size_t i = 0; i < boxes.size(); i++) {
    const Box &b = boxes[i];
    box4[i] = make_int4((b.lo[0] & 0xffff) | (b.hi[0] << 16), (b.lo[1] & 0xffff) | (b.hi[1] << 16),
                        (b.lo[2] & 0xffff) | (b.hi[2] << 16), layer_of[i] | (b.np << 8) | (b.t << 16));
    gpb[i] = ngp;
    ngp += b.np;
  }
  const int pm = pmax <= 1 ? 1 : 3;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  const long long evol_all = (long long)c->ex * c->ey * c->ez;
  const bool usable = (int)layers.size() <= LAYERS && pmax <= LAY_PMAX && ngp + pm < 65535 &&
                      evol_all * LAYERS * LAY_PMAX < (1LL << 31) &&
                      sweep_rows_supported(c->n, 2) && sweep_smem(c->n, pm, ngp, 2) <= (size_t)optin &&
                      c->n_typ < 256;
  if (!usable) return SQB_OK;
  const long long evol = (long long)c->ex * c->ey * c->ez;
  c->n_gproj = ngp;
  c->lay_pmax = pm;
  c->n_lrep = (int)boxes.size();
  CK(dalloc(&c->d_lay_id, (size_t)evol));
  CK(dalloc(&c->d_lay_chi, (size_t)LAYERS * pm * evol));
  CK(dalloc(&c->d_rep_box, box4.size()));
  CK(dalloc(&c->d_rep_gpb, gpb.size()));
  CK(cudaMemcpy(c->d_rep_box, box4.data(), box4.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_rep_gpb, gpb.data(), gpb.size() * sizeof(int), cudaMemcpyHostToDevice));
  {
    std::vector<int> atom_all(std::max(c->n_rep, 1)), atom_l(std::max<size_t>(boxes.size(), 1));
    CK(cudaMemcpy(atom_all.data(), c->d_rep_atom, atom_all.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < boxes.size(); i++) atom_l[i] = atom_all[boxes[i].r];
    CK(dalloc(&c->d_rep_atom_l, atom_l.size()));
    CK(cudaMemcpy(c->d_rep_atom_l, atom_l.data(), atom_l.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  // the fill kernel indexes the padded tables by box: the offsets of the boxes' replicas
  std::vector<long long> off_all(std::max(c->n_rep, 1));
  CK(cudaMemcpy(off_all.data(), c->d_rep_off, off_all.size() * sizeof(long long), cudaMemcpyDeviceToHost));
  std::vector<long long> off(std::max<size_t>(boxes.size(), 1));
  for (size_t i = 0; i < boxes.size(); i++) off[i] = off_all[boxes[i].r];
  long long *d_off = nullptr;
  CK(cudaMalloc((void **)&d_off, off.size() * sizeof(long long)));
  CK(cudaMemcpy(d_off, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice));
  const cudaError_t e = launch_fill_layers((int)boxes.size(), c->d_rep_box, c->d_rep_gpb, c->d_typ_nlocc, d_off,
                                           c->d_tab64, c->ex, c->ey, c->ez, pm, ngp, c->d_lay_id, c->d_lay_chi,
                                           c->stream);
  const cudaError_t e2 = cudaStreamSynchronize(c->stream);
  cudaFree(d_off);
  CK(e);
  CK(e2);
  c->lay_state = 1;
  return SQB_OK;
}

// Whether the SQ node work of this context runs on the sweep kernel.
int use_sweep(sqb_ctx *c, bool *yes) {
  *yes = false;
  if (c->node_kernel == SQB_KERNEL_PLANE) return SQB_OK;
  int rc = ensure_layers(c);
  if (rc) return rc;
  if (c->lay_state != 1) return c->node_kernel == SQB_KERNEL_SWEEP ? SQB_ERR_UNSUPPORTED : SQB_OK;
  *yes = true;
  return SQB_OK;
}

// Sweep-kernel scratch for `grid` CTAs (grown on demand).
int ensure_sweep_scratch(sqb_ctx *c, int grid, size_t *stride) {
  *stride = sweep_scratch_bytes(c->n, c->lay_pmax);
  if (c->scratch_bytes < *stride * (size_t)grid) {
    drop_graph(c);  // captured launches hold the old buffer's address
    if (c->d_scratch) cudaFree(c->d_scratch);
    c->d_scratch = nullptr;
    c->scratch_bytes = 0;
    CK(cudaMalloc((void **)&c->d_scratch, *stride * (size_t)grid));
    c->scratch_bytes = *stride * (size_t)grid;
  }
  return SQB_OK;
}

// Window rows per sweep-kernel thread: the requested count where the kernel
// covers it (sqb_set_sweep_rows, sqb_autotune_sweep), else 2.  (Three rows
// give fewer threads more registers; measured on the B200 they were slower
// also where the fields carry three projectors per slot: c3 FP64 199 against
// 167 ms on a 296-node sample, forces 34.8 against 27.9 s.)
int sweep_rows(const sqb_ctx *c) {
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  auto fits = [&](int ry) {
    return sweep_rows_supported(c->n, ry) && sweep_smem(c->n, c->lay_pmax, c->n_gproj, ry) <= (size_t)optin;
  };
  if (c->sweep_ry && fits(c->sweep_ry)) return c->sweep_ry;
  return 2;
}

// The context's part of a sweep-kernel launch (grid, fields, replicas, queue).
void fill_sweep_args(sqb_ctx *c, const int *d_list, int count, size_t stride, SweepArgs &s) {
  std::memset(&s, 0, sizeof(s));
  s.n = c->n;
  s.nloc = c->g.nloc;
  s.npl = c->g.npl;
  for (int d = 0; d < 3; d++) s.np[d] = c->g.np[d];
  s.ex = c->ex;
  s.ey = c->ey;
  s.evol = (long long)c->ex * c->ey * c->ez;
  s.h3 = c->h3;
  s.lanczos_tol = c->g.lanczos_tol;
  for (int k = 0; k <= FDN; k++) s.coeff_lap[k] = c->g.coeff_lap[k];
  for (int k = 0; k <= FDN; k++) s.coeff_grad[k] = c->g.coeff_grad[k];
  s.veff64 = c->d_veff64;
  s.n_gproj = c->n_gproj;
  s.pmax = c->lay_pmax;
  s.lay_id = c->d_lay_id;
  s.lay_chi = c->d_lay_chi;
  s.n_rep = c->n_lrep;
  s.rep_box = c->d_rep_box;
  s.rep_gpb = c->d_rep_gpb;
  s.rep_atom = c->d_rep_atom_l;
  s.typ_nlocc = c->d_typ_nlocc;
  s.proj_denom = c->d_proj_denom;
  s.node_list = d_list;
  s.n_list = count;
  s.counter = c->d_counter;
  s.status = c->d_status;
  s.scratch = c->d_scratch;
  s.scratch_stride = stride;
  s.ry = sweep_rows(c);
  s.nsweep = sweep_threads(c->n, s.ry);
  s.proj_points = c->d_proj_points;
}

// Lanczos bounds and Chebyshev moments (MODE_SQ) of `count` nodes of d_list
// with the outputs of `a`, on the sweep kernel where it covers the context,
// else on the plane-streaming node kernel.
int run_sq_nodes(sqb_ctx *c, NodeArgs &a, const int *d_list, int count) {
  bool sw = false;
  int rc = use_sweep(c, &sw);
  if (rc) return rc;
  c->stats.node_kernel = sw ? SQB_KERNEL_SWEEP : SQB_KERNEL_PLANE;
  if (!sw) return run_nodes(c, a, d_list, count);
  int grid = c->sms;
  if (grid > count) grid = count;
  if (grid < 1) grid = 1;
  size_t stride = 0;
  rc = ensure_sweep_scratch(c, grid, &stride);
  if (rc) return rc;
  SweepArgs s;
  fill_sweep_args(c, d_list, count, stride, s);
  s.form = a.lq ? 2 : (a.mixed ? 1 : 0);
  s.lanczos_tol = a.lanczos_tol;
  s.lz_chk = a.lz_chk;
  s.chi = a.chi;
  s.zee = a.zee;
  s.rho_pj = a.rho_pj;
  s.lmin = a.lmin;
  s.lmax = a.lmax;
  s.lanczos_iters = a.lanczos_iters;
  CK(cudaMemsetAsync(c->d_counter, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->d_proj_points, 0, 3 * sizeof(unsigned long long), c->stream));
  CK(launch_sweep(s, grid, c->stream));
  return SQB_OK;
}

int read_status(sqb_ctx *c) {
  int st = 0;
  CK(cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return status_to_err(st);
}

FermiArgs fermi_args(sqb_ctx *c) {
  FermiArgs f{};
  f.n_nodes = c->nnode;
  f.npl = c->g.npl;
  f.bet0 = c->g.bet;
  f.h3 = c->h3;
  f.chi = c->d_chi;
  f.zee = c->d_zee;
  f.rho_pj = c->d_rho_pj;
  f.xk = c->d_xk;
  f.ctab = c->d_ctab;
  f.partial = c->d_partial;
  f.result = c->d_result;
  f.rho = c->d_rho;
  f.ci = c->d_ci;
  f.status = c->d_status;
  return f;
}

// NeConstraint / NeConstraint_derv: g (and dg) before the h^3 scaling,
// summed over ranks.
int ne_sums(sqb_ctx *c, double lambda, int deriv, double *g, double *dg) {
  CK(launch_ne_constraint(fermi_args(c), lambda, deriv, c->stream));
  double r[2];
  CK(cudaMemcpyAsync(r, c->d_result, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->stats.kernel_launches += 2;
  *g = r[0];
  *dg = r[1];
  return SQB_OK;
}

int ne_constraint(sqb_ctx *c, double lambda, double *fval) {
  double g, dg;
  int rc = ne_sums(c, lambda, 0, &g, &dg);
  if (rc) return rc;
  g = g * pow(c->g.delta, 3);  // sq.cpp:1214
  rc = reduce(c, &g, 1, SQB_SUM);
  if (rc) return rc;
  *fval = g - (-c->g.ncharge);
  return std::isfinite(*fval) ? SQB_OK : SQB_ERR_NONFINITE;
}

#define SIGN(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))

// BrentsAlgorithm (sq.cpp:1289-1404), same control flow and tolerances.
int brent(sqb_ctx *c, double x1, double x2, int scf_iter, double lambda_warm, double *root, int *iters) {
  const double EPS = 2.5e-16, tol = c->g.fermi_tol;
  double tol1q, eq, a = x1, b = x2, cc = x2, d = 0.0, e = 0.0, min1, min2;
  if (scf_iter > 1) {
    a = lambda_warm - 2;
    b = lambda_warm + 2;
  }
  double fa, fb, fc, p, q, r, s, tol1, xm;
  int rc = ne_constraint(c, a, &fa);
  if (!rc) rc = ne_constraint(c, b, &fb);
  if (rc) return rc;
  if ((fa > 0.0 && fb > 0.0) || (fa < 0.0 && fb < 0)) return SQB_ERR_NOT_BRACKETED;
  fc = fb;
  for (int iter = 1; iter <= 100; iter++) {
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) {
      cc = a;
      fc = fa;
      e = d = b - a;
    }
    if (fabs(fc) < fabs(fb)) {
      a = b;
      b = cc;
      cc = a;
      fa = fb;
      fb = fc;
      fc = fa;
    }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * tol;
    xm = 0.5 * (cc - b);
    if (fabs(xm) <= tol1 || fb == 0.0) {
      *root = b;
      *iters = iter;
      return SQB_OK;
    }
    if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
      s = fb / fa;
      if (a == cc) {
        p = 2.0 * xm * s;
        q = 1.0 - s;
      } else {
        q = fa / fc;
        r = fb / fc;
        p = s * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (p > 0.0) q = -q;
      p = fabs(p);
      tol1q = tol1 * q;
      min1 = 3.0 * xm * q - fabs(tol1q);
      eq = e * q;
      min2 = fabs(eq);
      if (2.0 * p < (min1 < min2 ? min1 : min2)) {
        e = d;
        d = p / q;
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
    rc = ne_constraint(c, b, &fb);
    if (rc) return rc;
  }
  return SQB_ERR_FERMI_MAXITER;
}

// NewtonRaphson (sq.cpp:1459-1490) with NeConstraint_derv (sq.cpp:1407-1449).
int newton(sqb_ctx *c, double lambda0, double *root, int *iters) {
  double lnew = 0.0, lold = lambda0, err = 1.0;
  int count = 0;
  while (err > c->g.fermi_tol && count < 200) {
    double g, dg;
    int rc = ne_sums(c, lold, 1, &g, &dg);
    if (rc) return rc;
    dg = dg * c->g.bet;
    dg = dg * pow(c->g.delta, 3);
    g = g * pow(c->g.delta, 3);
    double t[2] = {g, dg};
    rc = reduce(c, t, 2, SQB_SUM);
    if (rc) return rc;
    const double fa = t[0] - (-c->g.ncharge), dfa = t[1];
    lnew = lold - (fa / dfa);
    err = fabs(lnew - lold);
    lold = lnew;
    count += 1;
  }
  *root = lnew;
  *iters = count;
  return std::isfinite(lnew) ? SQB_OK : SQB_ERR_NONFINITE;
}

// Lanczos counts and projector points of the last full SQ launch into the stats.
int lanczos_stats(sqb_ctx *c, std::vector<int> &its) {
  const size_t N = c->nnode;
  its.resize(N);
  CK(cudaMemcpy(its.data(), c->d_iters, N * sizeof(int), cudaMemcpyDeviceToHost));
  unsigned long long pp[3] = {0, 0, 0};
  CK(cudaMemcpy(pp, c->d_proj_points, sizeof(pp), cudaMemcpyDeviceToHost));
  long long sum = 0;
  int mx = 0;
  for (size_t i = 0; i < N; i++) {
    sum += its[i];
    mx = std::max(mx, its[i]);
  }
  c->stats.lanczos_iters = sum;
  c->stats.max_lanczos_iters = mx;
  long long capped = 0;
  // (the quadrature form reports rows - 1 iterations, so its cap shows as 499)
  const int cap = LANCZOS_MAX_ITER - (c->precision == SQB_FP64_LANCZOS_QUAD ? 1 : 0);
  for (size_t i = 0; i < N; i++) capped += its[i] >= cap;
  c->stats.lanczos_maxiter_nodes = capped;
  // passes: Lanczos 2 per iteration + 2, Chebyshev npl/2 (matvec passes only)
  c->stats.matvecs = sum + (long long)N + (c->precision == SQB_FP64_LANCZOS_QUAD ? 0LL : (long long)N * (c->g.npl / 2));
  c->stats.proj_points = (long long)pp[0];
  c->stats.proj_points_cheb = (long long)pp[1];
  c->stats.proj_points_window = (long long)pp[2];
  return SQB_OK;
}

float elapsed(sqb_ctx *c) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  return ms;
}

// Drop the captured SQ sequence (its kernel arguments may have changed).
void drop_graph(sqb_ctx *c) {
  if (c->sq_graph) cudaGraphExecDestroy(c->sq_graph);
  c->sq_graph = nullptr;
  c->sq_graph_warm = 0;
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  c->step_graph = nullptr;
}

}  // namespace

extern "C" {

const char *sqb_version(void) { return "sqdft_b200 0.1 (sm_100a)"; }

const char *sqb_status_string(int st) {
  switch (st) {
    case SQB_OK: return "ok";
    case SQB_ERR_ARG: return "invalid argument";
    case SQB_ERR_CUDA: return "CUDA error";
    case SQB_ERR_UNSUPPORTED: return "unsupported configuration";
    case SQB_ERR_NOT_BRACKETED: return "Root must be bracketed in Brent's method";
    case SQB_ERR_FERMI_MAXITER: return "Maximum iterations exceeded in brents root finding method";
    case SQB_ERR_NEGATIVE_RHO: return "Element of rho is negative";
    case SQB_ERR_LANCZOS_MAXITER: return "Lanczos exceeded max_iter";
    case SQB_ERR_DENOM_ZERO: return "Denom=0.0 in Nonlocal";
    case SQB_ERR_SPLINE_RANGE: return "out of range in spline interpolation";
    case SQB_ERR_CAPACITY: return "too many projector atoms in one truncation window";
    case SQB_ERR_NONFINITE: return "non-finite value";
    case SQB_ERR_STATE: return "inputs not set";
    case SQB_ERR_BOUNDS: return "device index check failed (bounds-check build)";
    default: return "unknown status";
  }
}

int sqb_create(const sqb_grid *grid, int device, sqb_ctx **out) {
  if (!grid || !out) return SQB_ERR_ARG;
  *out = nullptr;
  const sqb_grid &g = *grid;
  for (int d = 0; d < 3; d++)
    if (g.np[d] <= 0 || g.n_int[d] <= 0) return SQB_ERR_ARG;
  if (g.nloc < 1 || g.npl < 4 || g.npl % 4 != 0 || !(g.delta > 0) || !(g.bet > 0)) return SQB_ERR_ARG;
  if (g.fdn != FDN) return SQB_ERR_UNSUPPORTED;
  if (g.fermi_alg != 1 && g.fermi_alg != 2) return SQB_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) return SQB_ERR_CUDA;
  sqb_ctx *c = new sqb_ctx();
  c->g = g;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return SQB_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  c->n = 2 * g.nloc + 1;
  if (node_kernel_threads(c->n, 2) > 1024) {
    delete c;
    return SQB_ERR_UNSUPPORTED;
  }
  c->nnode = g.np[0] * g.np[1] * g.np[2];
  c->ex = g.np[0] + 2 * g.nloc;
  c->ey = g.np[1] + 2 * g.nloc;
  c->ez = g.np[2] + 2 * g.nloc;
  c->h3 = pow(g.delta, 3);
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  CK(cudaEventCreateWithFlags(&c->ev_order, cudaEventDisableTiming));
  CK(node_kernel_setup(c->n));
  CK(sweep_setup(c->n));
  CK(sweep_forces_setup(c->n));
  const size_t N = c->nnode, K = g.npl + 1;
  CK(dalloc(&c->d_counter, 1));
  CK(dalloc(&c->d_status, 1));
  CK(dalloc(&c->d_proj_points, 3));
  CK(dalloc(&c->d_nodes, N));
  CK(dalloc(&c->d_iters, N));
  CK(dalloc(&c->d_chi, N));
  CK(dalloc(&c->d_zee, N));
  CK(dalloc(&c->d_lmin, N));
  CK(dalloc(&c->d_lmax, N));
  CK(dalloc(&c->d_rho, N));
  CK(dalloc(&c->d_rho_pj, N * K));
  CK(dalloc(&c->d_ci, N * K));
  CK(dalloc(&c->d_xk, K));
  CK(dalloc(&c->d_ctab, K * K));
  CK(dalloc(&c->d_partial, (size_t)2 * (c->sms + 8)));
  CK(dalloc(&c->d_result, 4));
  std::vector<int> nodes(N);
  for (size_t i = 0; i < N; i++) nodes[i] = (int)i;
  CK(cudaMemcpy(c->d_nodes, nodes.data(), N * sizeof(int), cudaMemcpyHostToDevice));
  // Chebyshev-Gauss nodes and cosine table with the expressions of
  // sq.cpp:1239-1255, so the values are the reference's.
  const int npl = g.npl;
  std::vector<double> xk(K), ctab(K * K);
  for (int k = 0; k < npl + 1; k++) xk[k] = cos(M_PI * ((double)((k - 0.5 + 1) / (npl + 1))));
  for (int j = 0; j < npl + 1; j++)
    for (int k = 0; k < npl + 1; k++) ctab[(size_t)j * K + k] = cos((M_PI * (j - 1 + 1)) * ((double)((k - 0.5 + 1) / (npl + 1))));
  CK(cudaMemcpy(c->d_xk, xk.data(), K * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_ctab, ctab.data(), K * K * sizeof(double), cudaMemcpyHostToDevice));
  c->stats.window_points = (long long)c->n * c->n * c->n;
  if (const char *mp = std::getenv("SQDFT_B200_METRICS")) c->metrics_path = mp;
  *out = c;
  return SQB_OK;
}

int sqb_destroy(sqb_ctx *c) {
  if (!c) return SQB_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  void *ptrs[] = {c->d_lay_id, c->d_lay_chi, c->d_rep_box, c->d_rep_gpb, c->d_rep_atom_l, c->d_veff64, c->d_rep_nn, c->d_rep_atom, c->d_rep_off, c->d_typ_tab,
                  c->d_typ_nlocc, c->d_typ_nproj, c->d_typ_lmax, c->d_typ_lloc, c->d_typ_size, c->d_proj_denom,
                  c->d_tables, c->d_rep_xyz, c->d_rep_off_ref, c->d_vjp, c->d_vjp_at, c->d_dtab, c->d_tab64, c->d_scratch, c->d_counter, c->d_nodes,
                  c->d_status, c->d_iters, c->d_proj_points, c->d_chi, c->d_zee, c->d_rho_pj, c->d_lmin,
                  c->d_lmax, c->d_xk, c->d_ctab, c->d_partial, c->d_result, c->d_rho, c->d_ci, c->d_fslots,
                  c->d_f, c->d_tmp, c->d_sens, c->d_loss, c->d_fermi, c->d_loc_type, c->d_loc_atom,
                  c->d_loc_box, c->d_loc_size, c->d_loc_off, c->d_loc_scr_off, c->d_loc_xyz, c->d_loc_tab,
                  c->d_loc_Z, c->d_loc_fields, c->d_loc_scr};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  drop_graph(c);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_order) cudaEventDestroy(c->ev_order);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SQB_OK;
}

int sqb_set_precision(sqb_ctx *c, int precision) {
  if (!c || (precision != SQB_FP64 && precision != SQB_FP32_MIXED && precision != SQB_FP64_LANCZOS_QUAD))
    return SQB_ERR_ARG;
  c->precision = precision;
  drop_graph(c);
  return SQB_OK;
}

int sqb_set_mixed_lanczos(sqb_ctx *c, double tol, double checkerboard) {
  if (!c || !(tol >= 0.0) || !std::isfinite(tol) || !(checkerboard >= 0.0 && checkerboard <= 1.0)) return SQB_ERR_ARG;
  c->mixed_lanczos_tol = tol;
  c->mixed_lanczos_chk = checkerboard;
  drop_graph(c);
  return SQB_OK;
}

int sqb_set_allreduce(sqb_ctx *c, sqb_allreduce_fn fn, void *user) {
  if (!c) return SQB_ERR_ARG;
  c->allreduce = fn;
  c->allreduce_user = user;
  return SQB_OK;
}

int sqb_set_launch(sqb_ctx *c, int ctas_per_sm, int cols_per_thread) {
  if (!c || ctas_per_sm < 0 || ctas_per_sm > 4 || cols_per_thread < -2 || cols_per_thread > 2 ||
      cols_per_thread == -1)
    return SQB_ERR_ARG;
  if (cols_per_thread == -2 && c->n > 32) return SQB_ERR_UNSUPPORTED;
  if (cols_per_thread > 0 && node_kernel_threads(c->n, cols_per_thread) > 1024) return SQB_ERR_UNSUPPORTED;
  c->ctas_per_sm = ctas_per_sm > 0 ? ctas_per_sm : 1;
  c->cols = cols_per_thread;
  drop_graph(c);
  return SQB_OK;
}

int sqb_set_veff(sqb_ctx *c, const double *veff_ext) {
  if (!c || !veff_ext) return SQB_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->ex * c->ey * c->ez;
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(veff_ext[i])) return SQB_ERR_NONFINITE;
  if (!c->d_veff64) CK(dalloc(&c->d_veff64, n));
  CK(cudaMemcpyAsync(c->d_veff64, veff_ext, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->have_veff = true;
  c->have_moments = false;
  return SQB_OK;
}

int sqb_set_veff_device(sqb_ctx *c, const double *veff_ext) {
  if (!c || !veff_ext) return SQB_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t n = (size_t)c->ex * c->ey * c->ez;
  if (!c->d_veff64) CK(dalloc(&c->d_veff64, n));
  // after the work the caller queued on the legacy default stream (which
  // wrote the block), then a device copy; the caller may reuse its buffer
  // once this returns
  CK(cudaEventRecord(c->ev_order, cudaStreamLegacy));
  CK(cudaStreamWaitEvent(c->stream, c->ev_order, 0));
  CK(cudaMemcpyAsync(c->d_veff64, veff_ext, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->have_veff = true;
  c->have_moments = false;
  return SQB_OK;
}

int sqb_set_atoms(sqb_ctx *c, int n_typ, const sqb_species *types, int n_rep, const int *rep_type,
                  const int *rep_atom, const double *rep_xyz, int n_atm) {
  if (!c || n_typ < 0 || n_rep < 0 || n_atm < 0 || (n_typ > 0 && !types)) return SQB_ERR_ARG;
  if (n_rep > 0 && (!rep_type || !rep_atom || !rep_xyz)) return SQB_ERR_ARG;
  cudaSetDevice(c->device);
  c->n_typ = n_typ;
  c->n_rep = n_rep;
  c->n_atm = n_atm;
  c->typ_nproj.assign(n_typ, 0);
  c->typ_nlocc.assign(n_typ, 0);
  std::vector<int> lmax(n_typ), lloc(n_typ), size(n_typ);
  std::vector<long long> ttab(n_typ);
  std::vector<double> denom((size_t)std::max(n_typ, 1) * MAXPROJ_TYPE, 0.0);
  long long tables_len = 0;
  bool all_tables = n_typ > 0;
  for (int t = 0; t < n_typ; t++) {
    const sqb_species &s = types[t];
    if (s.lmax < 0 || s.lmax > 3 || s.nlocc < 0 || s.natm < 0) return SQB_ERR_ARG;
    int np = 0;
    for (int l = 0; l <= s.lmax; l++) {
      if (l == s.lloc) continue;
      for (int m = -l; m <= l; m++) denom[(size_t)t * MAXPROJ_TYPE + np++] = s.denom[l];
      if (s.denom[l] == 0.0) return SQB_ERR_DENOM_ZERO;  // nonlocal.cpp:163
    }
    c->typ_nproj[t] = np;
    c->typ_nlocc[t] = s.nlocc;
    lmax[t] = s.lmax;
    lloc[t] = s.lloc;
    size[t] = s.size;
    ttab[t] = tables_len;
    if (s.tables && s.size >= 3) tables_len += 19LL * s.size;
    else all_tables = false;
  }
  std::vector<int> nn((size_t)4 * std::max(n_rep, 1));
  c->lay_state = 0;  // the layered fields follow the projector tables
  drop_graph(c);    // (their buffers are rebuilt; captured launches hold the old addresses)
  std::vector<long long> off(std::max(n_rep, 1)), off_ref(std::max(n_rep, 1));
  long long total = 0, total_pad = 0;
  for (int r = 0; r < n_rep; r++) {
    const int t = rep_type[r];
    if (t < 0 || t >= n_typ || rep_atom[r] < 0 || rep_atom[r] >= n_atm) return SQB_ERR_ARG;
    nn[4 * r] = nearest_node(rep_xyz[3 * r], c->g.delta);
    nn[4 * r + 1] = nearest_node(rep_xyz[3 * r + 1], c->g.delta);
    nn[4 * r + 2] = nearest_node(rep_xyz[3 * r + 2], c->g.delta);
    nn[4 * r + 3] = t;
    off_ref[r] = total;
    off[r] = total_pad;
    const long long S = 2LL * c->typ_nlocc[t] + 1;
    total += c->typ_nproj[t] * S * S * S;
    total_pad += c->typ_nproj[t] * S * plane_stride((int)S);
  }
  c->tab_total = total;
  c->tab_pad_total = total_pad;
  CK(dalloc(&c->d_rep_nn, nn.size()));
  CK(dalloc(&c->d_rep_atom, std::max(n_rep, 1)));
  CK(dalloc(&c->d_rep_off, off.size()));
  CK(dalloc(&c->d_rep_off_ref, off_ref.size()));
  CK(dalloc(&c->d_rep_xyz, (size_t)3 * std::max(n_rep, 1)));
  CK(dalloc(&c->d_typ_nlocc, std::max(n_typ, 1)));
  CK(dalloc(&c->d_typ_nproj, std::max(n_typ, 1)));
  CK(dalloc(&c->d_typ_lmax, std::max(n_typ, 1)));
  CK(dalloc(&c->d_typ_lloc, std::max(n_typ, 1)));
  CK(dalloc(&c->d_typ_size, std::max(n_typ, 1)));
  CK(dalloc(&c->d_typ_tab, std::max(n_typ, 1)));
  CK(dalloc(&c->d_proj_denom, denom.size()));
  CK(dalloc(&c->d_tab64, (size_t)std::max(total_pad, 1LL)));
  CK(cudaMemset(c->d_tab64, 0, (size_t)std::max(total_pad, 1LL) * sizeof(double)));
  CK(dalloc(&c->d_fslots, (size_t)c->nnode * FSLOTS * 4));
  CK(dalloc(&c->d_f, (size_t)3 * std::max(n_atm, 1)));
  CK(cudaMemcpy(c->d_rep_nn, nn.data(), nn.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (n_rep > 0) {
    CK(cudaMemcpy(c->d_rep_atom, rep_atom, n_rep * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_rep_xyz, rep_xyz, (size_t)3 * n_rep * sizeof(double), cudaMemcpyHostToDevice));
    c->h_rep_xyz.assign(rep_xyz, rep_xyz + (size_t)3 * n_rep);
  }
  CK(cudaMemcpy(c->d_rep_off, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_rep_off_ref, off_ref.data(), off_ref.size() * sizeof(long long), cudaMemcpyHostToDevice));
  if (n_typ > 0) {
    CK(cudaMemcpy(c->d_typ_nlocc, c->typ_nlocc.data(), n_typ * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_typ_nproj, c->typ_nproj.data(), n_typ * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_typ_lmax, lmax.data(), n_typ * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_typ_lloc, lloc.data(), n_typ * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_typ_size, size.data(), n_typ * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_typ_tab, ttab.data(), n_typ * sizeof(long long), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(c->d_proj_denom, denom.data(), denom.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->have_tables = all_tables;
  if (all_tables) {
    CK(dalloc(&c->d_tables, (size_t)tables_len));
    for (int t = 0; t < n_typ; t++)
      CK(cudaMemcpy(c->d_tables + ttab[t], types[t].tables, 19ULL * types[t].size * sizeof(double),
                    cudaMemcpyHostToDevice));
  }
  // Size the node kernel's projector-slice stages for the largest per-plane
  // footprint any window of this block meets.
  {
    unsigned *d_fp = reinterpret_cast<unsigned *>(c->d_counter);
    unsigned fp = 0;
    CK(launch_plane_footprint(c->n, c->g.nloc, c->g.np, c->g.pnode_s, n_rep, c->d_rep_nn, c->d_typ_nlocc,
                              c->d_typ_nproj, d_fp, c->stream));
    CK(cudaMemcpyAsync(&fp, d_fp, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->stage_elems = fp;
  }
  c->h_rep_nn = nn;
  c->have_atoms = true;
  c->have_dtab = false;
  drop_graph(c);
  c->have_proj = total == 0;
  c->have_moments = false;
  return SQB_OK;
}

int sqb_nonlocal_projectors(sqb_ctx *c, double *udvtm_out) {
  NvtxRange nvtx_range("sqb_nonlocal_projectors");
  if (!c) return SQB_ERR_ARG;
  if (!c->have_atoms || !c->have_tables) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  ProjArgs p{};
  p.n_rep = c->n_rep;
  p.delta = c->g.delta;
  p.rep_nn = c->d_rep_nn;
  p.rep_xyz = c->d_rep_xyz;
  p.rep_off = c->d_rep_off;
  p.typ_nlocc = c->d_typ_nlocc;
  p.typ_lmax = c->d_typ_lmax;
  p.typ_lloc = c->d_typ_lloc;
  p.typ_size = c->d_typ_size;
  p.typ_tab = c->d_typ_tab;
  p.tables = c->d_tables;
  p.out64 = c->d_tab64;
  p.total = c->tab_total;
  p.status = c->d_status;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaEventRecord(c->ev0, c->stream));
  CK(launch_projectors(p, c->stream));
  CK(cudaEventRecord(c->ev1, c->stream));
  int rc = read_status(c);
  c->stats.ms_projectors = elapsed(c);
  if (rc) return rc;
  if (udvtm_out && c->tab_total > 0) {
    rc = ensure_tmp(c, (size_t)c->tab_total * sizeof(double));
    if (rc) return rc;
    double *d_ref = reinterpret_cast<double *>(c->d_tmp);
    CK(launch_repack(c->n_rep, c->d_rep_nn, c->d_typ_nlocc, c->d_typ_nproj, c->d_rep_off_ref, c->d_rep_off,
                     c->d_tab64, d_ref, 0, c->stream));
    CK(cudaMemcpyAsync(udvtm_out, d_ref, (size_t)c->tab_total * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  c->have_proj = true;
  c->have_moments = false;
  c->lay_state = 0;
  drop_graph(c);  // the layered fields are rebuilt from the new tables
  return SQB_OK;
}

int sqb_set_projectors(sqb_ctx *c, const double *udvtm) {
  if (!c || (!udvtm && c->tab_total > 0)) return SQB_ERR_ARG;
  if (!c->have_atoms) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  if (c->tab_total > 0) {
    int rc = ensure_tmp(c, (size_t)c->tab_total * sizeof(double));
    if (rc) return rc;
    double *d_ref = reinterpret_cast<double *>(c->d_tmp);
    CK(cudaMemcpyAsync(d_ref, udvtm, (size_t)c->tab_total * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(launch_repack(c->n_rep, c->d_rep_nn, c->d_typ_nlocc, c->d_typ_nproj, c->d_rep_off_ref, c->d_rep_off, d_ref,
                     c->d_tab64, 1, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  c->have_proj = true;
  c->have_moments = false;
  c->lay_state = 0;
  drop_graph(c);  // the layered fields are rebuilt from the new tables
  return SQB_OK;
}

int sqb_hsub_times_vec(sqb_ctx *c, int count, const int *nodes, const double *vin, double *vout) {
  if (!c || count < 0 || (count > 0 && (!nodes || !vin || !vout))) return SQB_ERR_ARG;
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  if (count == 0) return SQB_OK;
  for (int i = 0; i < count; i++)
    if (nodes[i] < 0 || nodes[i] >= c->nnode) return SQB_ERR_ARG;
  cudaSetDevice(c->device);
  const size_t nw = (size_t)c->n * c->n * c->n;
  int rc = ensure_tmp(c, (2 * nw * count) * sizeof(double) + count * sizeof(int) + 64);
  if (rc) return rc;
  double *d_in = c->d_tmp, *d_out = c->d_tmp + nw * count;
  int *d_list = reinterpret_cast<int *>(d_out + nw * count);
  CK(cudaMemcpyAsync(d_in, vin, nw * count * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(d_list, nodes, count * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  NodeArgs a;
  fill_node_args(c, a);
  a.mode = MODE_APPLY;
  a.apply_in = d_in;
  a.apply_out = d_out;
  rc = run_nodes(c, a, d_list, count);
  if (rc) return rc;
  rc = read_status(c);
  if (rc) return rc;
  CK(cudaMemcpy(vout, d_out, nw * count * sizeof(double), cudaMemcpyDeviceToHost));
  return SQB_OK;
}

int sqb_lanczos_moments(sqb_ctx *c, double *chi, double *zee, double *rho_pj, int *lanczos_iters,
                        double *lambda_min, double *lambda_max) {
  NvtxRange nvtx_range("sqb_lanczos_moments");
  if (!c) return SQB_ERR_ARG;
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  NodeArgs a;
  fill_node_args(c, a);
  a.mode = MODE_SQ;
  a.chi = c->d_chi;
  a.zee = c->d_zee;
  a.rho_pj = c->d_rho_pj;
  a.lmin = c->d_lmin;
  a.lmax = c->d_lmax;
  a.lanczos_iters = c->d_iters;
  c->stats.kernel_launches = 0;
  int rc = SQB_OK;
  if (c->use_graph && c->sq_graph_warm && !c->sq_graph) {
    // capture the sequence once its buffers exist (a plain run allocated them)
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    rc = run_sq_nodes(c, a, c->d_nodes, c->nnode);
    if (!rc && launch_minmax(c->d_lmin, c->d_lmax, c->nnode, c->d_result, c->stream) != cudaSuccess) rc = SQB_ERR_CUDA;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (!rc && e == cudaSuccess && cudaGraphInstantiate(&c->sq_graph, g, 0) != cudaSuccess) c->sq_graph = nullptr;
    if (g) cudaGraphDestroy(g);
    if (rc || e != cudaSuccess || !c->sq_graph) {
      c->use_graph = 0;  // fall back to plain launches
      cudaGetLastError();
    }
  }
  CK(cudaEventRecord(c->ev0, c->stream));
  if (c->use_graph && c->sq_graph) {
    CK(cudaGraphLaunch(c->sq_graph, c->stream));
  } else {
    rc = run_sq_nodes(c, a, c->d_nodes, c->nnode);
    if (rc) return rc;
    CK(launch_minmax(c->d_lmin, c->d_lmax, c->nnode, c->d_result, c->stream));
    c->sq_graph_warm = 1;
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  c->stats.kernel_launches += 2;
  rc = read_status(c);
  c->stats.ms_lanczos_moments = elapsed(c);
  if (rc) return rc;
  double mm[2];
  CK(cudaMemcpy(mm, c->d_result, sizeof(mm), cudaMemcpyDeviceToHost));
  rc = reduce(c, &mm[0], 1, SQB_MIN);
  if (!rc) rc = reduce(c, &mm[1], 1, SQB_MAX);
  if (rc) return rc;
  c->lmin_all = mm[0];
  c->lmax_all = mm[1];
  const size_t N = c->nnode, K = c->g.npl + 1;
  std::vector<int> its;
  rc = lanczos_stats(c, its);
  if (rc) return rc;
  if (lanczos_iters) std::memcpy(lanczos_iters, its.data(), N * sizeof(int));
  if (chi) CK(cudaMemcpy(chi, c->d_chi, N * sizeof(double), cudaMemcpyDeviceToHost));
  if (zee) CK(cudaMemcpy(zee, c->d_zee, N * sizeof(double), cudaMemcpyDeviceToHost));
  if (rho_pj) CK(cudaMemcpy(rho_pj, c->d_rho_pj, N * K * sizeof(double), cudaMemcpyDeviceToHost));
  if (lambda_min) CK(cudaMemcpy(lambda_min, c->d_lmin, N * sizeof(double), cudaMemcpyDeviceToHost));
  if (lambda_max) CK(cudaMemcpy(lambda_max, c->d_lmax, N * sizeof(double), cudaMemcpyDeviceToHost));
  c->have_moments = true;
  c->have_ci = false;
  return SQB_OK;
}

int sqb_lanczos_moments_nodes(sqb_ctx *c, int count, const int *nodes, double *chi, double *zee, double *rho_pj,
                              int *lanczos_iters) {
  if (!c || count < 0 || (count > 0 && !nodes)) return SQB_ERR_ARG;
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  if (count == 0) return SQB_OK;
  for (int i = 0; i < count; i++)
    if (nodes[i] < 0 || nodes[i] >= c->nnode) return SQB_ERR_ARG;
  cudaSetDevice(c->device);
  int rc = ensure_tmp(c, (size_t)count * sizeof(int));
  if (rc) return rc;
  int *d_list = reinterpret_cast<int *>(c->d_tmp);
  CK(cudaMemcpyAsync(d_list, nodes, (size_t)count * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  NodeArgs a;
  fill_node_args(c, a);
  a.mode = MODE_SQ;
  a.chi = c->d_chi;
  a.zee = c->d_zee;
  a.rho_pj = c->d_rho_pj;
  a.lmin = c->d_lmin;
  a.lmax = c->d_lmax;
  a.lanczos_iters = c->d_iters;
  c->stats.kernel_launches = 0;
  CK(cudaEventRecord(c->ev0, c->stream));
  rc = run_sq_nodes(c, a, d_list, count);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev1, c->stream));
  c->stats.kernel_launches += 1;
  rc = read_status(c);
  c->stats.ms_lanczos_moments = elapsed(c);
  // the per-node arrays now mix this call's nodes with older results
  c->have_moments = false;
  c->have_ci = false;
  if (rc) return rc;
  const size_t N = c->nnode, K = c->g.npl + 1;
  std::vector<double> buf(N * K);
  std::vector<int> its(N);
  CK(cudaMemcpy(its.data(), c->d_iters, N * sizeof(int), cudaMemcpyDeviceToHost));
  if (lanczos_iters)
    for (int i = 0; i < count; i++) lanczos_iters[i] = its[nodes[i]];
  long long capped = 0, sum = 0;
  int mx = 0;
  const int cap = LANCZOS_MAX_ITER - (c->precision == SQB_FP64_LANCZOS_QUAD ? 1 : 0);
  for (int i = 0; i < count; i++) {
    capped += its[nodes[i]] >= cap;
    sum += its[nodes[i]];
    mx = std::max(mx, its[nodes[i]]);
  }
  c->stats.lanczos_maxiter_nodes = capped;
  c->stats.lanczos_iters = sum;
  c->stats.max_lanczos_iters = mx;
  c->stats.matvecs = sum + count + (c->precision == SQB_FP64_LANCZOS_QUAD ? 0LL : (long long)count * (c->g.npl / 2));
  unsigned long long pp[3] = {0, 0, 0};
  CK(cudaMemcpy(pp, c->d_proj_points, sizeof(pp), cudaMemcpyDeviceToHost));
  c->stats.proj_points = (long long)pp[0];
  c->stats.proj_points_cheb = (long long)pp[1];
  c->stats.proj_points_window = (long long)pp[2];
  if (chi) {
    CK(cudaMemcpy(buf.data(), c->d_chi, N * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < count; i++) chi[i] = buf[nodes[i]];
  }
  if (zee) {
    CK(cudaMemcpy(buf.data(), c->d_zee, N * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < count; i++) zee[i] = buf[nodes[i]];
  }
  if (rho_pj) {
    CK(cudaMemcpy(buf.data(), c->d_rho_pj, N * K * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < count; i++) std::memcpy(rho_pj + (size_t)i * K, &buf[(size_t)nodes[i] * K], K * sizeof(double));
  }
  return SQB_OK;
}

int sqb_ne_constraint(sqb_ctx *c, double lambda_f, double *fval) {
  if (!c || !fval) return SQB_ERR_ARG;
  if (!c->have_moments) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  return ne_constraint(c, lambda_f, fval);
}

int sqb_fermi_level(sqb_ctx *c, int scf_iter, double lambda_warm, double *lambda_f, int *iters) {
  NvtxRange nvtx_range("sqb_fermi_level");
  if (!c || !lambda_f) return SQB_ERR_ARG;
  if (!c->have_moments) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  int it = 0, rc;
  double root = 0.0;
  CK(cudaEventRecord(c->ev0, c->stream));
  if (c->g.fermi_alg == 1) rc = brent(c, c->lmin_all - 1, c->lmax_all + 1, scf_iter, lambda_warm, &root, &it);
  else rc = newton(c, scf_iter <= 1 ? 0.2 : lambda_warm, &root, &it);  // sq.cpp:721-730
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  c->stats.ms_fermi = elapsed(c);
  c->stats.fermi_iters = it;
  if (rc) return rc;
  *lambda_f = root;
  if (iters) *iters = it;
  return SQB_OK;
}

int sqb_density_energy(sqb_ctx *c, double lambda_f, double *rho, double *ci, double *ebs, double *eent) {
  NvtxRange nvtx_range("sqb_density_energy");
  if (!c) return SQB_ERR_ARG;
  if (!c->have_moments) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaEventRecord(c->ev0, c->stream));
  CK(launch_density_energy(fermi_args(c), lambda_f, c->stream));
  CK(cudaEventRecord(c->ev1, c->stream));
  c->stats.kernel_launches += 2;
  int st = 0;
  double r[2];
  CK(cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(r, c->d_result, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->stats.ms_density = elapsed(c);
  c->have_ci = true;
  c->lambda_last = lambda_f;
  if (st & 2) return SQB_ERR_NONFINITE;
  int rc = reduce(c, r, 2, SQB_SUM);
  if (rc) return rc;
  const size_t N = c->nnode, K = c->g.npl + 1;
  if (rho) CK(cudaMemcpy(rho, c->d_rho, N * sizeof(double), cudaMemcpyDeviceToHost));
  if (ci) CK(cudaMemcpy(ci, c->d_ci, N * K * sizeof(double), cudaMemcpyDeviceToHost));
  if (ebs) *ebs = r[0];
  if (eent) *eent = r[1];
  if (st & 1) return SQB_ERR_NEGATIVE_RHO;
  return SQB_OK;
}

// Defect check of the fast forms (FP32-mixed, Lanczos quadrature) when their
// Lanczos stop is looser than the grid's: the density of every node at
// bounds moved by 4x the stop at either end is evaluated from the node's own
// moments (re-expansion, bound_sens_kernel); nodes whose density moves by
// more than half the budget times max rho are redone by the FP64 parity path
// (the reference's bounds and moments), and the Fermi level is solved again.
int defect_check(sqb_ctx *c, int scf_iter, double lambda_warm, double *lam) {
  NvtxRange nvtx_range("sqb_defect_check");
  c->stats.defect_nodes = 0;
  c->stats.ms_defect = 0.0;
  const double tol_eff = std::max(c->g.lanczos_tol, c->mixed_lanczos_tol);
  if (c->precision == SQB_FP64 || !(c->defect_budget > 0.0) || !(tol_eff > c->g.lanczos_tol)) return SQB_OK;
  const int N = c->nnode;
  if (!c->d_sens) CK(dalloc(&c->d_sens, (size_t)std::max(N, 1)));
  const double ms_first_fermi = c->stats.ms_fermi;
  CK(cudaEventRecord(c->ev0, c->stream));
  CK(launch_bound_sens(fermi_args(c), *lam, 4.0 * tol_eff, c->d_sens, c->d_rho, c->stream));
  std::vector<double> sens(N), r0(N);
  CK(cudaMemcpyAsync(sens.data(), c->d_sens, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(r0.data(), c->d_rho, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double mx = 0.0;
  for (int i = 0; i < N; i++) mx = std::max(mx, r0[i]);
  int rc = reduce(c, &mx, 1, SQB_MAX);
  if (rc) return rc;
  const double thr = 0.5 * c->defect_budget * mx;
  std::vector<int> list;
  for (int i = 0; i < N; i++)
    if (!(sens[i] <= thr)) list.push_back(i);
  double cnt = (double)list.size();
  rc = reduce(c, &cnt, 1, SQB_SUM);
  if (rc) return rc;
  c->stats.defect_nodes = (long long)cnt;
  c->stats.kernel_launches += 1;
  if (cnt > 0) {
    if (!list.empty()) {
      rc = ensure_tmp(c, list.size() * sizeof(int));
      if (rc) return rc;
      int *d_list = reinterpret_cast<int *>(c->d_tmp);
      CK(cudaMemcpyAsync(d_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
      NodeArgs a;
      fill_node_args(c, a);
      a.mode = MODE_SQ;
      a.mixed = 0;  // the FP64 parity path
      a.lq = 0;
      a.lz_chk = 0.0;
      a.lanczos_tol = c->g.lanczos_tol;
      a.chi = c->d_chi;
      a.zee = c->d_zee;
      a.rho_pj = c->d_rho_pj;
      a.lmin = c->d_lmin;
      a.lmax = c->d_lmax;
      a.lanczos_iters = c->d_iters;
      rc = run_sq_nodes(c, a, d_list, (int)list.size());
      if (rc) return rc;
      c->stats.kernel_launches += 1;
    }
    CK(launch_minmax(c->d_lmin, c->d_lmax, c->nnode, c->d_result, c->stream));
    c->stats.kernel_launches += 1;
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  rc = read_status(c);
  c->stats.ms_defect = elapsed(c);
  if (rc || cnt == 0) return rc;
  double mm[2];
  CK(cudaMemcpy(mm, c->d_result, sizeof(mm), cudaMemcpyDeviceToHost));
  rc = reduce(c, &mm[0], 1, SQB_MIN);
  if (!rc) rc = reduce(c, &mm[1], 1, SQB_MAX);
  if (rc) return rc;
  c->lmin_all = mm[0];
  c->lmax_all = mm[1];
  rc = sqb_fermi_level(c, scf_iter, lambda_warm, lam, nullptr);
  c->stats.ms_defect += ms_first_fermi;  // the first Fermi solve, now superseded
  return rc;
}

int sqb_set_defect_check(sqb_ctx *c, double budget) {
  if (!c || !(budget >= 0.0) || !std::isfinite(budget)) return SQB_ERR_ARG;
  c->defect_budget = budget;
  return SQB_OK;
}

static int spectral_quadrature(sqb_ctx *c, int scf_iter, double *lambda_f, double *rho, double *rho_pj, double *ci,
                               double *chi, double *zee, double *ebs, double *eent);

int sqb_spectral_quadrature(sqb_ctx *c, int scf_iter, double *lambda_f, double *rho, double *rho_pj, double *ci,
                            double *chi, double *zee, double *ebs, double *eent) {
  if (!c || !lambda_f) return SQB_ERR_ARG;
  NvtxRange r("sqb_spectral_quadrature");
  const int rc = spectral_quadrature(c, scf_iter, lambda_f, rho, rho_pj, ci, chi, zee, ebs, eent);
  write_metrics(c, "spectral_quadrature", rc, *lambda_f);
  return rc;
}

// The whole SQ step as one CUDA graph (sqb_set_graph(ctx, 2)): the node
// kernel and the bound min/max, the Fermi solve as a conditional while node
// (NeConstraint, block sums, fermi_step) and the density assembly; one launch
// and one synchronisation per step.  Single rank only (the reductions of
// several ranks go through the host) and without the defect check.
static int build_step_graph(sqb_ctx *c) {
  if (!c->d_fermi) CK(cudaMalloc((void **)&c->d_fermi, sizeof(FermiDev)));
  {  // allocate what the captured launches use (no allocation inside a capture)
    size_t stride = 0;
    const int rc0 = ensure_sweep_scratch(c, std::max(1, std::min(c->sms, c->nnode)), &stride);
    if (rc0) return rc0;
  }
  NodeArgs a;
  fill_node_args(c, a);
  a.mode = MODE_SQ;
  a.chi = c->d_chi;
  a.zee = c->d_zee;
  a.rho_pj = c->d_rho_pj;
  a.lmin = c->d_lmin;
  a.lmax = c->d_lmax;
  a.lanczos_iters = c->d_iters;
  FermiArgs fa = fermi_args(c);
  fa.lam_dev = &c->d_fermi->x;
  FermiArgs fd = fermi_args(c);
  fd.lam_dev = &c->d_fermi->root;
  fd.status = &c->d_fermi->dstat;
  const int deriv = c->g.fermi_alg == 2;
  cudaGraph_t g = nullptr;
  int rc = SQB_OK;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  rc = run_sq_nodes(c, a, c->d_nodes, c->nnode);
  if (!rc && launch_minmax(c->d_lmin, c->d_lmax, c->nnode, c->d_result, c->stream) != cudaSuccess) rc = SQB_ERR_CUDA;
  if (!rc && launch_fermi_init(c->d_fermi, c->d_result, c->stream) != cudaSuccess) rc = SQB_ERR_CUDA;
  cudaGraphConditionalHandle h{};
  if (!rc) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraphNode_t wnode = nullptr;
    cudaGraphNodeParams cp{};
    if (cudaStreamGetCaptureInfo(c->stream, &cs, nullptr, &cg, &deps, &ndeps) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
      rc = SQB_ERR_CUDA;
    } else {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      if (cudaGraphAddNode(&wnode, cg, deps, ndeps, &cp) != cudaSuccess ||
          cudaStreamUpdateCaptureDependencies(c->stream, &wnode, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
        rc = SQB_ERR_CUDA;
    }
    if (!rc) {  // the loop body, captured on a second stream into the while node's graph
      cudaStream_t bs = nullptr;
      if (cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking) != cudaSuccess) {
        rc = SQB_ERR_CUDA;
      } else {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaGraph_t got = nullptr;
        if (cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
          rc = SQB_ERR_CUDA;
        if (!rc && launch_ne_constraint(fa, 0.0, deriv, bs) != cudaSuccess) rc = SQB_ERR_CUDA;
        if (!rc && launch_fermi_step(c->d_fermi, c->d_result, h, bs) != cudaSuccess) rc = SQB_ERR_CUDA;
        if (cudaStreamEndCapture(bs, &got) != cudaSuccess) rc = SQB_ERR_CUDA;
        cudaStreamDestroy(bs);
      }
    }
  }
  if (!rc && launch_density_energy(fd, 0.0, c->stream) != cudaSuccess) rc = SQB_ERR_CUDA;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (!rc && e == cudaSuccess && cudaGraphInstantiate(&c->step_graph, g, 0) != cudaSuccess) c->step_graph = nullptr;
  if (g) cudaGraphDestroy(g);
  if (rc || e != cudaSuccess || !c->step_graph) {
    cudaGetLastError();
    c->step_graph = nullptr;
    return rc ? rc : SQB_ERR_CUDA;
  }
  return SQB_OK;
}

static int run_step_graph(sqb_ctx *c, int scf_iter, double lambda_warm, double *lambda_f, double *rho,
                          double *rho_pj, double *ci, double *chi, double *zee, double *ebs, double *eent) {
  if (!c->step_graph) {
    int rc0 = build_step_graph(c);
    if (rc0) return rc0;
  }
  FermiDev st{};
  st.alg = c->g.fermi_alg;
  st.scf_iter = scf_iter;
  st.lambda_warm = lambda_warm;
  st.tol = c->g.fermi_tol;
  st.h3 = pow(c->g.delta, 3);
  st.ncharge = c->g.ncharge;
  st.bet = c->g.bet;
  CK(cudaMemcpyAsync(c->d_fermi, &st, sizeof(st), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  c->stats = sqb_stats{};
  c->stats.window_points = (long long)c->n * c->n * c->n;
  CK(cudaEventRecord(c->ev0, c->stream));
  CK(cudaGraphLaunch(c->step_graph, c->stream));
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaMemcpyAsync(&st, c->d_fermi, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  double r[2];
  CK(cudaMemcpyAsync(r, c->d_result, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
  int stw = 0;
  CK(cudaMemcpyAsync(&stw, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->stats.ms_lanczos_moments = elapsed(c);  // the whole step in graph mode
  c->stats.node_kernel = SQB_KERNEL_SWEEP;
  c->stats.kernel_launches = 1;
  int rc = status_to_err(stw);
  if (rc) return rc;
  std::vector<int> its;
  rc = lanczos_stats(c, its);
  if (rc) return rc;
  c->have_moments = true;
  c->have_ci = true;
  c->lmin_all = st.lmin_all;
  c->lmax_all = st.lmax_all;
  c->stats.fermi_iters = st.iters;
  if (st.status == -1) return SQB_ERR_NOT_BRACKETED;
  if (st.status == -2) return SQB_ERR_FERMI_MAXITER;
  if (st.status != 1) return SQB_ERR_NONFINITE;
  c->lambda_last = st.root;
  *lambda_f = st.root;
  if (st.dstat & 2) return SQB_ERR_NONFINITE;
  const size_t N = c->nnode, K = c->g.npl + 1;
  if (chi) CK(cudaMemcpy(chi, c->d_chi, N * sizeof(double), cudaMemcpyDeviceToHost));
  if (zee) CK(cudaMemcpy(zee, c->d_zee, N * sizeof(double), cudaMemcpyDeviceToHost));
  if (rho_pj) CK(cudaMemcpy(rho_pj, c->d_rho_pj, N * K * sizeof(double), cudaMemcpyDeviceToHost));
  if (rho) CK(cudaMemcpy(rho, c->d_rho, N * sizeof(double), cudaMemcpyDeviceToHost));
  if (ci) CK(cudaMemcpy(ci, c->d_ci, N * K * sizeof(double), cudaMemcpyDeviceToHost));
  if (ebs) *ebs = r[0];
  if (eent) *eent = r[1];
  if (st.dstat & 1) return SQB_ERR_NEGATIVE_RHO;
  return SQB_OK;
}

static int spectral_quadrature(sqb_ctx *c, int scf_iter, double *lambda_f, double *rho, double *rho_pj, double *ci,
                               double *chi, double *zee, double *ebs, double *eent) {
  const double tol_eff = std::max(c->g.lanczos_tol, c->mixed_lanczos_tol);
  const bool defect = c->precision != SQB_FP64 && c->defect_budget > 0.0 && tol_eff > c->g.lanczos_tol;
  if (c->use_graph == 2 && !c->allreduce && !defect && c->have_veff && c->have_atoms && c->have_proj) {
    bool sw = false;
    int rc0 = use_sweep(c, &sw);
    if (rc0) return rc0;
    if (sw) return run_step_graph(c, scf_iter, *lambda_f, lambda_f, rho, rho_pj, ci, chi, zee, ebs, eent);
  }
  int rc = sqb_lanczos_moments(c, chi, zee, rho_pj, nullptr, nullptr, nullptr);
  if (rc) return rc;
  double lam = 0.0;
  rc = sqb_fermi_level(c, scf_iter, *lambda_f, &lam, nullptr);
  if (rc) return rc;
  rc = defect_check(c, scf_iter, *lambda_f, &lam);
  if (rc) return rc;
  if (c->stats.defect_nodes > 0) {  // the redone nodes' bounds and moments
    const size_t N = c->nnode, K = c->g.npl + 1;
    if (chi) CK(cudaMemcpy(chi, c->d_chi, N * sizeof(double), cudaMemcpyDeviceToHost));
    if (zee) CK(cudaMemcpy(zee, c->d_zee, N * sizeof(double), cudaMemcpyDeviceToHost));
    if (rho_pj) CK(cudaMemcpy(rho_pj, c->d_rho_pj, N * K * sizeof(double), cudaMemcpyDeviceToHost));
  }
  *lambda_f = lam;
  return sqb_density_energy(c, lam, rho, ci, ebs, eent);
}

int sqb_set_sweep_rows(sqb_ctx *c, int rows) {
  if (!c || (rows != 0 && rows != 2 && rows != 3)) return SQB_ERR_ARG;
  if (rows == 3 && !sweep_rows_supported(c->n, 3)) return SQB_ERR_UNSUPPORTED;
  c->sweep_ry = rows;
  drop_graph(c);
  return SQB_OK;
}

int sqb_test_stage_wait(sqb_ctx *c, unsigned extra_bytes, double wait_ms) {
  if (!c || !(wait_ms >= 0.0) || wait_ms > 10000.0 || extra_bytes % 16 != 0 || extra_bytes > 4096u)
    return SQB_ERR_ARG;
  c->test_extra_tx = extra_bytes;
  c->test_wait_ns = (unsigned long long)(wait_ms * 1e6);
  return SQB_OK;
}

int sqb_set_node_kernel(sqb_ctx *c, int kernel) {
  if (!c || kernel < SQB_KERNEL_AUTO || kernel > SQB_KERNEL_SWEEP) return SQB_ERR_ARG;
  if (kernel == SQB_KERNEL_SWEEP && c->have_proj) {
    cudaSetDevice(c->device);
    const int rc = ensure_layers(c);
    if (rc) return rc;
    if (c->lay_state != 1) return SQB_ERR_UNSUPPORTED;
  }
  c->node_kernel = kernel;
  drop_graph(c);
  return SQB_OK;
}

int sqb_set_graph(sqb_ctx *c, int on) {
  if (!c || on < 0 || on > 2) return SQB_ERR_ARG;
  c->use_graph = on;
  drop_graph(c);
  return SQB_OK;
}

int sqb_autotune(sqb_ctx *c, int sample, int *chosen, double *ms_out) {
  if (!c || sample < 0) return SQB_ERR_ARG;
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  const int N = c->nnode;
  int count = sample > 0 ? sample : 2 * c->sms;
  if (count > N) count = N;
  std::vector<int> list(count);
  for (int i = 0; i < count; i++) list[i] = (int)((long long)i * N / count);  // evenly spaced nodes
  int rc = ensure_tmp(c, (size_t)count * sizeof(int));
  if (rc) return rc;
  int *d_list = reinterpret_cast<int *>(c->d_tmp);
  CK(cudaMemcpy(d_list, list.data(), (size_t)count * sizeof(int), cudaMemcpyHostToDevice));
  const int cands[3] = {1, 2, -2};
  double ms[3] = {-1.0, -1.0, -1.0};
  const int keep = c->cols;
  int best = -1;
  for (int k = 0; k < 3; k++) {
    const int cols = cands[k];
    if (cols == -2 && c->n > 32) continue;
    if (node_kernel_threads(c->n, cols) > 1024) continue;
    c->cols = cols;
    NodeArgs a;
    fill_node_args(c, a);
    a.mode = MODE_SQ;
    a.chi = c->d_chi;
    a.zee = c->d_zee;
    a.rho_pj = c->d_rho_pj;
    a.lmin = c->d_lmin;
    a.lmax = c->d_lmax;
    a.lanczos_iters = c->d_iters;
    float t = 0.f;
    for (int rep = 0; rep < 2; rep++) {  // the first launch of a variant is a warm-up
      CK(cudaEventRecord(c->ev0, c->stream));
      rc = run_nodes(c, a, d_list, count);
      if (rc) {
        c->cols = keep;
        return rc;
      }
      CK(cudaEventRecord(c->ev1, c->stream));
      rc = read_status(c);
      if (rc) {
        c->cols = keep;
        return rc;
      }
      t = elapsed(c);
    }
    ms[k] = t;
    if (best < 0 || ms[k] < ms[best]) best = k;
  }
  c->cols = best >= 0 ? cands[best] : keep;
  drop_graph(c);
  // the sample runs overwrote part of the per-node outputs
  c->have_moments = false;
  c->have_ci = false;
  if (chosen) *chosen = c->cols;
  if (ms_out)
    for (int k = 0; k < 3; k++) ms_out[k] = ms[k];
  return SQB_OK;
}

int sqb_autotune_sweep(sqb_ctx *c, int sample, int *rows, double *ms_out) {
  if (!c || sample < 0) return SQB_ERR_ARG;
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  bool sw = false;
  int rc = use_sweep(c, &sw);
  if (rc) return rc;
  if (!sw) return SQB_ERR_UNSUPPORTED;
  const int N = c->nnode;
  int count = sample > 0 ? sample : 2 * c->sms;
  if (count > N) count = N;
  std::vector<int> list(count);
  for (int i = 0; i < count; i++) list[i] = (int)((long long)i * N / count);  // evenly spaced nodes
  rc = ensure_tmp(c, (size_t)count * sizeof(int));
  if (rc) return rc;
  int *d_list = reinterpret_cast<int *>(c->d_tmp);
  CK(cudaMemcpy(d_list, list.data(), (size_t)count * sizeof(int), cudaMemcpyHostToDevice));
  const int keep = c->sweep_ry;
  double ms[2] = {-1.0, -1.0};
  int best = 0;
  for (int k = 0; k < 2; k++) {
    c->sweep_ry = 2 + k;
    if (sweep_rows(c) != c->sweep_ry) continue;  // not covered for this window
    NodeArgs a;
    fill_node_args(c, a);
    a.mode = MODE_SQ;
    a.chi = c->d_chi;
    a.zee = c->d_zee;
    a.rho_pj = c->d_rho_pj;
    a.lmin = c->d_lmin;
    a.lmax = c->d_lmax;
    a.lanczos_iters = c->d_iters;
    float t = 0.f;
    for (int rep = 0; rep < 2; rep++) {  // the first launch of a variant is a warm-up
      CK(cudaEventRecord(c->ev0, c->stream));
      rc = run_sq_nodes(c, a, d_list, count);
      if (!rc) {
        CK(cudaEventRecord(c->ev1, c->stream));
        rc = read_status(c);
      }
      if (rc) {
        c->sweep_ry = keep;
        return rc;
      }
      t = elapsed(c);
    }
    ms[k] = t;
    if (ms[best] < 0.0 || ms[k] < ms[best]) best = k;
  }
  c->sweep_ry = 2 + best;
  drop_graph(c);
  c->have_moments = false;  // the sample runs overwrote part of the per-node outputs
  c->have_ci = false;
  if (rows) *rows = c->sweep_ry;
  if (ms_out) {
    ms_out[0] = ms[0];
    ms_out[1] = ms[1];
  }
  return SQB_OK;
}

int sqb_moments_at(sqb_ctx *c, const double *chi, const double *zee, double *rho_pj) {
  if (!c || !chi || !zee) return SQB_ERR_ARG;
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  const size_t N = c->nnode, K = c->g.npl + 1;
  for (size_t i = 0; i < N; i++)
    if (!std::isfinite(chi[i]) || !(zee[i] > 0.0) || !std::isfinite(zee[i])) return SQB_ERR_ARG;
  cudaSetDevice(c->device);
  CK(cudaMemcpy(c->d_chi, chi, N * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_zee, zee, N * sizeof(double), cudaMemcpyHostToDevice));
  NodeArgs a;
  fill_node_args(c, a);
  a.mode = MODE_MOMENTS;
  a.chi_in = c->d_chi;
  a.zee_in = c->d_zee;
  a.rho_pj = c->d_rho_pj;
  CK(cudaEventRecord(c->ev0, c->stream));
  int rc = run_nodes(c, a, c->d_nodes, c->nnode);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev1, c->stream));
  rc = read_status(c);
  c->stats.ms_lanczos_moments = elapsed(c);
  if (rc) return rc;
  c->have_moments = true;
  c->have_ci = false;
  if (rho_pj) CK(cudaMemcpy(rho_pj, c->d_rho_pj, N * K * sizeof(double), cudaMemcpyDeviceToHost));
  return SQB_OK;
}

// Derivative tables dchi/dR_alpha of every replica's projectors: central
// differences of the projector kernel at the replica positions +-eps along
// each axis, the balls' grid centres held fixed (the nearest node does not
// move for so small a step).  O(eps^2) = 1e-8 relative.
static int ensure_dtab(sqb_ctx *c) {
  if (c->have_dtab) return SQB_OK;
  if (!c->have_tables) return SQB_ERR_STATE;
  const long long T = c->tab_pad_total;
  if (T == 0) {
    c->have_dtab = true;
    return SQB_OK;
  }
  if (c->d_dtab) cudaFree(c->d_dtab);
  c->d_dtab = nullptr;
  CK(dalloc(&c->d_dtab, (size_t)3 * T));
  const size_t nr3 = (size_t)3 * c->n_rep;
  int rc = ensure_tmp(c, (2 * (size_t)T + nr3) * sizeof(double));
  if (rc) return rc;
  double *plus = reinterpret_cast<double *>(c->d_tmp), *minus = plus + T, *xyz = minus + T;
  const double eps = 1e-4;
  std::vector<double> sh(nr3);
  ProjArgs p{};
  p.n_rep = c->n_rep;
  p.delta = c->g.delta;
  p.rep_nn = c->d_rep_nn;
  p.rep_xyz = xyz;
  p.rep_off = c->d_rep_off;
  p.typ_nlocc = c->d_typ_nlocc;
  p.typ_lmax = c->d_typ_lmax;
  p.typ_lloc = c->d_typ_lloc;
  p.typ_size = c->d_typ_size;
  p.typ_tab = c->d_typ_tab;
  p.tables = c->d_tables;
  p.total = c->tab_total;
  p.status = c->d_status;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(plus, 0, 2 * (size_t)T * sizeof(double), c->stream));  // plane padding stays zero
  for (int al = 0; al < 3; al++) {
    for (int s = 0; s < 2; s++) {
      sh = c->h_rep_xyz;
      for (int r = 0; r < c->n_rep; r++) sh[3 * r + al] += s == 0 ? eps : -eps;
      CK(cudaMemcpyAsync(xyz, sh.data(), nr3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      p.out64 = s == 0 ? plus : minus;
      CK(launch_projectors(p, c->stream));
      CK(cudaStreamSynchronize(c->stream));  // sh is reused
    }
    CK(launch_fd_combine(plus, minus, c->d_dtab + (size_t)al * T, T, 0.5 / eps, c->stream));
  }
  rc = read_status(c);
  if (rc) return rc;
  c->have_dtab = true;
  return SQB_OK;
}

}  // extern "C"

// Moment adjoint on the plane-streaming kernel (node_vjp): buffers, then the
// weights dL/dmu [N][npl+1] filled by `fill` into the device array it is
// given (a copy from the host, or a kernel), then the launch.
template <typename Fill>
static int moments_vjp(sqb_ctx *c, Fill fill, double *g_veff, double *g_atoms) {
  const size_t N = c->nnode, K = c->g.npl + 1;
  const size_t nw = (size_t)c->n * c->n * c->n;
  const size_t ext = (size_t)c->ex * c->ey * c->ez;
  const int nseg = (c->g.npl + VJP_K - 1) / VJP_K;
  const size_t per = ((size_t)(2 * nseg + VJP_K + 4) * nw + (size_t)nseg * MAXP + 31) & ~size_t(31);  // doubles
  int grid = c->sms * (c->ctas_per_sm > 0 ? c->ctas_per_sm : 1);
  if ((size_t)grid > N) grid = (int)N;
  const size_t need = (per * grid + N * K + ext) * sizeof(double);
  if (c->vjp_bytes < need) {
    if (c->d_vjp) cudaFree(c->d_vjp);
    c->d_vjp = nullptr;
    c->vjp_bytes = 0;
    CK(cudaMalloc((void **)&c->d_vjp, need));
    c->vjp_bytes = need;
  }
  double *d_scr = c->d_vjp, *d_g = d_scr + per * grid, *d_out = d_g + N * K;
  const size_t per_at = (size_t)(4 * VJP_K + 12) * MAXP;  // doubles per CTA
  double *d_gat = nullptr;
  if (g_atoms) {
    int rc0 = ensure_dtab(c);
    if (rc0) return rc0;
    const size_t need_at = (per_at * grid + (size_t)3 * std::max(c->n_atm, 1)) * sizeof(double);
    if (c->vjp_at_bytes < need_at) {
      if (c->d_vjp_at) cudaFree(c->d_vjp_at);
      c->d_vjp_at = nullptr;
      c->vjp_at_bytes = 0;
      CK(cudaMalloc((void **)&c->d_vjp_at, need_at));
      c->vjp_at_bytes = need_at;
    }
    d_gat = c->d_vjp_at + per_at * grid;
    CK(cudaMemsetAsync(d_gat, 0, (size_t)3 * std::max(c->n_atm, 1) * sizeof(double), c->stream));
  }
  int rc = fill(d_g);
  if (rc) return rc;
  CK(cudaMemsetAsync(d_out, 0, ext * sizeof(double), c->stream));
  NodeArgs a;
  fill_node_args(c, a);
  a.mode = MODE_VJP;
  a.chi_in = c->d_chi;
  a.zee_in = c->d_zee;
  a.gmu = d_g;
  a.vjp = d_scr;
  a.vjp_stride = per;
  a.g_veff = d_out;
  if (g_atoms) {
    a.dtab = c->d_dtab;
    a.dtab_stride = c->tab_pad_total;
    a.g_atoms = d_gat;
    a.vjp_at = c->d_vjp_at;
    a.vjp_at_stride = per_at;
  }
  CK(cudaEventRecord(c->ev0, c->stream));
  rc = run_nodes(c, a, c->d_nodes, c->nnode);
  if (rc) return rc;
  CK(cudaEventRecord(c->ev1, c->stream));
  rc = read_status(c);
  c->stats.ms_vjp = elapsed(c);
  if (rc) return rc;
  CK(cudaMemcpy(g_veff, d_out, ext * sizeof(double), cudaMemcpyDeviceToHost));
  if (g_atoms && c->n_atm > 0) {
    CK(cudaMemcpy(g_atoms, d_gat, (size_t)3 * c->n_atm * sizeof(double), cudaMemcpyDeviceToHost));
    return reduce(c, g_atoms, 3 * c->n_atm, SQB_SUM);
  }
  return SQB_OK;
}

extern "C" {

int sqb_moments_vjp(sqb_ctx *c, const double *g_mu, double *g_veff, double *g_atoms) {
  NvtxRange nvtx_range("sqb_moments_vjp");
  if (!c || !g_mu || !g_veff) return SQB_ERR_ARG;
  if (!c->have_moments) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  const size_t NK = (size_t)c->nnode * (c->g.npl + 1);
  return moments_vjp(
      c,
      [&](double *d_g) -> int {
        CK(cudaMemcpyAsync(d_g, g_mu, NK * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        return SQB_OK;
      },
      g_veff, g_atoms);
}

int sqb_density_loss(sqb_ctx *c, const double *w, double *loss) {
  if (!c || !w || !loss) return SQB_ERR_ARG;
  if (!c->have_ci) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  std::vector<double> rho(c->nnode);
  CK(cudaMemcpy(rho.data(), c->d_rho, rho.size() * sizeof(double), cudaMemcpyDeviceToHost));
  double l = 0.0;
  for (int p = 0; p < c->nnode; p++) l += w[p] * rho[p];
  const int rc = reduce(c, &l, 1, SQB_SUM);
  if (rc) return rc;
  *loss = l;
  return SQB_OK;
}

int sqb_density_loss_vjp(sqb_ctx *c, const double *w, int fixed_electrons, double grad_l, double *g_veff,
                         double *g_atoms) {
  NvtxRange nvtx_range("sqb_density_loss_vjp");
  if (!c || !w || !g_veff || !std::isfinite(grad_l)) return SQB_ERR_ARG;
  if (!c->have_moments || !c->have_ci) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  const int N = c->nnode, K = c->g.npl + 1;
  if (c->loss_n < N) {
    CK(dalloc(&c->d_loss, (size_t)2 * std::max(N, 1)));
    c->loss_n = N;
  }
  double *d_w = c->d_loss, *d_sgn = c->d_loss + N;
  CK(cudaMemcpyAsync(d_w, w, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(launch_loss_lambda(fermi_args(c), c->lambda_last, d_w, fixed_electrons ? 1 : 0, d_sgn, c->stream));
  double sums[2];
  CK(cudaMemcpyAsync(sums, c->d_result, sizeof(sums), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int rc = reduce(c, sums, 2, SQB_SUM);
  if (rc) return rc;
  // a fixed electron count N_e = h^3 sum_p rho_p moves the Fermi level with
  // Veff: dL/dVeff = dL/dVeff|_lambda - kappa dN_e/dVeff|_lambda,
  // kappa = (dL/dlambda) / (dN_e/dlambda), one adjoint with weights w - kappa h^3
  double off = 0.0;
  if (fixed_electrons) {
    if (!(sums[1] != 0.0) || !std::isfinite(sums[0] / sums[1])) return SQB_ERR_NONFINITE;
    off = sums[0] / sums[1];  // kappa h^3
  }
  return moments_vjp(
      c,
      [&](double *d_g) -> int {
        CK(launch_loss_gmu(N, K, c->d_ci, d_w, d_sgn, 2.0 * grad_l, off, d_g, c->stream));
        return SQB_OK;
      },
      g_veff, g_atoms);
}
static int forces_nonlocal(sqb_ctx *c, const double *chi, const double *zee, const double *ci, double *forces);

int sqb_forces_nonlocal(sqb_ctx *c, const double *chi, const double *zee, const double *ci, double *forces) {
  if (!c || !forces) return SQB_ERR_ARG;
  NvtxRange r("sqb_forces_nonlocal");
  const int rc = forces_nonlocal(c, chi, zee, ci, forces);
  write_metrics(c, "forces_nonlocal", rc, 0.0);
  return rc;
}

static int forces_nonlocal(sqb_ctx *c, const double *chi, const double *zee, const double *ci, double *forces) {
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  const size_t N = c->nnode, K = c->g.npl + 1;
  if (chi || zee || ci) {
    if (!chi || !zee || !ci) return SQB_ERR_ARG;
    CK(cudaMemcpy(c->d_chi, chi, N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_zee, zee, N * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_ci, ci, N * K * sizeof(double), cudaMemcpyHostToDevice));
  } else if (!c->have_ci) {
    return SQB_ERR_STATE;
  }
  bool sw = false;
  int rc = use_sweep(c, &sw);
  if (rc) return rc;
  c->stats.kernel_launches = 0;
  c->stats.node_kernel = sw ? SQB_KERNEL_SWEEP : SQB_KERNEL_PLANE;
  if (sw) {
    const int grid = std::max(1, std::min(c->sms, c->nnode));
    size_t stride = 0;
    rc = ensure_sweep_scratch(c, grid, &stride);
    if (rc) return rc;
    SweepArgs s;
    fill_sweep_args(c, c->d_nodes, c->nnode, stride, s);
    s.chi = c->d_chi;
    s.zee = c->d_zee;
    s.ci = c->d_ci;
    s.fslots = c->d_fslots;
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(cudaMemsetAsync(c->d_counter, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->d_proj_points, 0, 3 * sizeof(unsigned long long), c->stream));
    CK(launch_sweep_forces(s, c->precision == SQB_FP32_MIXED, grid, c->stream));
  } else {
    NodeArgs a;
    fill_node_args(c, a);
    a.mode = MODE_FORCES;
    a.chi_in = c->d_chi;
    a.zee_in = c->d_zee;
    a.ci = c->d_ci;
    a.fslots = c->d_fslots;
    CK(cudaEventRecord(c->ev0, c->stream));
    rc = run_nodes(c, a, c->d_nodes, c->nnode);
    if (rc) return rc;
  }
  CK(launch_force_reduce(c->d_fslots, c->nnode, c->n_atm, c->d_f, c->stream));
  CK(cudaEventRecord(c->ev1, c->stream));
  c->stats.kernel_launches += 2;
  rc = read_status(c);
  c->stats.ms_forces = elapsed(c);
  if (rc) return rc;
  if (c->n_atm > 0) CK(cudaMemcpy(forces, c->d_f, (size_t)3 * c->n_atm * sizeof(double), cudaMemcpyDeviceToHost));
  if (sw) {  // the projector points the pass touched (roofline accounting)
    unsigned long long pp[3] = {0, 0, 0};
    CK(cudaMemcpy(pp, c->d_proj_points, sizeof(pp), cudaMemcpyDeviceToHost));
    c->stats.proj_points = (long long)pp[0];
    c->stats.proj_points_cheb = (long long)pp[1];
    c->stats.proj_points_window = (long long)pp[2];
  }
  return reduce(c, forces, 3 * c->n_atm, SQB_SUM);
}

// Fixed scratch of sqb_lanczos_moments_noalloc: header (work-queue counter,
// status word), then the node list, then the per-CTA window slots.  Host code
// must not pass this symbol to a kernel: its device address comes from
// cudaGetSymbolAddress, looked up once per device with that device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SQB_NOALLOC_SCRATCH_BYTES];
static void *g_noalloc_addr[256];
static std::mutex g_noalloc_mu;

static int noalloc_base(int device, unsigned char **base) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (device < 0 || device >= 256) return SQB_ERR_ARG;
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "sqdft_b200: cudaGetSymbolAddress of the no-alloc scratch: %s\n", cudaGetErrorString(e));
      return SQB_ERR_CUDA;
    }
    g_noalloc_addr[device] = p;
  }
  *base = static_cast<unsigned char *>(g_noalloc_addr[device]);
  return SQB_OK;
}

int sqb_lanczos_moments_noalloc(sqb_ctx *c, int count, const int *nodes, double *d_chi, double *d_zee,
                                double *d_rho_pj, int *d_lanczos_iters) {
  if (!c || count < 0 || (count > 0 && (!nodes || !d_chi || !d_zee || !d_rho_pj))) return SQB_ERR_ARG;
  if (!c->have_veff || !c->have_atoms || !c->have_proj) return SQB_ERR_STATE;
  if (count == 0) return SQB_OK;
  for (int i = 0; i < count; i++)
    if (nodes[i] < 0 || nodes[i] >= c->nnode) return SQB_ERR_ARG;
  CK(cudaSetDevice(c->device));
  const size_t nw = (size_t)c->n * c->n * c->n;
  const size_t stride = ((4 * nw * sizeof(double)) + 255) & ~size_t(255);
  const size_t header = 256, list_bytes = ((size_t)count * sizeof(int) + 255) & ~size_t(255);
  if (header + list_bytes + stride > SQB_NOALLOC_SCRATCH_BYTES) {
    std::fprintf(stderr,
                 "sqdft_b200: sqb_lanczos_moments_noalloc needs %zu bytes of scratch for one CTA and %d nodes; "
                 "the fixed array holds %u\n",
                 header + list_bytes + stride, count, SQB_NOALLOC_SCRATCH_BYTES);
    return SQB_ERR_CAPACITY;
  }
  unsigned char *base = nullptr;
  int rc = noalloc_base(c->device, &base);
  if (rc) return rc;
  const int cols = choose_cols(c);
  if (node_kernel_threads(c->n, cols) > 1024) return SQB_ERR_UNSUPPORTED;
  int grid = c->sms * (c->ctas_per_sm > 0 ? c->ctas_per_sm : 1);
  const size_t fit = (SQB_NOALLOC_SCRATCH_BYTES - header - list_bytes) / stride;
  if ((size_t)grid > fit) grid = (int)fit;
  if (grid > count) grid = count;
  int *d_counter = reinterpret_cast<int *>(base);
  int *d_status = reinterpret_cast<int *>(base + 64);
  int *d_list = reinterpret_cast<int *>(base + header);
  NodeArgs a;
  fill_node_args(c, a);
  a.mode = MODE_SQ;
  a.chi = d_chi;
  a.zee = d_zee;
  a.rho_pj = d_rho_pj;
  a.lmin = nullptr;
  a.lmax = nullptr;
  a.lanczos_iters = d_lanczos_iters;
  a.counter = d_counter;
  a.status = d_status;
  a.proj_points = nullptr;
  a.scratch = base + header + list_bytes;
  a.scratch_stride = stride;
  a.node_list = d_list;
  a.n_list = count;
  // The outputs are the caller's device arrays: the work below runs on the
  // context's own (non-blocking) stream, so it first waits for everything the
  // caller queued on the legacy default stream (where torch and most callers
  // queue by default) before it writes them.
  CK(cudaEventRecord(c->ev_order, cudaStreamLegacy));
  CK(cudaStreamWaitEvent(c->stream, c->ev_order, 0));
  // The array keeps the previous call's contents: the counter and status
  // start at zero, the node list is written; window slots need no clearing.
  CK(cudaMemsetAsync(base, 0, header, c->stream));
  CK(cudaMemcpyAsync(d_list, nodes, (size_t)count * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(launch_node_kernel(a, grid, cols, c->stream));
  int st = 0;
  CK(cudaMemcpyAsync(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return status_to_err(st);
}

int sqb_get_stats(const sqb_ctx *c, sqb_stats *out, size_t out_size) {
  if (!c || !out || out_size == 0) return SQB_ERR_ARG;
  std::memcpy(out, &c->stats, out_size < sizeof(sqb_stats) ? out_size : sizeof(sqb_stats));
  return SQB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Pseudocharge density and local forces (sqb_local.cu)

namespace {

LocalArgs local_args(const sqb_ctx *c) {
  LocalArgs a{};
  for (int d = 0; d < 3; d++) {
    a.np[d] = c->g.np[d];
    a.pnode_s[d] = c->g.pnode_s[d];
  }
  a.delta = c->g.delta;
  a.h3 = c->h3;  // pow(delta, 3), as the reference forms it
  for (int k = 0; k <= FDN; k++) {
    a.coeff_lap[k] = c->g.coeff_lap[k];
    a.coeff_grad[k] = c->g.coeff_grad[k];
  }
  a.n_rep = c->loc_nrep;
  a.rep_type = c->d_loc_type;
  a.rep_atom = c->d_loc_atom;
  a.rep_xyz = c->d_loc_xyz;
  a.rep_box = c->d_loc_box;
  a.tab = c->d_loc_tab;
  a.typ_off = c->d_loc_off;
  a.typ_size = c->d_loc_size;
  a.Z = c->d_loc_Z;
  a.rc_tilda = c->loc_rc_tilda;
  a.status = c->d_status;
  return a;
}

// Block fields of the pseudocharge calls: b, b_tilda, Vc, rho_at (N each),
// phi with its FDN halo, and the per-CTA sums.
int ensure_local_fields(sqb_ctx *c, double **f, double **phi, double **partial) {
  const size_t N = (size_t)c->nnode;
  const size_t P = (size_t)(c->g.np[0] + 2 * FDN) * (c->g.np[1] + 2 * FDN) * (c->g.np[2] + 2 * FDN);
  const size_t parts = (size_t)5 * charge_density_ctas(c->g.np);
  const size_t need = (4 * N + P + parts) * sizeof(double);
  if (c->loc_fields_bytes < need) {
    if (c->d_loc_fields) cudaFree(c->d_loc_fields);
    c->d_loc_fields = nullptr;
    CK(cudaMalloc((void **)&c->d_loc_fields, need));
    c->loc_fields_bytes = need;
  }
  *f = c->d_loc_fields;
  *phi = c->d_loc_fields + 4 * N;
  *partial = *phi + P;
  return SQB_OK;
}

// Sum of a device array of n doubles in index order, on the host.
int host_sum(sqb_ctx *c, const double *d, size_t n, int stride_count, double *out) {
  std::vector<double> h(n * (size_t)stride_count);
  CK(cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < stride_count; k++) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += h[(size_t)k * n + i];
    out[k] = s;
  }
  return SQB_OK;
}

}  // namespace

extern "C" {

int sqb_set_local_atoms(sqb_ctx *c, int n_typ, const sqb_local_species *types, int n_rep, const int *rep_type,
                        const int *rep_atom, const double *rep_xyz, const int *rep_box, double rc_tilda, int n_atm) {
  if (!c || n_typ <= 0 || !types || n_rep < 0 || n_atm <= 0 || !(rc_tilda > 0)) return SQB_ERR_ARG;
  if (n_rep > 0 && (!rep_type || !rep_atom || !rep_xyz || !rep_box)) return SQB_ERR_ARG;
  if (c->g.fdn != FDN) return SQB_ERR_UNSUPPORTED;
  cudaSetDevice(c->device);
  std::vector<long long> off(n_typ);
  std::vector<int> size(n_typ);
  std::vector<double> Z(n_typ);
  long long total = 0;
  for (int t = 0; t < n_typ; t++) {
    if (types[t].size < 2 || !types[t].tables) return SQB_ERR_ARG;
    off[t] = total;
    size[t] = types[t].size;
    Z[t] = types[t].Z;
    total += 5LL * types[t].size;
  }
  for (int r = 0; r < n_rep; r++) {
    if (rep_type[r] < 0 || rep_type[r] >= n_typ || rep_atom[r] < 0 || rep_atom[r] >= n_atm) return SQB_ERR_ARG;
    for (int d = 0; d < 3; d++) {
      const int lo = rep_box[6 * r + 2 * d], hi = rep_box[6 * r + 2 * d + 1];
      if (lo > hi || lo < c->g.pnode_s[d] || hi >= c->g.pnode_s[d] + c->g.np[d]) return SQB_ERR_ARG;
    }
  }
  std::vector<double> tab((size_t)std::max<long long>(total, 1));
  for (int t = 0; t < n_typ; t++)
    std::memcpy(&tab[(size_t)off[t]], types[t].tables, sizeof(double) * 5 * (size_t)types[t].size);
  const size_t nr = (size_t)std::max(n_rep, 1);
  CK(dalloc(&c->d_loc_tab, tab.size()));
  CK(dalloc(&c->d_loc_off, (size_t)n_typ));
  CK(dalloc(&c->d_loc_size, (size_t)n_typ));
  CK(dalloc(&c->d_loc_Z, (size_t)n_typ));
  CK(dalloc(&c->d_loc_type, nr));
  CK(dalloc(&c->d_loc_atom, nr));
  CK(dalloc(&c->d_loc_xyz, 3 * nr));
  CK(dalloc(&c->d_loc_box, 6 * nr));
  CK(cudaMemcpy(c->d_loc_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_loc_off, off.data(), n_typ * sizeof(long long), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_loc_size, size.data(), n_typ * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_loc_Z, Z.data(), n_typ * sizeof(double), cudaMemcpyHostToDevice));
  if (n_rep > 0) {
    CK(cudaMemcpy(c->d_loc_type, rep_type, n_rep * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_loc_atom, rep_atom, n_rep * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_loc_xyz, rep_xyz, 3 * (size_t)n_rep * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_loc_box, rep_box, 6 * (size_t)n_rep * sizeof(int), cudaMemcpyHostToDevice));
  }
  c->h_loc_atom.assign(rep_atom, rep_atom + n_rep);
  c->h_loc_box.assign(rep_box, rep_box + 6 * (size_t)n_rep);
  c->loc_nrep = n_rep;
  c->loc_natm = n_atm;
  c->loc_rc_tilda = rc_tilda;
  c->have_local = true;
  return SQB_OK;
}

int sqb_charge_density(sqb_ctx *c, double *b, double *b_tilda, double *vc, double *rho_at, double *scal) {
  if (!c || !scal) return SQB_ERR_ARG;
  if (!c->have_local) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  NvtxRange nr("sqb_charge_density");
  const size_t N = (size_t)c->nnode;
  double *f = nullptr, *phi = nullptr, *partial = nullptr;
  int rc = ensure_local_fields(c, &f, &phi, &partial);
  if (rc) return rc;
  LocalArgs a = local_args(c);
  a.b = f;
  a.b_tilda = f + N;
  a.vc = f + 2 * N;
  a.rho_at = f + 3 * N;
  a.partial = partial;
  const int ncta = charge_density_ctas(c->g.np);
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaEventRecord(c->ev0, c->stream));
  CK(launch_charge_density(a, c->stream));
  int st = 0;
  CK(cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  // sums in CTA order: Eself, Ncharge, integral of rho_at, Ncharge_tilda, Eself_tilda
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  rc = host_sum(c, partial, (size_t)ncta, 5, v);
  if (rc) return rc;
  rc = status_to_err(st);
  if (rc) return rc;
  // V000 (rank 0's Vc[0][0][0]) and Vcon (Vt - V summed at the main
  // domain's first node over the replicas that hold it, initialize.cpp:631-635)
  // both come from the block that starts at the main domain's first node: the
  // unshifted Vc there is the same sum in the same order.  Other blocks add 0.
  const int *ps = c->g.pnode_s;
  if (ps[0] == 0 && ps[1] == 0 && ps[2] == 0) {
    double v0 = 0.0;
    CK(cudaMemcpyAsync(&v0, a.vc, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    v[5] = v0;
    v[6] = v0;
  }
  rc = reduce(c, v, 7, SQB_SUM);  // initialize.cpp:717-723 and the broadcasts of :741-742
  if (rc) return rc;
  const double scale = fabs(v[1] / v[3]), shift = -v[5] + v[6];
  CK(launch_charge_finish(a, scale, shift, c->stream));
  CK(cudaEventRecord(c->ev1, c->stream));
  double ecorr = 0.0;
  rc = host_sum(c, partial, (size_t)ncta, 1, &ecorr);
  if (rc) return rc;
  rc = reduce(c, &ecorr, 1, SQB_SUM);  // initialize.cpp:770
  if (rc) return rc;
  c->stats.ms_charge_density = elapsed(c);
  double *outs[4] = {b, b_tilda, vc, rho_at};
  for (int k = 0; k < 4; k++)
    if (outs[k]) CK(cudaMemcpyAsync(outs[k], f + k * N, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  scal[0] = v[0];
  scal[1] = v[1];
  scal[2] = v[2];
  scal[3] = v[3];
  scal[4] = v[4];
  scal[5] = v[6];
  scal[6] = ecorr + v[0] - v[4];  // Ecorr_global + Eself - Eself_tilda (initialize.cpp:775)
  return SQB_OK;
}

int sqb_forces_local(sqb_ctx *c, const double *phi, const double *vc, const double *b, const double *b_tilda,
                     double *floc, double *fcorr) {
  if (!c || !phi || !vc || !b || !b_tilda || !floc || !fcorr) return SQB_ERR_ARG;
  if (!c->have_local) return SQB_ERR_STATE;
  cudaSetDevice(c->device);
  NvtxRange nr("sqb_forces_local");
  const size_t N = (size_t)c->nnode;
  const size_t P = (size_t)(c->g.np[0] + 2 * FDN) * (c->g.np[1] + 2 * FDN) * (c->g.np[2] + 2 * FDN);
  double *f = nullptr, *d_phi = nullptr, *partial = nullptr;
  int rc = ensure_local_fields(c, &f, &d_phi, &partial);
  if (rc) return rc;
  CK(cudaMemcpyAsync(d_phi, phi, P * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(f, b, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(f + N, b_tilda, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(f + 2 * N, vc, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  LocalArgs a = local_args(c);
  a.phi = d_phi;
  a.bf = f;
  a.btf = f + N;
  a.vcf = f + 2 * N;
  // replicas in batches whose scratch boxes (4 fields each, box + 2 fdn
  // per side) fit 1 GiB
  const int n = c->loc_nrep;
  std::vector<long long> vol(n);
  for (int r = 0; r < n; r++) {
    const int *bx = &c->h_loc_box[6 * (size_t)r];
    vol[r] = (long long)(bx[1] - bx[0] + 1 + 4 * FDN) * (bx[3] - bx[2] + 1 + 4 * FDN) * (bx[5] - bx[4] + 1 + 4 * FDN);
  }
  const long long budget = (1LL << 30) / (long long)sizeof(double);
  std::vector<double> fsum((size_t)6 * c->loc_natm, 0.0);
  CK(dalloc(&c->d_loc_scr_off, (size_t)std::max(n, 1)));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaEventRecord(c->ev0, c->stream));
  for (int r0 = 0; r0 < n;) {
    int r1 = r0;
    long long used = 0;
    std::vector<long long> offs;
    while (r1 < n && (r1 == r0 || used + 4 * vol[r1] <= budget)) {
      offs.push_back(used);
      used += 4 * vol[r1];
      r1++;
    }
    const size_t nb = (size_t)(r1 - r0);
    const size_t need = (size_t)used * sizeof(double) + nb * LOC_FORCE_CTAS * 6 * sizeof(double);
    if (c->loc_scr_bytes < need) {
      if (c->d_loc_scr) cudaFree(c->d_loc_scr);
      c->d_loc_scr = nullptr;
      CK(cudaMalloc((void **)&c->d_loc_scr, need));
      c->loc_scr_bytes = need;
    }
    // the kernels index the scratch by replica: offsets of [r0, r1) at slots r0..
    CK(cudaMemcpyAsync(c->d_loc_scr_off + r0, offs.data(), nb * sizeof(long long), cudaMemcpyHostToDevice,
                       c->stream));
    a.scr = c->d_loc_scr;
    a.scr_off = c->d_loc_scr_off;
    a.fpart = c->d_loc_scr + used;
    CK(launch_forces_local(a, r0, r1, c->stream));
    std::vector<double> part(nb * LOC_FORCE_CTAS * 6);
    CK(cudaMemcpyAsync(part.data(), a.fpart, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < nb; i++) {
      double rs[6] = {0, 0, 0, 0, 0, 0};
      for (int k = 0; k < LOC_FORCE_CTAS; k++)
        for (int q = 0; q < 6; q++) rs[q] += part[(i * LOC_FORCE_CTAS + k) * 6 + q];
      const int atom = c->h_loc_atom[r0 + i];
      for (int q = 0; q < 6; q++) fsum[(size_t)6 * atom + q] += rs[q];
    }
    r0 = r1;
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  int st = 0;
  CK(cudaMemcpyAsync(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->stats.ms_forces_local = elapsed(c);
  rc = status_to_err(st);
  if (rc) return rc;
  for (int at = 0; at < c->loc_natm; at++)
    for (int d = 0; d < 3; d++) {
      floc[3 * at + d] = fsum[(size_t)6 * at + d];
      fcorr[3 * at + d] = fsum[(size_t)6 * at + 3 + d];
    }
  return SQB_OK;
}

}  // extern "C"
