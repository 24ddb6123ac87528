// Drop-in replacement of SQDFT's SQ entry points, calling the GPU library
// through its C ABI (include/sqdft_b200.h).
//
// Compiled against the reference headers and linked into the reference
// program in place of the three functions the SCF loop and the force routine
// call:
//   ClenshawCurtisSpectralQuadrature(DS_SQ*, int)  func_sq.h:515, sq.cpp:377
//   NonlocalProjectors(DS_SQ*)                     func_sq.h:368, nonlocal.cpp:317
//   ForcesNonLocal(DS_SQ*)                         func_sq.h:540, forces.cpp:318
// (the reference definitions are weakened in their objects, see Makefile),
// and, with SQDFT_B200_LOCAL=1, the per-atom loops of
//   ChargeDensity(DS_SQ*)                          func_sq.h:133, initialize.cpp:470
//   ForcesLocal(DS_SQ*)                            func_sq.h:534, forces.cpp:20
// (otherwise the reference's own, kept as ref_ChargeDensity / ref_ForcesLocal).
// It reads and writes the same DS_SQ fields as the functions it replaces.
// Failures print the reference's message and exit(1), as the reference does.
//
// Environment:
//   SQDFT_B200_PRECISION=fp32   FP32-mixed form (default FP64, the parity path)
//   SQDFT_B200_PRECISION=lq     FP64 Lanczos-quadrature form
//   SQDFT_B200_LANCZOS_TOL=T    Lanczos stop (Ha) of the two forms above
//                               (default: the input's lanczos_tol)
//   SQDFT_B200_DEVICE=k         CUDA device (default: MPI rank)
//   SQDFT_B200_LOCAL=1          pseudocharge density and local forces on the GPU
//   SQDFT_B200_EXPORT=path      at the first SQ call, write the SQ inputs and
//                               the pseudocharge inputs and fields as a case
//                               container (sqdft_b200/csrc/sq_case.h) and
//                               exit; no GPU is touched in this mode.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ds_sq.h"
#include "func_sq.h"
#include "sq_export.h"
#include "sqdft_b200.h"

namespace {

sqb_ctx *g_ctx = nullptr;

bool export_mode() { return std::getenv("SQDFT_B200_EXPORT") != nullptr; }

void fail(int rc, const char *where) {
  int rank = 0;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  std::printf("Rank=%d, Error: %s (%s, status %d)\n", rank, sqb_status_string(rc), where, rc);
  std::exit(1);
}

int mpi_reduce(double *v, int count, int op, void *) {
  MPI_Op o = op == SQB_SUM ? MPI_SUM : op == SQB_MIN ? MPI_MIN : MPI_MAX;
  return MPI_Allreduce(MPI_IN_PLACE, v, count, MPI_DOUBLE, o, MPI_COMM_WORLD) == MPI_SUCCESS ? 0 : 1;
}

sqb_ctx *g_lctx = nullptr;  // the pseudocharge calls' context (SQDFT_B200_LOCAL=1)

void destroy_ctx() {
  if (g_ctx) sqb_destroy(g_ctx);
  g_ctx = nullptr;
  if (g_lctx) sqb_destroy(g_lctx);
  g_lctx = nullptr;
}

// The block grid of DS_SQ (ds_sq.h:133-161) in the C-ABI layout.
sqb_grid grid_of(DS_SQ *p) {
  sqb_grid g;
  std::memset(&g, 0, sizeof(g));
  g.np[0] = p->np_x;
  g.np[1] = p->np_y;
  g.np[2] = p->np_z;
  for (int d = 0; d < 3; d++) {
    g.pnode_s[d] = p->pnode_s[d];
    g.n_int[d] = p->n_int[d];
  }
  g.nloc = p->nloc;
  g.fdn = p->FDn;
  g.npl = p->npl;
  g.fermi_alg = p->fermi_alg;
  g.delta = p->delta;
  g.bet = p->bet;
  g.lanczos_tol = p->lanczos_tol;
  g.fermi_tol = p->fermi_tol;
  g.ncharge = p->Ncharge;
  for (int k = 0; k <= p->FDn && k < 8; k++) {
    g.coeff_lap[k] = p->coeff_lap[k];
    g.coeff_grad[k] = p->coeff_grad[k];
  }
  return g;
}

int device_of() {
  int rank = 0;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  const char *dev_env = std::getenv("SQDFT_B200_DEVICE");
  return dev_env ? std::atoi(dev_env) : rank;
}

// The SQ context: created at the first SQ call, when DS_SQ::Ncharge (the
// electron count the Fermi level is solved for) is set.
void ensure_ctx(DS_SQ *p) {
  if (g_ctx) return;
  const sqb_grid g = grid_of(p);
  int rc = sqb_create(&g, device_of(), &g_ctx);
  if (rc) fail(rc, "sqb_create");
  const char *prec = std::getenv("SQDFT_B200_PRECISION");
  if (prec && (!std::strcmp(prec, "fp32") || !std::strcmp(prec, "mixed"))) sqb_set_precision(g_ctx, SQB_FP32_MIXED);
  if (prec && !std::strcmp(prec, "lq")) sqb_set_precision(g_ctx, SQB_FP64_LANCZOS_QUAD);
  if (const char *tol = std::getenv("SQDFT_B200_LANCZOS_TOL")) {
    rc = sqb_set_mixed_lanczos(g_ctx, std::atof(tol), 0.5);
    if (rc) fail(rc, "sqb_set_mixed_lanczos");
  }
  if (p->nproc > 1) sqb_set_allreduce(g_ctx, mpi_reduce, nullptr);
  // SQDFT_B200_GRAPH=2: every SCF iteration's SQ step replays one CUDA graph
  // (node kernel, device-side Fermi solve, density); 1: the node kernel only
  if (const char *gr = std::getenv("SQDFT_B200_GRAPH")) {
    rc = sqb_set_graph(g_ctx, std::atoi(gr));
    if (rc) fail(rc, "sqb_set_graph");
  }
  std::atexit(destroy_ctx);
}

// Replica atoms and radial tables of DS_SQ in the C-ABI layout.
void upload_atoms(DS_SQ *p) {
  std::vector<sqb_species> types(p->n_typ);
  std::vector<std::vector<double>> tabs(p->n_typ);
  std::vector<int> rt, ra;
  std::vector<double> rx;
  int atom_count = 0;
  for (int t = 0; t < p->n_typ; t++) {
    const DS_Psd &ps = p->Psd[t];
    sqb_species &s = types[t];
    s.natm = p->Atm[t].natm;
    s.lmax = ps.lmax;
    s.lloc = p->Atm[t].lloc;
    s.nlocc = (int)ceil(ps.rc / p->delta);  // nonlocal.cpp:43
    s.size = ps.size;
    s.rc = ps.rc;
    s.denom[0] = ps.Denom_s;
    s.denom[1] = ps.Denom_p;
    s.denom[2] = ps.Denom_d;
    s.denom[3] = ps.Denom_f;
    const double *rows[19] = {ps.RadialGrid, ps.rVloc, ps.rVs, ps.rVp, ps.rVd, ps.rVf, ps.rUs,
                              ps.rUp, ps.rUd, ps.rUf, ps.DVloc, ps.DVsJ, ps.DVpJ, ps.DVdJ,
                              ps.DVfJ, ps.DUsJ, ps.DUpJ, ps.DUdJ, ps.DUfJ};
    tabs[t].assign((size_t)19 * ps.size, 0.0);
    for (int q = 0; q < 19; q++)
      if (rows[q]) std::memcpy(&tabs[t][(size_t)q * ps.size], rows[q], sizeof(double) * ps.size);
    s.tables = tabs[t].data();
    for (int a = 0; a < p->Atm[t].natm; a++, atom_count++)
      for (int r = 0; r < p->Atm[t].Rx[a].n_replica_Rcut; r++) {
        rt.push_back(t);
        ra.push_back(atom_count);
        rx.push_back(p->Atm[t].Rx[a].ProcAtmRcut[r].coord);
        rx.push_back(p->Atm[t].Ry[a].ProcAtmRcut[r].coord);
        rx.push_back(p->Atm[t].Rz[a].ProcAtmRcut[r].coord);
      }
  }
  int rc = sqb_set_atoms(g_ctx, p->n_typ, types.data(), (int)rt.size(), rt.data(), ra.data(), rx.data(), p->n_atm);
  if (rc) fail(rc, "sqb_set_atoms");
}

// Veff halo of width nloc from the neighbouring processor blocks, with the
// communication indices SQ_Comm_Indices (sq.cpp:20-49) prepared: the exchange
// of sq.cpp:386-492 (pack edge regions, neighbourhood all-to-all, unpack).
void fill_veff_halo(DS_SQ *p) {
  const int nl = p->nloc;
  const int np_edge = (2 * nl + p->np_x) * (2 * nl + p->np_x) * (2 * nl + p->np_x) - p->np_x * p->np_x * p->np_x;
  std::vector<double> out((size_t)np_edge), in((size_t)np_edge);
  const int nnproc = (int)ceil((double)(nl - 1e-12) / p->np_x);
  int neigh = 0;
  size_t cnt = 0;
  for (int kk = -nnproc; kk <= nnproc; kk++)
    for (int jj = -nnproc; jj <= nnproc; jj++)
      for (int ii = -nnproc; ii <= nnproc; ii++, neigh++) {
        if (!ii && !jj && !kk) continue;
        for (int k = p->SqInd.eout_s[2][neigh]; k <= p->SqInd.eout_e[2][neigh]; k++)
          for (int j = p->SqInd.eout_s[1][neigh]; j <= p->SqInd.eout_e[1][neigh]; j++)
            for (int i = p->SqInd.eout_s[0][neigh]; i <= p->SqInd.eout_e[0][neigh]; i++)
              out[cnt++] = p->Veff[k + nl][j + nl][i + nl];
      }
  MPI_Neighbor_alltoallv(out.data(), p->SqInd.ncounts_send, p->SqInd.displs_send, MPI_DOUBLE, in.data(),
                         p->SqInd.ncounts_recv, p->SqInd.displs_recv, MPI_DOUBLE, p->comm_sq);
  neigh = 0;
  cnt = 0;
  for (int kk = -nnproc; kk <= nnproc; kk++)
    for (int jj = -nnproc; jj <= nnproc; jj++)
      for (int ii = -nnproc; ii <= nnproc; ii++, neigh++) {
        if (!ii && !jj && !kk) continue;
        for (int k = p->SqInd.ein_s[2][neigh]; k <= p->SqInd.ein_e[2][neigh]; k++)
          for (int j = p->SqInd.ein_s[1][neigh]; j <= p->SqInd.ein_e[1][neigh]; j++)
            for (int i = p->SqInd.ein_s[0][neigh]; i <= p->SqInd.ein_e[0][neigh]; i++)
              p->Veff[k][j][i] = in[cnt++];
      }
}

}  // namespace

void NonlocalProjectors(DS_SQ *p) {
  if (export_mode()) return;  // the exporter stores the radial tables instead
  ensure_ctx(p);
  upload_atoms(p);
  long long total = 0;
  for (int t = 0; t < p->n_typ; t++) {
    const long long S = 2LL * (int)ceil(p->Psd[t].rc / p->delta) + 1;
    for (int a = 0; a < p->Atm[t].natm; a++)
      total += (long long)p->Atm[t].Rx[a].n_replica_Rcut * sqb::proj_count(p, t) * S * S * S;
  }
  std::vector<double> all((size_t)(total > 0 ? total : 1));
  int rc = sqb_nonlocal_projectors(g_ctx, all.data());
  if (rc) fail(rc, "NonlocalProjectors");
  // Host copies of UdVtm, allocated as the reference allocates them
  // (Deallocate_memory frees them).
  size_t off = 0;
  for (int t = 0; t < p->n_typ; t++) {
    const int S = 2 * (int)ceil(p->Psd[t].rc / p->delta) + 1, nnd = S * S * S, np = sqb::proj_count(p, t);
    for (int a = 0; a < p->Atm[t].natm; a++)
      for (int r = 0; r < p->Atm[t].Rx[a].n_replica_Rcut; r++) {
        double **u = new double *[np]();
        for (int c = 0; c < np; c++) {
          u[c] = new double[nnd];
          std::memcpy(u[c], &all[off], sizeof(double) * nnd);
          off += nnd;
        }
        p->Atm[t].Rx[a].ProcAtmRcut[r].UdVtm = u;
      }
  }
}

void ClenshawCurtisSpectralQuadrature(DS_SQ *p, int scf_iter) {
  int rank = 0;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  const double t0 = MPI_Wtime();
  p->mpi_time = 0.0;
  fill_veff_halo(p);
  if (export_mode()) {
    sqb::export_case(p, std::getenv("SQDFT_B200_EXPORT"), scf_iter, false, true);
    if (rank == 0) std::printf("sqdft_b200: SQ inputs written to %s\n", std::getenv("SQDFT_B200_EXPORT"));
    std::exit(0);
  }
  ensure_ctx(p);
  const int nl = p->nloc, ex = p->np_x + 2 * nl, ey = p->np_y + 2 * nl, ez = p->np_z + 2 * nl;
  std::vector<double> veff((size_t)ex * ey * ez);
  for (int k = 0; k < ez; k++)
    for (int j = 0; j < ey; j++) std::memcpy(&veff[((size_t)k * ey + j) * ex], p->Veff[k][j], sizeof(double) * ex);
  int rc = sqb_set_veff(g_ctx, veff.data());
  if (rc) fail(rc, "Veff");
  const int N = p->np_x * p->np_y * p->np_z, K = p->npl + 1;
  std::vector<double> rho(N), rpj((size_t)N * K), ci((size_t)N * K);
  double lam = p->lambda_f, ebs = 0.0, eent = 0.0;
  rc = sqb_spectral_quadrature(g_ctx, scf_iter, &lam, rho.data(), rpj.data(), ci.data(), p->chi, p->zee, &ebs, &eent);
  if (rc) fail(rc, "ClenshawCurtisSpectralQuadrature");
  for (int k = 0; k < p->np_z; k++)
    for (int j = 0; j < p->np_y; j++)
      std::memcpy(p->rho[k][j], &rho[((size_t)k * p->np_y + j) * p->np_x], sizeof(double) * p->np_x);
  for (int nd = 0; nd < N; nd++) {
    std::memcpy(p->rho_pj[nd], &rpj[(size_t)nd * K], sizeof(double) * K);
    std::memcpy(p->Ci[nd], &ci[(size_t)nd * K], sizeof(double) * K);
  }
  p->lambda_f = lam;
  p->Ebs = ebs;
  p->Eent = eent;
  sqb_stats st;
  sqb_get_stats(g_ctx, &st, sizeof(st));
  if (st.lanczos_maxiter_nodes > 0)  // sq.cpp:1073-1074: reported, the run goes on
    std::printf("Error: Lanczos exceeded max_iter. count=%d on %lld nodes of rank %d \n", st.max_lanczos_iters,
                st.lanczos_maxiter_nodes, rank);
  if (rank == 0) {
    std::printf("Lanczos took %d iterations (max over nodes, GPU). \n", st.max_lanczos_iters);
    std::printf("Brent's algorithm took %d iterations. \n", st.fermi_iters);
    std::printf("Time stats (sec): GPU Lanczos+Cheb_Comps = %.3f, Fermi_energy calc = %.3f, Rho_Ebs_Eent = %.3f \n",
                st.ms_lanczos_moments * 1e-3, st.ms_fermi * 1e-3, st.ms_density * 1e-3);
  }
  p->sq_time += MPI_Wtime() - t0;
}

void ForcesNonLocal(DS_SQ *p) {
  ensure_ctx(p);
  const int N = p->np_x * p->np_y * p->np_z, K = p->npl + 1;
  std::vector<double> ci((size_t)N * K), f((size_t)3 * p->n_atm);
  for (int nd = 0; nd < N; nd++) std::memcpy(&ci[(size_t)nd * K], p->Ci[nd], sizeof(double) * K);
  int rc = sqb_forces_nonlocal(g_ctx, p->chi, p->zee, ci.data(), f.data());
  if (rc) fail(rc, "ForcesNonLocal");
  for (int a = 0; a < p->n_atm; a++) {
    p->fnlocx[a] = f[3 * a];
    p->fnlocy[a] = f[3 * a + 1];
    p->fnlocz[a] = f[3 * a + 2];
  }
}

// ---------------------------------------------------------------------------
// ChargeDensity and ForcesLocal.  By default the reference's own functions
// run (kept in the program under the names ref_ChargeDensity and
// ref_ForcesLocal, see Makefile); with SQDFT_B200_LOCAL=1 their per-atom
// loops run on the GPU (sqb_charge_density, sqb_forces_local) and the rest
// of ChargeDensity -- the initial density guess, its scaling to the nuclear
// charge, the Poisson right-hand side -- follows here on the host as
// initialize.cpp:637-784 does.  Export mode always runs the reference path.

void ref_ChargeDensity(DS_SQ *p);  // initialize.cpp:470 (renamed)
void ref_ForcesLocal(DS_SQ *p);    // forces.cpp:20 (renamed)

namespace {

bool local_on_device() {
  const char *v = std::getenv("SQDFT_B200_LOCAL");
  return v && !std::strcmp(v, "1") && !export_mode();
}

// The pseudocharge calls run on a context of their own: ChargeDensity comes
// before the SQ context can be made (it sets the electron count).
void ensure_local_ctx(DS_SQ *p) {
  if (g_lctx) return;
  const sqb_grid g = grid_of(p);
  int rc = sqb_create(&g, device_of(), &g_lctx);
  if (rc) fail(rc, "sqb_create");
  if (p->nproc > 1) sqb_set_allreduce(g_lctx, mpi_reduce, nullptr);
  std::atexit(destroy_ctx);
}

void upload_local_atoms(DS_SQ *p) {
  ensure_local_ctx(p);
  const sqb::LocalInputs L = sqb::gather_local(p);
  std::vector<sqb_local_species> sp(p->n_typ);
  for (int t = 0; t < p->n_typ; t++) {
    sp[t].size = (int)(L.tables[t].size() / 5);
    sp[t].Z = L.Z[t];
    sp[t].tables = L.tables[t].data();
  }
  const int rc = sqb_set_local_atoms(g_lctx, p->n_typ, sp.data(), (int)L.rep_type.size(), L.rep_type.data(),
                                     L.rep_atom.data(), L.rep_xyz.data(), L.rep_box.data(), p->rc_tilda, p->n_atm);
  if (rc) fail(rc, "local atoms");
}

void put_block(double ***a, const std::vector<double> &v, int nz, int ny, int nx) {
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++) std::memcpy(a[k][j], &v[((size_t)k * ny + j) * nx], sizeof(double) * nx);
}

}  // namespace

void ChargeDensity(DS_SQ *p) {
  if (!local_on_device()) {
    ref_ChargeDensity(p);
    return;
  }
  int rank = 0;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  p->rc_tilda = 0.5;  // initialize.cpp:483
  upload_local_atoms(p);
  const int nz = p->np_z, ny = p->np_y, nx = p->np_x;
  const size_t N = (size_t)nz * ny * nx;
  std::vector<double> b(N), bt(N), vc(N), ra(N);
  double scal[7];
  int rc = sqb_charge_density(g_lctx, b.data(), bt.data(), vc.data(), ra.data(), scal);
  if (rc) fail(rc, "ChargeDensity");
  // b, the scaled b_tilda and the shifted Vc replace the block's; rho_at
  // accumulates as the reference's loop adds into it (initialize.cpp:585)
  put_block(p->b, b, nz, ny, nx);
  put_block(p->b_tilda, bt, nz, ny, nx);
  put_block(p->Vc, vc, nz, ny, nx);
  size_t q = 0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) p->rho_at[k][j][i] += ra[q++];
  p->Eself = scal[0];
  p->Ncharge = scal[1];
  // the density guess: rho_at on the first MD step, a restart file, or the
  // extrapolated density from the fourth MD step on (initialize.cpp:637-694)
  if (p->MDstepCount == 1)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++) std::memcpy(p->rho[k][j], p->rho_at[k][j], sizeof(double) * nx);
  if (p->restart_scf == 1) RestartSCF(p);
  if (p->MDstepCount > 3 && p->ChgExtrap == 1) {
    if (rank == 0) std::printf("Using Charge extrapolation for rho_guess! \n");
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          p->rho[k][j][i] = p->rho_at[k][j][i] + p->drho_new[k][j][i];
          if (p->rho[k][j][i] < 0.0) p->rho[k][j][i] = pow(10.0, -6.0);
        }
  }
  double nel = 0.0;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) nel += p->rho[k][j][i] * p->delta * p->delta * p->delta;
  MPI_Allreduce(MPI_IN_PLACE, &nel, 1, MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD);
  // scale rho to the nuclear charge (initialize.cpp:728-739)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) p->rho[k][j][i] = fabs(p->Ncharge / nel) * p->rho[k][j][i];
  p->Nelectron = -p->Ncharge;
  // Poisson right-hand side and the first MD step's phi guess
  // (initialize.cpp:755-767; the whole block)
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        if (p->MDstepCount == 1) p->phi_guess[k + p->FDn][j + p->FDn][i + p->FDn] = 1;
        p->rhs[k][j][i] = p->b[k][j][i] + p->rho[k][j][i];
      }
  p->Ecorr = scal[6];
  if (p->Correction == 1 && rank == 0) std::printf("Energy Correction (Ha/atom) : %.14f \n", p->Ecorr / p->n_atm);
}

void ForcesLocal(DS_SQ *p) {
  if (!local_on_device()) {
    ref_ForcesLocal(p);
    return;
  }
  upload_local_atoms(p);
  const int nz = p->np_z, ny = p->np_y, nx = p->np_x;
  const std::vector<double> phi = sqb::block_field(p->phi, nz, ny, nx, p->FDn);
  const std::vector<double> vc = sqb::block_field(p->Vc, nz, ny, nx, 0), b = sqb::block_field(p->b, nz, ny, nx, 0),
                            bt = sqb::block_field(p->b_tilda, nz, ny, nx, 0);
  std::vector<double> fl((size_t)3 * p->n_atm), fc((size_t)3 * p->n_atm);
  const int rc = sqb_forces_local(g_lctx, phi.data(), vc.data(), b.data(), bt.data(), fl.data(), fc.data());
  if (rc) fail(rc, "ForcesLocal");
  for (int a = 0; a < p->n_atm; a++) {
    p->flocx[a] = fl[3 * a];
    p->flocy[a] = fl[3 * a + 1];
    p->flocz[a] = fl[3 * a + 2];
    p->fcorrx[a] = fc[3 * a];
    p->fcorry[a] = fc[3 * a + 1];
    p->fcorrz[a] = fc[3 * a + 2];
  }
}
