// Oracle driver around the reference SQDFT objects (test infrastructure).
//
// Runs the reference's own set-up for an input stem exactly as main.cpp:30-106
// and SQDFT_forces (scf.cpp:341-372) do up to the first SQ call, then calls
// the reference's ClenshawCurtisSpectralQuadrature (sq.cpp:377),
// HsubTimesVec (sq.cpp:838) and ForcesNonLocal (forces.cpp:318), and writes
// their inputs and outputs as case containers (sqdft_b200/csrc/sq_case.h).
//
// usage: sqref_driver <run_dir> <stem> <out_prefix> [options]
//   --veff FILE      replace the Veff block interior (np_z*np_y*np_x float64,
//                    z-major) before the SQ call
//   --scf-iter K     scf_iter passed to the SQ call (default 1)
//   --lambda-f X     warm-start Fermi level used when K > 1
//   --no-forces      skip ForcesNonLocal
//   --hv K           also apply HsubTimesVec to K seeded vectors at K nodes
//   --nodes-only     stop after the SQ set-up (export the inputs only)
//   --local          also write <out_prefix>_local.sqc: the pseudocharge
//                    replicas and radial tables, ChargeDensity's outputs
//                    (initialize.cpp:470-784) as the call leaves them, and
//                    ForcesLocal (forces.cpp:20-315) with the fields it read,
//                    with the time of both calls (with --nodes-only: before
//                    the SQ step, on the set-up's phi)
//   --sample K       CPU baseline: time the reference's per-node work
//                    (LanczosAlgorithm, sq.cpp:965, and the moment loop of
//                    sq.cpp:564-655 over HsubTimesVec) on K nodes spread over
//                    the block, on --threads T host threads; writes the
//                    sampled chi, zee, rho_pj, the Veff block and the wall time
// Writes <out_prefix>_in.sqc (inputs, incl. the reference's UdVtm tables) and
// <out_prefix>_out.sqc (outputs and timings).
#include <unistd.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ds_sq.h"
#include "func_sq.h"
#include "../sqdft_b200/dropin/sq_export.h"

// double*** window array as the reference allocates them (sq.cpp:496-517).
static double ***new3(int n) {
  double ***a = new double **[n];
  for (int k = 0; k < n; k++) {
    a[k] = new double *[n];
    for (int j = 0; j < n; j++) a[k][j] = new double[n]();
  }
  return a;
}
static void del3(double ***a, int n) {
  for (int k = 0; k < n; k++) {
    for (int j = 0; j < n; j++) delete[] a[k][j];
    delete[] a[k];
  }
  delete[] a;
}

// Per-node work of ClenshawCurtisSpectralQuadrature for one node with the
// reference's own LanczosAlgorithm and HsubTimesVec; the moment loop restates
// sq.cpp:566-655 with the same expressions.
static void sample_node(DS_SQ *p, int nd, double *chi, double *zee, double *rpj) {
  const int nl = p->nloc, n = 2 * nl + 1;
  const int i = nd % p->np_x + nl, j = (nd / p->np_x) % p->np_y + nl, k = nd / (p->np_x * p->np_y) + nl;
  double ***vec = new3(n), ***hv = new3(n), ***t0 = new3(n), ***t1 = new3(n), ***t2 = new3(n);
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++)
      for (int c = 0; c < n; c++) vec[a][b][c] = 1.0;
  double lmin, lmax;
  LanczosAlgorithm(p, vec, i, j, k, &lmin, &lmax, nd + 1);
  const double ch = (lmax + lmin) / 2, ze = (lmax - lmin) / 2;
  *chi = ch;
  *zee = ze;
  const double h3 = pow(p->delta, 3);
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++)
      for (int c = 0; c < n; c++) t0[a][b][c] = (a == nl && b == nl && c == nl) ? 1.0 : 0.0;
  HsubTimesVec(p, t0, i, j, k, hv);
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++)
      for (int c = 0; c < n; c++) t1[a][b][c] = (hv[a][b][c] - ch * t0[a][b][c]) / ze;
  const double htemp = t1[nl][nl][nl];
  const int q1 = (int)round(0.25 * p->npl), q2 = (int)round(0.5 * p->npl);
  rpj[0] = t0[nl][nl][nl] / h3;
  rpj[1] = t1[nl][nl][nl] / h3;
  for (int nq = 2; nq <= q2; nq++) {
    double d1 = 0.0, d2 = 0.0;
    HsubTimesVec(p, t1, i, j, k, hv);
    for (int a = 0; a < n; a++)
      for (int b = 0; b < n; b++)
        for (int c = 0; c < n; c++) {
          t2[a][b][c] = (2 * (hv[a][b][c] - ch * t1[a][b][c]) / ze) - t0[a][b][c];
          d1 += t2[a][b][c] * t2[a][b][c];
          d2 += t2[a][b][c] * t1[a][b][c];
          t0[a][b][c] = t1[a][b][c];
          t1[a][b][c] = t2[a][b][c];
        }
    rpj[nq] = t2[nl][nl][nl] / h3;
    if (nq > q1) {
      rpj[2 * nq] = (2 * d1 - 1) / h3;
      rpj[2 * nq - 1] = (2 * d2 - htemp) / h3;
    }
  }
  del3(vec, n);
  del3(hv, n);
  del3(t0, n);
  del3(t1, n);
  del3(t2, n);
}

static unsigned long long lcg_state = 0x9E3779B97F4A7C15ull;
static double lcg_uniform() {  // deterministic [-1, 1) values for the HsubTimesVec fixture
  lcg_state = lcg_state * 6364136223846793005ull + 1442695040888963407ull;
  return ((double)(lcg_state >> 11) / 9007199254740992.0) * 2.0 - 1.0;
}

int main(int argc, char **argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s run_dir stem out_prefix [options]\n", argv[0]);
    return 2;
  }
  std::string run_dir = argv[1], stem = argv[2], out = argv[3];
  std::string veff_file;
  int scf_iter = 1, hv_count = 0, do_forces = 1, nodes_only = 0, sample = 0, threads = 1, do_local = 0;
  double lambda_warm = 0.0;
  int have_lambda = 0;
  for (int a = 4; a < argc; a++) {
    if (!std::strcmp(argv[a], "--veff") && a + 1 < argc) veff_file = argv[++a];
    else if (!std::strcmp(argv[a], "--scf-iter") && a + 1 < argc) scf_iter = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--lambda-f") && a + 1 < argc) { lambda_warm = std::atof(argv[++a]); have_lambda = 1; }
    else if (!std::strcmp(argv[a], "--no-forces")) do_forces = 0;
    else if (!std::strcmp(argv[a], "--hv") && a + 1 < argc) hv_count = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--nodes-only")) nodes_only = 1;
    else if (!std::strcmp(argv[a], "--local")) do_local = 1;
    else if (!std::strcmp(argv[a], "--sample") && a + 1 < argc) sample = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--threads") && a + 1 < argc) threads = std::atoi(argv[++a]);
    else { std::fprintf(stderr, "unknown option %s\n", argv[a]); return 2; }
  }
  // Output paths are made absolute before changing into the run directory.
  if (out[0] != '/') {
    char cwd[4096];
    if (getcwd(cwd, sizeof(cwd))) out = std::string(cwd) + "/" + out;
  }
  if (chdir(run_dir.c_str()) != 0) { std::perror("chdir"); return 2; }

  DS_SQ SQ = {};
  MPI_Init(&argc, &argv);
  SQ.nproc = 1;
  // CheckInputs reads the stem from the bytes after "-name" (readfiles.cpp:72-80).
  std::string argblob = std::string("-name") + '\0' + stem + '\0';
  std::vector<char> blob(argblob.begin(), argblob.end());
  char *fake_argv[3] = {argv[0], blob.data(), blob.data() + 6};
  CheckInputs(&SQ, fake_argv);
  SQ.mpi_time = 0.0;
  Read_input(&SQ);
  Read_atoms(&SQ);
  Read_psd(&SQ);
  Processor_domain(&SQ);
  AllocateArrays(&SQ);
  Comm_topologies(&SQ);
  Laplacian_Comm_Indices(&SQ);
  SQ_Comm_Indices(&SQ);
  SQ.MDstepCount = 1;

  Replica_atoms(&SQ);
  // ChargeDensity accumulates rho_at; the allocation zeroed it
  double t0 = MPI_Wtime();
  ChargeDensity(&SQ);
  const double t_cd = MPI_Wtime() - t0;
  std::vector<double> cd_b, cd_bt, cd_vc, cd_rho_at;
  if (do_local) {
    cd_b = sqb::block_field(SQ.b, SQ.np_z, SQ.np_y, SQ.np_x, 0);
    cd_bt = sqb::block_field(SQ.b_tilda, SQ.np_z, SQ.np_y, SQ.np_x, 0);
    cd_vc = sqb::block_field(SQ.Vc, SQ.np_z, SQ.np_y, SQ.np_x, 0);
    cd_rho_at = sqb::block_field(SQ.rho_at, SQ.np_z, SQ.np_y, SQ.np_x, 0);
  }
  if (SQ.Correction == 2) OverlapCorrection(&SQ);
  Replica_atoms_Rcut(&SQ);
  t0 = MPI_Wtime();
  NonlocalProjectors(&SQ);
  double t_proj = MPI_Wtime() - t0;
  PoissonSolver_AAJ(&SQ);
  ExchangeCorrelationPotential(&SQ);
  EvaluateEffectivePotential(&SQ);

  const int nl = SQ.nloc, nx = SQ.np_x, ny = SQ.np_y, nz = SQ.np_z;
  const int nnode = nx * ny * nz;
  if (!veff_file.empty()) {
    std::vector<double> vb((size_t)nnode);
    FILE *f = std::fopen(veff_file.c_str(), "rb");
    if (!f || std::fread(vb.data(), sizeof(double), vb.size(), f) != vb.size()) {
      std::fprintf(stderr, "cannot read %s\n", veff_file.c_str());
      return 2;
    }
    std::fclose(f);
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) SQ.Veff[k + nl][j + nl][i + nl] = vb[((size_t)k * ny + j) * nx + i];
  }
  if (have_lambda) SQ.lambda_f = lambda_warm;
  const double lambda_in = SQ.lambda_f;

  if (sample > 0) {
    // Single rank: the Rcut halo of Veff is the periodic wrap of the block
    // (what the exchange of sq.cpp:400-492 produces with one process).
    const int ex = nx + 2 * nl, ey = ny + 2 * nl, ez = nz + 2 * nl;
    for (int k = 0; k < ez; k++)
      for (int j = 0; j < ey; j++)
        for (int i = 0; i < ex; i++) {
          const int kk = ((k - nl) % nz + nz) % nz, jj = ((j - nl) % ny + ny) % ny, ii = ((i - nl) % nx + nx) % nx;
          SQ.Veff[k][j][i] = SQ.Veff[kk + nl][jj + nl][ii + nl];
        }
    if (sample > nnode) sample = nnode;
    std::vector<int> nodes(sample);
    for (int q = 0; q < sample; q++) nodes[q] = (int)(((long long)q * nnode) / sample + (nnode / sample) / 2) % nnode;
    std::vector<double> chi(sample), zee(sample), rpj((size_t)sample * (SQ.npl + 1));
    std::atomic<int> next(0);
    auto t_start = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < (threads > 0 ? threads : 1); t++)
      pool.emplace_back([&]() {
        for (int q; (q = next++) < sample;) sample_node(&SQ, nodes[q], &chi[q], &zee[q], &rpj[(size_t)q * (SQ.npl + 1)]);
      });
    for (auto &th : pool) th.join();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    sqb::CaseWriter w(out + "_sample.sqc");
    w.i32("sample_nodes", nodes.data(), {sample});
    w.f64("sample_chi", chi.data(), {sample});
    w.f64("sample_zee", zee.data(), {sample});
    w.f64("sample_rho_pj", rpj.data(), {sample, SQ.npl + 1});
    std::vector<double> vb((size_t)nnode);  // the Veff block the sample ran on
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) vb[((size_t)k * ny + j) * nx + i] = SQ.Veff[k + nl][j + nl][i + nl];
    w.f64("veff_block", vb.data(), {nz, ny, nx});
    w.f64s("t_sample", secs);
    w.i32s("threads", threads);
    w.close();
    std::printf("sqref_driver: %d nodes in %.3f s on %d threads\n", sample, secs, threads);
    return 0;
  }

  // --local: the pseudocharge inputs, ChargeDensity's outputs as the call
  // left them, and ForcesLocal with the fields it reads (phi, Vc, b, b_tilda)
  auto write_local = [&]() {
    sqb::CaseWriter wl(out + "_local.sqc");
    // the pseudocharge inputs and the fields ForcesLocal reads (phi, Vc, b, b_tilda)
    sqb::export_local(&SQ, wl);
    const int nz = SQ.np_z, ny = SQ.np_y, nx = SQ.np_x;
    wl.f64("cd_b", cd_b.data(), {nz, ny, nx});
    wl.f64("cd_b_tilda", cd_bt.data(), {nz, ny, nx});
    wl.f64("cd_vc", cd_vc.data(), {nz, ny, nx});
    wl.f64("cd_rho_at", cd_rho_at.data(), {nz, ny, nx});
    wl.f64s("cd_Eself", SQ.Eself);
    wl.f64s("cd_Ncharge", SQ.Ncharge);
    wl.f64s("cd_Ecorr", SQ.Ecorr);
    wl.f64s("t_charge_density", t_cd);
    t0 = MPI_Wtime();
    ForcesLocal(&SQ);
    const double t_fl = MPI_Wtime() - t0;
    std::vector<double> fl((size_t)SQ.n_atm * 3), fc((size_t)SQ.n_atm * 3);
    for (int a = 0; a < SQ.n_atm; a++) {
      fl[3 * a] = SQ.flocx[a];
      fl[3 * a + 1] = SQ.flocy[a];
      fl[3 * a + 2] = SQ.flocz[a];
      fc[3 * a] = SQ.fcorrx[a];
      fc[3 * a + 1] = SQ.fcorry[a];
      fc[3 * a + 2] = SQ.fcorrz[a];
    }
    wl.f64("fl_floc", fl.data(), {SQ.n_atm, 3});
    wl.f64("fl_fcorr", fc.data(), {SQ.n_atm, 3});
    wl.f64s("t_forces_local", t_fl);
    wl.close();
  };

  if (nodes_only) {
    // Only the block interior is valid here; the SQ call fills the halo.
    sqb::export_case(&SQ, (out + "_in.sqc").c_str(), scf_iter, true);
    if (do_local) write_local();  // phi is the set-up's Poisson solution; no SQ step needed
    return 0;
  }

  t0 = MPI_Wtime();
  ClenshawCurtisSpectralQuadrature(&SQ, scf_iter);
  const double t_sq = MPI_Wtime() - t0;
  const double lambda_out = SQ.lambda_f;

  // Inputs: the SQ call filled the Veff halo by its own exchange; the warm
  // start is the value the call began with.
  SQ.lambda_f = lambda_in;
  sqb::export_case(&SQ, (out + "_in.sqc").c_str(), scf_iter, true);
  SQ.lambda_f = lambda_out;

  sqb::CaseWriter w(out + "_out.sqc");
  std::vector<double> rho((size_t)nnode), rpj((size_t)nnode * (SQ.npl + 1)), ci((size_t)nnode * (SQ.npl + 1));
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) rho[((size_t)k * ny + j) * nx + i] = SQ.rho[k][j][i];
  for (int n = 0; n < nnode; n++)
    for (int q = 0; q <= SQ.npl; q++) {
      rpj[(size_t)n * (SQ.npl + 1) + q] = SQ.rho_pj[n][q];
      ci[(size_t)n * (SQ.npl + 1) + q] = SQ.Ci[n][q];
    }
  w.f64("rho", rho.data(), {nz, ny, nx});
  w.f64("rho_pj", rpj.data(), {nnode, SQ.npl + 1});
  w.f64("Ci", ci.data(), {nnode, SQ.npl + 1});
  w.f64("chi", SQ.chi, {nnode});
  w.f64("zee", SQ.zee, {nnode});
  w.f64s("lambda_f", lambda_out);
  w.f64s("Ebs", SQ.Ebs);
  w.f64s("Eent", SQ.Eent);
  w.f64s("t_sq", t_sq);
  w.f64s("t_projectors", t_proj);

  if (hv_count > 0) {
    const int n = 2 * nl + 1;
    const size_t nw = (size_t)n * n * n;
    std::vector<int> nodes;
    std::vector<double> vin, vout;
    double ***vec = new double **[n], ***hv = new double **[n];
    for (int k = 0; k < n; k++) {
      vec[k] = new double *[n];
      hv[k] = new double *[n];
      for (int j = 0; j < n; j++) {
        vec[k][j] = new double[n];
        hv[k][j] = new double[n];
      }
    }
    for (int c = 0; c < hv_count; c++) {
      const int node = (int)(((long long)c * 7919 + 13) % nnode);
      const int i = node % nx, j = (node / nx) % ny, k = node / (nx * ny);
      nodes.push_back(node);
      for (int kk = 0; kk < n; kk++)
        for (int jj = 0; jj < n; jj++)
          for (int ii = 0; ii < n; ii++) {
            vec[kk][jj][ii] = lcg_uniform();
            vin.push_back(vec[kk][jj][ii]);
          }
      HsubTimesVec(&SQ, vec, i + nl, j + nl, k + nl, hv);
      for (int kk = 0; kk < n; kk++)
        for (int jj = 0; jj < n; jj++)
          for (int ii = 0; ii < n; ii++) vout.push_back(hv[kk][jj][ii]);
    }
    w.i32("hv_nodes", nodes.data(), {hv_count});
    w.f64("hv_in", vin.data(), {hv_count, (int64_t)nw});
    w.f64("hv_out", vout.data(), {hv_count, (int64_t)nw});
  }

  if (do_forces) {
    t0 = MPI_Wtime();
    ForcesNonLocal(&SQ);
    const double t_f = MPI_Wtime() - t0;
    std::vector<double> f((size_t)SQ.n_atm * 3);
    for (int a = 0; a < SQ.n_atm; a++) {
      f[3 * a] = SQ.fnlocx[a];
      f[3 * a + 1] = SQ.fnlocy[a];
      f[3 * a + 2] = SQ.fnlocz[a];
    }
    w.f64("fnloc", f.data(), {SQ.n_atm, 3});
    w.f64s("t_forces", t_f);
  }
  w.close();

  if (do_local) write_local();
  std::printf("sqref_driver: wrote %s_in.sqc and %s_out.sqc (SQ %.3f s)\n", out.c_str(), out.c_str(), t_sq);
  return 0;
}
