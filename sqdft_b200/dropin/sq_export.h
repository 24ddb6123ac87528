// Serialise the SQ-step inputs held in a DS_SQ into a case container.
//
// Compiled against the reference headers (ds_sq.h, func_sq.h).  It reads the
// fields that ClenshawCurtisSpectralQuadrature (sq.cpp:377-834),
// NonlocalProjectors (nonlocal.cpp:317-518) and ForcesNonLocal
// (forces.cpp:318-578) read, in the layouts ds_sq.h gives them:
//   * Veff on the processor + Rcut block, [np_z+2nloc][np_y+2nloc][np_x+2nloc]
//     (initialize.cpp:940-967), halo already filled;
//   * replica atoms whose rc-ball meets the processor + Rcut block
//     (Replica_atoms_Rcut, initialize.cpp:1003-1196), type-major, main atoms
//     in input order, replicas in the reference's z-y-x image order;
//   * per type the radial tables and spline derivatives (ds_sq.h:76-102) and
//     the Kleinman-Bylander denominators (readfiles.cpp:1154-1216);
//   * optionally (export_local) the pseudocharge inputs and fields of
//     ChargeDensity (initialize.cpp:470-784) and ForcesLocal (forces.cpp:20-315).
#pragma once
#include <cmath>
#include <string>
#include <vector>

#include "sq_case.h"

namespace sqb {

// Block field (np_z x np_y x np_x, with a halo of h) as a flat z-major array.
inline std::vector<double> block_field(double ***a, int nz, int ny, int nx, int h) {
  std::vector<double> v((size_t)(nz + 2 * h) * (ny + 2 * h) * (nx + 2 * h));
  size_t q = 0;
  for (int k = 0; k < nz + 2 * h; k++)
    for (int j = 0; j < ny + 2 * h; j++)
      for (int i = 0; i < nx + 2 * h; i++) v[q++] = a[k][j][i];
  return v;
}

// Pseudocharge replicas (Replica_atoms, initialize.cpp:21-160: the atoms
// whose rb-box meets the processor domain, DS_coord::ProcAtm) in the loop
// order of ChargeDensity and ForcesLocal (type, main atom, replica): type,
// global atom, coordinates and the intersection box; per type the radial
// grid, rVloc, uu and their spline derivatives (getYD_gen, as both functions
// form them) as 5 x size rows, and the valence charge.
struct LocalInputs {
  std::vector<int> rep_type, rep_atom, rep_box;
  std::vector<double> rep_xyz, Z;
  std::vector<std::vector<double>> tables;
};

inline LocalInputs gather_local(DS_SQ *p) {
  LocalInputs L;
  int atom_count = 0;
  for (int t = 0; t < p->n_typ; t++) {
    L.Z.push_back(p->Atm[t].Z);
    for (int a = 0; a < p->Atm[t].natm; a++, atom_count++)
      for (int r = 0; r < p->Atm[t].Rx[a].n_replica; r++) {
        const DS_ProcAtm &X = p->Atm[t].Rx[a].ProcAtm[r], &Y = p->Atm[t].Ry[a].ProcAtm[r],
                         &W = p->Atm[t].Rz[a].ProcAtm[r];
        L.rep_type.push_back(t);
        L.rep_atom.push_back(atom_count);
        L.rep_xyz.insert(L.rep_xyz.end(), {X.coord, Y.coord, W.coord});
        L.rep_box.insert(L.rep_box.end(), {X.start, X.end, Y.start, Y.end, W.start, W.end});
      }
    const int len = p->Psd[t].size;
    std::vector<double> tab((size_t)5 * len), dv(len), du(len);
    getYD_gen(p->Psd[t].RadialGrid, p->Psd[t].rVloc, dv.data(), len);
    getYD_gen(p->Psd[t].RadialGrid, p->Psd[t].uu, du.data(), len);
    for (int i = 0; i < len; i++) {
      tab[i] = p->Psd[t].RadialGrid[i];
      tab[(size_t)len + i] = p->Psd[t].rVloc[i];
      tab[(size_t)2 * len + i] = dv[i];
      tab[(size_t)3 * len + i] = p->Psd[t].uu[i];
      tab[(size_t)4 * len + i] = du[i];
    }
    L.tables.push_back(std::move(tab));
  }
  return L;
}

// The pseudocharge inputs (gather_local) and rc_tilda, and the block fields
// as the caller holds them: b, b_tilda, Vc, rho_at and phi with its FDn halo.
inline void export_local(DS_SQ *p, CaseWriter &w) {
  const LocalInputs L = gather_local(p);
  for (int t = 0; t < p->n_typ; t++)
    w.f64(("loc_tab" + std::to_string(t)).c_str(), L.tables[t].data(), {5, (int64_t)L.tables[t].size() / 5});
  const int64_t n = (int64_t)L.rep_type.size();
  w.i32("loc_rep_type", L.rep_type.data(), {n});
  w.i32("loc_rep_atom", L.rep_atom.data(), {n});
  w.f64("loc_rep_xyz", L.rep_xyz.data(), {n, 3});
  w.i32("loc_rep_box", L.rep_box.data(), {n, 6});
  w.f64("loc_Z", L.Z.data(), {p->n_typ});
  w.f64s("loc_rc_tilda", p->rc_tilda);
  const int nz = p->np_z, ny = p->np_y, nx = p->np_x, h = p->FDn;
  w.f64("loc_b", block_field(p->b, nz, ny, nx, 0).data(), {nz, ny, nx});
  w.f64("loc_b_tilda", block_field(p->b_tilda, nz, ny, nx, 0).data(), {nz, ny, nx});
  w.f64("loc_vc", block_field(p->Vc, nz, ny, nx, 0).data(), {nz, ny, nx});
  w.f64("loc_rho_at", block_field(p->rho_at, nz, ny, nx, 0).data(), {nz, ny, nx});
  w.f64("loc_phi", block_field(p->phi, nz, ny, nx, h).data(), {nz + 2 * h, ny + 2 * h, nx + 2 * h});
}

inline int proj_count(const DS_SQ *p, int t) {
  int n = 0;
  for (int l = 0; l <= p->Psd[t].lmax; l++)
    if (l != p->Atm[t].lloc) n += 2 * l + 1;
  return n;
}

inline void export_case(DS_SQ *p, const char *path, int scf_iter, bool with_udvtm, bool with_local = false) {
  CaseWriter w(path);
  const int nl = p->nloc;
  const int ex = p->np_x + 2 * nl, ey = p->np_y + 2 * nl, ez = p->np_z + 2 * nl;
  int pi[17] = {p->n_int[0], p->n_int[1], p->n_int[2], p->np_x, p->np_y, p->np_z,
                p->pnode_s[0], p->pnode_s[1], p->pnode_s[2], p->nloc, p->FDn, p->npl,
                p->fermi_alg, p->n_typ, p->n_atm, scf_iter, p->nproc};
  w.i32("params_i", pi, {17});
  double pd[8] = {p->delta, p->bet, p->lanczos_tol, p->fermi_tol, p->Ncharge, p->lambda_f, p->T, p->Rcut};
  w.f64("params_d", pd, {8});
  w.f64("coeff_lap", p->coeff_lap, {p->FDn + 1});
  w.f64("coeff_grad", p->coeff_grad, {p->FDn + 1});

  std::vector<double> v((size_t)ex * ey * ez);
  for (int k = 0; k < ez; k++)
    for (int j = 0; j < ey; j++)
      for (int i = 0; i < ex; i++) v[((size_t)k * ey + j) * ex + i] = p->Veff[k][j][i];
  w.f64("veff", v.data(), {ez, ey, ex});

  std::vector<int> ti;
  std::vector<double> td;
  std::vector<int> ri;
  std::vector<double> rx;
  std::vector<double> ud;
  std::vector<double> axyz;
  std::vector<int> atyp;
  int atom_count = 0;
  for (int t = 0; t < p->n_typ; t++) {
    const DS_Psd &ps = p->Psd[t];
    const int nlocc = (int)ceil(ps.rc / p->delta);  // nonlocal.cpp:43
    const int nproj = proj_count(p, t);
    const int nnd = (2 * nlocc + 1) * (2 * nlocc + 1) * (2 * nlocc + 1);
    int row[6] = {p->Atm[t].natm, ps.lmax, p->Atm[t].lloc, nlocc, ps.size, nproj};
    ti.insert(ti.end(), row, row + 6);
    double drow[6] = {ps.rc, ps.Denom_s, ps.Denom_p, ps.Denom_d, ps.Denom_f, (double)p->Atm[t].Z};
    td.insert(td.end(), drow, drow + 6);

    const double *tabs[19] = {ps.RadialGrid, ps.rVloc, ps.rVs, ps.rVp, ps.rVd, ps.rVf, ps.rUs,
                              ps.rUp, ps.rUd, ps.rUf, ps.DVloc, ps.DVsJ, ps.DVpJ, ps.DVdJ,
                              ps.DVfJ, ps.DUsJ, ps.DUpJ, ps.DUdJ, ps.DUfJ};
    std::vector<double> st((size_t)19 * ps.size, 0.0);
    for (int q = 0; q < 19; q++)
      if (tabs[q])
        for (int r = 0; r < ps.size; r++) st[(size_t)q * ps.size + r] = tabs[q][r];
    char nm[32];
    std::snprintf(nm, sizeof(nm), "psd%d", t);
    w.f64(nm, st.data(), {19, ps.size});

    for (int a = 0; a < p->Atm[t].natm; a++, atom_count++) {
      axyz.push_back(p->Atm[t].Rx[a].main_atm);
      axyz.push_back(p->Atm[t].Ry[a].main_atm);
      axyz.push_back(p->Atm[t].Rz[a].main_atm);
      atyp.push_back(t);
      for (int r = 0; r < p->Atm[t].Rx[a].n_replica_Rcut; r++) {
        int rr[3] = {t, a, atom_count};
        ri.insert(ri.end(), rr, rr + 3);
        rx.push_back(p->Atm[t].Rx[a].ProcAtmRcut[r].coord);
        rx.push_back(p->Atm[t].Ry[a].ProcAtmRcut[r].coord);
        rx.push_back(p->Atm[t].Rz[a].ProcAtmRcut[r].coord);
        if (with_udvtm && p->Atm[t].Rx[a].ProcAtmRcut[r].UdVtm)
          for (int c = 0; c < nproj; c++)
            ud.insert(ud.end(), p->Atm[t].Rx[a].ProcAtmRcut[r].UdVtm[c],
                      p->Atm[t].Rx[a].ProcAtmRcut[r].UdVtm[c] + nnd);
      }
    }
  }
  w.i32("typ_i", ti.data(), {p->n_typ, 6});
  w.f64("typ_d", td.data(), {p->n_typ, 6});
  const int64_t nrep = (int64_t)ri.size() / 3;
  w.i32("rep_i", ri.data(), {nrep, 3});
  w.f64("rep_xyz", rx.data(), {nrep, 3});
  w.f64("atoms_xyz", axyz.data(), {(int64_t)atyp.size(), 3});
  w.i32("atom_type", atyp.data(), {(int64_t)atyp.size()});
  if (with_udvtm) w.f64("udvtm", ud.data(), {(int64_t)ud.size()});
  if (with_local) export_local(p, w);
  w.close();
}

}  // namespace sqb
