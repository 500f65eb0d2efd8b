// Topology assembly; see topology.h.
#include "topology.h"

#include <vector_functions.h>

#include <algorithm>
#include <cmath>
#include <set>
#include <sstream>
#include <stdexcept>

namespace apo {

int Topology::num_shake_constraints() const {
  int n = 0;
  for (auto &s : shake_atoms) n += 1 + (s.z != -1) + (s.w != -1);
  return n;
}

int Topology::degrees_of_freedom(bool holonomic) const {
  int ndegf = 3 * natom - 3;
  if (holonomic) ndegf -= 3 * (int)waters.size() + num_shake_constraints();
  return ndegf;
}

Topology build_topology(const CharmmPSF &psf, const CharmmParameters &prm) {
  Topology t;
  const int n = psf.getNumAtoms();
  t.natom = n;
  t.charge = psf.getCharges();
  t.mass = psf.getMasses();
  const auto &at = psf.getAtomTypes();
  const auto &an = psf.getAtomNames();

  // ---- connectivity: 1-2, 1-3, 1-4 sets (src/CharmmPSF.cu:331-385)
  std::vector<std::set<int>> c12(n), c13(n), c14(n);
  for (auto &b : psf.getBonds()) {
    c12[b.i].insert(b.j);
    c12[b.j].insert(b.i);
  }
  for (auto &b : psf.getBonds()) {
    for (int k : c12[b.j])
      if (k != b.i) c13[b.i].insert(k);
    for (int k : c12[b.i])
      if (k != b.j) c13[b.j].insert(k);
  }
  for (int i = 0; i < n; ++i)
    for (int j : c13[i])
      for (int k : c12[j])
        if (!c12[i].count(k)) c14[i].insert(k);

  // ---- in14 / ex14 (src/CharmmPSF.cu:235-279) and symmetric exclusion CSR
  std::vector<std::vector<int>> nbr(n);
  for (int i = 0; i < n; ++i) {
    for (int j : c14[i])
      if (j > i && !c12[i].count(j) && !c13[i].count(j)) t.in14.push_back({i, j});
    std::set<int> ex;
    for (int j : c12[i])
      if (j > i) ex.insert(j);
    for (int j : c13[i])
      if (j > i) ex.insert(j);
    for (int j : ex) t.ex14.push_back({i, j});
    std::set<int> all = ex;
    for (int j : c14[i])
      if (j > i) all.insert(j);
    for (int j : all) {
      nbr[i].push_back(j);
      nbr[j].push_back(i);
    }
  }
  t.excl_ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    std::sort(nbr[i].begin(), nbr[i].end());
    t.excl_ptr[i + 1] = t.excl_ptr[i] + (int)nbr[i].size();
  }
  t.excl_idx.reserve(t.excl_ptr[n]);
  for (int i = 0; i < n; ++i)
    t.excl_idx.insert(t.excl_idx.end(), nbr[i].begin(), nbr[i].end());

  // ---- LJ tables (src/CharmmParameters.cu:718-844)
  std::set<std::string> tset(at.begin(), at.end());
  t.types.assign(tset.begin(), tset.end());
  const int T = (int)t.types.size();
  t.vdw.assign(T * T, make_float2(0.f, 0.f));
  t.vdw14.assign(T * T, make_float2(0.f, 0.f));
  for (int a = 0; a < T; ++a) {
    for (int b = 0; b <= a; ++b) {
      const std::string &ti = t.types[a], &tj = t.types[b];
      for (int which = 0; which < 2; ++which) {
        double eps, rmin;
        auto nf = prm.nbfix.find({tj, ti});
        if (nf != prm.nbfix.end()) {
          eps = nf->second.emin;
          rmin = nf->second.rmin;
        } else {
          auto fi = prm.vdw.find(ti), fj = prm.vdw.find(tj);
          if (fi == prm.vdw.end() || fj == prm.vdw.end())
            throw std::invalid_argument("vdw parameters not found for type " +
                                        (fi == prm.vdw.end() ? ti : tj));
          double ei = fi->second.eps, ri = fi->second.rmin2;
          double ej = fj->second.eps, rj = fj->second.rmin2;
          if (which == 1) {
            auto gi = prm.vdw14.find(ti), gj = prm.vdw14.find(tj);
            if (gi != prm.vdw14.end()) { ei = gi->second.eps; ri = gi->second.rmin2; }
            if (gj != prm.vdw14.end()) { ej = gj->second.eps; rj = gj->second.rmin2; }
          }
          eps = std::sqrt(ei * ej);
          rmin = ri + rj;
        }
        // the reference stores c6/c12 as float before scaling by 6 and 12
        float c12 = (float)(eps * std::pow(rmin, 12));
        float c6 = (float)(2.0 * eps * std::pow(rmin, 6));
        float2 v = make_float2(6.0f * c6, 12.0f * c12);
        auto &tab = which == 0 ? t.vdw : t.vdw14;
        tab[a * T + b] = v;
        tab[b * T + a] = v;
      }
    }
  }
  t.vdwtype.resize(n);
  for (int i = 0; i < n; ++i)
    t.vdwtype[i] = (int)(std::lower_bound(t.types.begin(), t.types.end(), at[i]) -
                         t.types.begin());

  // ---- bonded terms (src/CharmmParameters.cu:357-700)
  auto sorted2 = [](std::string a, std::string b) {
    if (a > b) std::swap(a, b);
    return Key2{a, b};
  };
  const auto &bonds = psf.getBonds();
  for (size_t k = 0; k < bonds.size(); ++k) {
    auto key = sorted2(at[bonds[k].i], at[bonds[k].j]);
    auto f = prm.bonds.find(key);
    if (f == prm.bonds.end()) {
      std::ostringstream m;
      m << "bond not found " << k << " (" << key.first << ", " << key.second << ") "
        << bonds[k].i << " " << bonds[k].j;
      throw std::invalid_argument(m.str());
    }
    t.bond_ij.push_back({bonds[k].i, bonds[k].j});
    t.bond_p.push_back({f->second.kb, f->second.b0});
  }
  const auto &angles = psf.getAngles();
  for (size_t k = 0; k < angles.size(); ++k) {
    std::string a1 = at[angles[k].i], a2 = at[angles[k].j], a3 = at[angles[k].k];
    if (a1 > a3) std::swap(a1, a3);
    Key3 key{a1, a2, a3};
    auto f = prm.angles.find(key);
    if (f == prm.angles.end()) {
      std::ostringstream m;
      m << "Angle not found " << k << " (" << a1 << ", " << a2 << ", " << a3 << ")";
      throw std::invalid_argument(m.str());
    }
    t.angle_ijk.push_back({angles[k].i, angles[k].j, angles[k].k, 0});
    t.angle_p.push_back({f->second.ktheta, f->second.theta0});
    auto u = prm.ureyb.find(key);
    if (u != prm.ureyb.end() && std::fabs(u->second.kb) > 0.01f) {
      t.ub_ij.push_back({angles[k].i, angles[k].k});
      t.ub_p.push_back({u->second.kb, u->second.b0});
    }
  }
  const auto &dihe = psf.getDihedrals();
  for (size_t k = 0; k < dihe.size(); ++k) {
    std::string a1 = at[dihe[k].i], a2 = at[dihe[k].j], a3 = at[dihe[k].k],
                a4 = at[dihe[k].l];
    if (a1 > a4) {
      std::swap(a1, a4);
      std::swap(a2, a3);
    }
    if (a1 == a4 && a2 > a3) std::swap(a2, a3);
    auto f = prm.dihedrals.find(Key4{a1, a2, a3, a4});
    if (f == prm.dihedrals.end()) {
      std::string b2 = a2, b3 = a3;
      if (b2 > b3) std::swap(b2, b3);
      f = prm.dihedrals.find(Key4{"X", b2, b3, "X"});
    }
    if (f == prm.dihedrals.end()) {
      std::ostringstream m;
      m << "dihedral not found " << k << " " << at[dihe[k].i] << " " << at[dihe[k].j]
        << " " << at[dihe[k].k] << " " << at[dihe[k].l] << "\t" << an[dihe[k].i]
        << " " << an[dihe[k].j] << " " << an[dihe[k].k] << " " << an[dihe[k].l];
      throw std::invalid_argument(m.str());
    }
    t.dihe_ijkl.push_back({dihe[k].i, dihe[k].j, dihe[k].k, dihe[k].l});
    t.dihe_terms.push_back({(int)t.dihe_coef.size(), (int)f->second.size()});
    for (auto &term : f->second) {
      double d = term.delta * M_PI / 180.0;
      t.dihe_coef.push_back(make_float4(term.k, (float)term.n, (float)std::cos(d),
                                        (float)std::sin(d)));
    }
  }
  const auto &imp = psf.getImpropers();
  for (size_t k = 0; k < imp.size(); ++k) {
    std::string a1 = at[imp[k].i], a2 = at[imp[k].j], a3 = at[imp[k].k],
                a4 = at[imp[k].l];
    if (a1 > a4) {
      std::swap(a1, a4);
      std::swap(a2, a3);
    }
    if (a1 == a4 && a2 > a3) std::swap(a2, a3);
    auto f = prm.impropers.find(Key4{a1, a2, a3, a4});
    if (f == prm.impropers.end()) f = prm.impropers.find(Key4{a1, "X", "X", a4});
    if (f == prm.impropers.end()) {
      std::ostringstream m;
      m << "improper not found " << k << " " << at[imp[k].i] << " " << at[imp[k].j]
        << " " << at[imp[k].k] << " " << at[imp[k].l];
      throw std::invalid_argument(m.str());
    }
    t.imp_ijkl.push_back({imp[k].i, imp[k].j, imp[k].k, imp[k].l});
    t.imp_p.push_back({f->second.kpsi, (float)(f->second.psi0 * M_PI / 180.0)});
  }

  // ---- constraints
  for (auto &w : psf.getWaterMolecules()) t.waters.push_back({w[0], w[1], w[2], 0});
  {
    // X-H clusters (src/ForceManager.cu:844-921); water is handled by SETTLE
    std::vector<std::vector<int>> hyd(n);
    for (auto &b : bonds) {
      const std::string &ti = at[b.i], &tj = at[b.j];
      bool hi = !ti.empty() && ti[0] == 'H', hj = !tj.empty() && tj[0] == 'H';
      if (!(hi || hj)) continue;
      if ((ti == "OT" && tj == "HT") || (ti == "HT" && tj == "OT") || (hi && hj)) continue;
      if (hi) hyd[b.j].push_back(b.i);
      else hyd[b.i].push_back(b.j);
    }
    for (int i = 0; i < n; ++i) {
      if (hyd[i].empty()) continue;
      if (hyd[i].size() > 3)
        throw std::invalid_argument("SHAKE cluster with more than 3 hydrogens at atom " +
                                    std::to_string(i));
      int4 g = {i, -1, -1, -1};
      int *slot = &g.y;
      float b0 = 0.f;
      for (size_t j = 0; j < hyd[i].size(); ++j) {
        slot[j] = hyd[i][j];
        auto f = prm.bonds.find(sorted2(at[i], at[hyd[i][j]]));
        if (f != prm.bonds.end()) b0 = f->second.b0;
      }
      t.shake_atoms.push_back(g);
      // inverse masses rounded as the reference rounds them (1.0f / (float)m)
      t.shake_p.push_back(make_float4(1.0f / (float)t.mass[i], 0.f, b0 * b0,
                                      1.0f / (float)t.mass[hyd[i].back()]));
    }
  }
  for (auto &g : psf.getConnectedComponents()) t.groups.push_back({g[0], g[1]});
  return t;
}

}  // namespace apo
