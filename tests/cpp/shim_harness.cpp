// The force/energy harness of the reference (oracle/ref_harness.cpp) written
// against the C++ host layer pb-sam_b200/cpp/pbsam_b200.hpp instead of the
// reference's classes: same spec file, same output format, so the tests compare
// the two line by line.
//
// spec: salt <mol/L>  idiel <eps_in>  poles <p>  dump 0  energy <0|1>
//       tol <max_polar_dev> <solve_tol> <solve_max_ct> <max_pol_rounds>
//       moltype <pqr> <imat dir> <exp dir> <exp name>   (per type)
//       frame / mol <type> <x> <y> <z> <qw> <qx> <qy> <qz>
// exit status: 0 done, 2 bad spec, 3 set-up failed (no GPU, unreadable files)
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "pbsam_b200.hpp"

struct Pose { int type; double v[7]; };

int main(int argc, char **argv)
{
  if (argc < 3) { std::fprintf(stderr, "usage: %s spec out\n", argv[0]); return 2; }
  std::ifstream in(argv[1]);
  if (!in) return 2;
  double salt = 0.05, idiel = 4.0;
  int poles = 10, energy = 1, dump = 0;
  std::vector<std::vector<std::string> > types;
  std::vector<std::vector<Pose> > frames;
  std::string tok;
  while (in >> tok) {
    if (tok == "salt") in >> salt;
    else if (tok == "idiel") in >> idiel;
    else if (tok == "poles") in >> poles;
    else if (tok == "energy") in >> energy;
    else if (tok == "dump") in >> dump;
    else if (tok == "tol") {
      double a, b;
      int c, d;
      in >> a >> b >> c >> d;
      CSystem::setTolerances(a, b, c, d);
    }
    else if (tok == "moltype") { std::vector<std::string> t(4); in >> t[0] >> t[1] >> t[2] >> t[3]; types.push_back(t); }
    else if (tok == "frame") frames.push_back(std::vector<Pose>());
    else if (tok == "mol") {
      if (frames.empty()) return 2;
      Pose p; in >> p.type; for (int k = 0; k < 7; k++) in >> p.v[k];
      frames.back().push_back(p);
    } else return 2;
  }
  if (frames.empty() || types.empty()) return 2;
  // kappa as the reference's drivers compute it (src/BDnam_main.cpp:53-55)
  const double sdiel = 78.0, temperature = 298.15;
  const double AVO = 6.0221415e23, ECHG = 1.60217646e-19, EPS0 = 8.854187817e-12;
  const double KBOLTZ = 1.3806503e-23, ANG = 1e-10, LIT = 1e-3;
  const double kappa = ANG * std::sqrt((2 * salt * AVO / LIT * ECHG * ECHG) / (sdiel * EPS0 * KBOLTZ * temperature));
  if (!CSystem::initConstants(kappa, sdiel, temperature, poles, idiel)) return 3;
  std::vector<int> ids;
  for (auto &t : types) {
    const int id = CMolecule::loadMolType(t[0].c_str(), t[1].c_str(), t[2].c_str(), t[3].c_str());
    if (id < 0) return 3;
    ids.push_back(id);
  }
  std::vector<CMolecule *> mols;
  for (const Pose &p : frames[0]) mols.push_back(new CMolecule(ids[p.type]));
  if (!CMolecule::initMutualConstants(mols, 10, 100, true)) return 3;
  FILE *out = std::fopen(argv[2], "w");
  if (!out) return 2;
  std::fprintf(out, "KAPPA %.17e\n", CSystem::getKappa());
  for (size_t f = 0; f < frames.size(); f++) {
    for (size_t i = 0; i < mols.size(); i++) {
      const double *v = frames[f][i].v;
      mols[i]->setPos(CPnt(v[0], v[1], v[2]));
      mols[i]->setOrient(CQuat(v[3], CPnt(v[4], v[5], v[6])));
    }
    std::vector<CPnt> force, torque;
    const bool ok = CMolecule::computeForces(mols, force, torque);
    std::fprintf(out, "FRAME %d %d 0\n", (int)f, ok ? 1 : 0);
    if (!ok) continue;
    for (size_t i = 0; i < mols.size(); i++) {
      std::fprintf(out, "FORCE %d %.17e %.17e %.17e\n", (int)i, force[i].x(), force[i].y(), force[i].z());
      std::fprintf(out, "TORQUE %d %.17e %.17e %.17e\n", (int)i, torque[i].x(), torque[i].y(), torque[i].z());
    }
    if (energy) std::fprintf(out, "ENERGY %.17e\n", CMolecule::computeTotalIntEnergy(mols));
    std::fflush(out);
  }
  std::fclose(out);
  for (CMolecule *m : mols) delete m;
  CSystem::clear();
  return 0;
}
