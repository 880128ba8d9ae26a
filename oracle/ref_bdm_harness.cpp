// Brownian-dynamics harness around the reference's own CBDmulti (test oracle only).
//
// Builds the reference's multi-molecule driver as bdm does (CSystem::initConstants,
// with the periodic box when the spec has `box <L>`, CBDmulti::initConstants(2) before the molecules exist,
// the CBDmulti constructor with np1 copies of species 0 and np2 of species 1,
// src/BDmulti_main.cpp:28-90, src/BDmulti.cpp:26-207), seeds drand48 with a given
// seed, places the molecules at the spec's poses (species 0 copies first), and runs
// the body of CBDmulti::runFirstDockTime's loop (computeMinSepDist, propagate:
// forces below the interaction cutoff, drifts, makeMove; src/BDmulti.cpp:340-440)
// for n steps, writing the poses after every step.
//
// The class's private members are reached by compiling this file with `private`
// defined as `public` around the reference header.
//
// spec: salt, idiel, two moltype lines, one frame of mol lines (types 0 then 1),
//       bd <mode (1)> <n steps> <seed> <unused>
// output: BDSTEP <steps> 0 <force evaluations> <time>, then POSE lines, and TIME <wall
// seconds of the steps after the first> <their count> at the end; exit status 4 when
// computeForces reports overlapping spheres (where bdm exits).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>
#include <map>
#include <set>
#include "molecule.h"
#include "system.h"
#include "readutil.h"
#include "contact.h"
#define private public
#include "BDmulti.h"
#undef private

int main(int argc, char **argv)
{
  if (argc < 3) return 2;
  std::ifstream in(argv[1]);
  if (!in) return 2;
  double salt = 0.05, idiel = 4.0;
  double box = 0.0;
  std::vector<std::vector<std::string> > types;
  std::vector<int> ptype;
  std::vector<std::vector<double> > poses;
  int mode = 1, nsteps = 0;
  long seed = 0, unused = 0;
  std::string tok;
  while (in >> tok) {
    if (tok == "salt") in >> salt;
    else if (tok == "idiel") in >> idiel;
    else if (tok == "moltype") { std::vector<std::string> t(4); in >> t[0] >> t[1] >> t[2] >> t[3]; types.push_back(t); }
    else if (tok == "frame") {}
    else if (tok == "mol") {
      int ty; std::vector<double> v(7); in >> ty; for (int k = 0; k < 7; k++) in >> v[k];
      ptype.push_back(ty); poses.push_back(v);
    }
    else if (tok == "bd") in >> mode >> nsteps >> seed >> unused;
    else if (tok == "box") in >> box;
    else if (tok == "poles" || tok == "dump" || tok == "energy") { std::string x; in >> x; }
    else if (tok == "tol") { std::string a, b, c, d; in >> a >> b >> c >> d; }
    else if (tok == "bdp" || tok == "bddiff" || tok == "bdnoise") { std::string rest; std::getline(in, rest); }
    else { fprintf(stderr, "bad token %s\n", tok.c_str()); return 2; }
  }
  if (types.size() != 2 || mode != 1) return 2;
  int np1 = 0, np2 = 0;
  for (size_t i = 0; i < ptype.size(); i++) {
    if (ptype[i] == 0) { if (np2) return 2; np1++; }   // species 0 copies come first
    else np2++;
  }
  const double sdiel = 78.0, temperature = 298.15;
  const double kappa = ANGSTROM * sqrt((2 * salt * AVOGADRO_NUM / LITRE * ELECT_CHG * ELECT_CHG) /
                                       (sdiel * PERMITTIVITY_VAC * KB * temperature));
  // a cubic periodic box when the spec gives one (bdm: src/BDmulti_main.cpp:67)
  if (box > 0) CSystem::initConstants(kappa, sdiel, temperature, true, box);
  else CSystem::initConstants(kappa, sdiel, temperature);
  CBDmulti::initConstants(2);
  std::vector<char *> f1, f2;
  for (int k = 0; k < 4; k++) {
    f1.push_back(const_cast<char *>(types[0][k].c_str()));
    f2.push_back(const_cast<char *>(types[1][k].c_str()));
  }
  std::streambuf *keep = std::cout.rdbuf();
  std::ofstream sink("/dev/null");
  std::cout.rdbuf(sink.rdbuf());                 // the constructor's progress messages
  CBDmulti bd(np1, np2, f1, f2, idiel);
  std::cout.rdbuf(keep);
  srand48(seed);
  for (size_t i = 0; i < poses.size(); i++) {
    const std::vector<double> &v = poses[i];
    bd.m_mols[i]->setPos(CPnt(v[0], v[1], v[2]));
    bd.m_mols[i]->setOrient(CQuat(v[3], CPnt(v[4], v[5], v[6])));
  }
  FILE *out = fopen(argv[2], "w");
  if (!out) return 2;
  int fevals = 0;
  double time = 0.0, t_start = 0.0;
  for (int k = 0; k < nsteps; k++) {
    if (k == 1) t_start = read_timer();
    const REAL minDist = bd.computeMinSepDist();
    if (minDist < CMolecule::m_interactRcutoff) fevals++;
    std::cout.rdbuf(sink.rdbuf());               // propagate's failure path prints and exits
    const double dt = bd.propagate(minDist, false);
    std::cout.rdbuf(keep);
    time += dt;
    fprintf(out, "BDSTEP %d 0 %d %.17e\n", k + 1, fevals, time);
    for (size_t i = 0; i < bd.m_mols.size(); i++) {
      const CPnt p = bd.m_mols[i]->getRCen();
      const CQuat q = bd.m_mols[i]->getOrient();
      fprintf(out, "POSE %d %.17e %.17e %.17e %.17e %.17e %.17e %.17e\n", (int)i, p.x(), p.y(), p.z(), q.real(),
              q.imag().x(), q.imag().y(), q.imag().z());
    }
    fflush(out);
  }
  if (nsteps > 1) fprintf(out, "TIME %.6e %d\n", read_timer() - t_start, nsteps - 1);
  fclose(out);
  return 0;
}
