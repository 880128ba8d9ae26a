// Brownian-dynamics harness around the reference's own CBDnam (test oracle only).
//
// Builds the reference's two-molecule NAM driver exactly as bdnam does
// (CSystem::initConstants, CBDnam::initConstants(2), the CBDnam constructor
// reading PQR, IMats and .exp files, src/BDnam_main.cpp:26-78,
// src/BDnam.cpp:48-150), seeds drand48 with a given seed instead of the clock,
// places the molecules at the spec's poses, and runs the body of CBDnam::run's
// loop (src/BDnam.cpp:196-243: compute_dt, computeForces inside f_DIST, the
// drifts, makeMove) for n steps, writing the poses after every step.  Contact
// definitions are loaded as bdnam loads them (CContact::setSepDist,
// CMolContact::readMolContact, CBDnam::addMolContact, src/BDnam_main.cpp:64-69) when
// the spec has a `contact` entry; without one IsDocked is always false.
//
// The class's private members (makeMove, m_mols, the diffusion constants) are
// reached by compiling this file with `private` defined as
// `public` around the reference header.
//
// spec: salt <mol/L>  idiel <eps_in>
//       moltype <pqr> <imat dir> <exp dir> <exp name>     (exactly two)
//       frame / mol <type> <x> <y> <z> <qw> <qx> <qy> <qz> (two molecules)
//       bd <mode (0)> <n steps> <seed> <unused>
//       contact <contactdef file> <docking distance>          (optional)
// output: BDSTEP <steps> <status> <force evaluations> <time>, then POSE lines,
// and TIME <wall seconds of the steps after the first> <their count> at the end;
// statuses numbered 0 running, 1 escaped, 2 stuck, 3 docked; exit status 4 when
// computeForces reports overlapping spheres (where bdnam exits).
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
#include "BDnam.h"
#undef private

int main(int argc, char **argv)
{
  if (argc < 3) return 2;
  std::ifstream in(argv[1]);
  if (!in) return 2;
  double salt = 0.05, idiel = 4.0;
  std::vector<std::vector<std::string> > types;
  std::vector<std::vector<double> > poses;
  int mode = 0, nsteps = 0;
  long seed = 0, unused = 0;
  std::string contactfile;
  double dockdist = 0.0;
  std::string tok;
  while (in >> tok) {
    if (tok == "salt") in >> salt;
    else if (tok == "idiel") in >> idiel;
    else if (tok == "moltype") { std::vector<std::string> t(4); in >> t[0] >> t[1] >> t[2] >> t[3]; types.push_back(t); }
    else if (tok == "frame") {}
    else if (tok == "mol") { int ty; std::vector<double> v(7); in >> ty; for (int k = 0; k < 7; k++) in >> v[k]; poses.push_back(v); }
    else if (tok == "bd") in >> mode >> nsteps >> seed >> unused;
    else if (tok == "contact") in >> contactfile >> dockdist;
    else if (tok == "poles" || tok == "dump" || tok == "energy") { std::string x; in >> x; }
    else if (tok == "tol") { std::string a, b, c, d; in >> a >> b >> c >> d; }
    else if (tok == "bdp" || tok == "bddiff" || tok == "bdnoise") { std::string rest; std::getline(in, rest); }
    else { fprintf(stderr, "bad token %s\n", tok.c_str()); return 2; }
  }
  if (types.size() != 2 || poses.size() != 2 || mode != 0) return 2;
  const double sdiel = 78.0, temperature = 298.15;
  const double kappa = ANGSTROM * sqrt((2 * salt * AVOGADRO_NUM / LITRE * ELECT_CHG * ELECT_CHG) /
                                       (sdiel * PERMITTIVITY_VAC * KB * temperature));
  CSystem::initConstants(kappa, sdiel, temperature);
  CBDnam::initConstants(2);
  if (!contactfile.empty()) {
    CContact::setSepDist(dockdist);
    std::vector<CMolContact> molcontactlist;
    int moltype = -1;
    std::streambuf *keep0 = std::cout.rdbuf();
    std::ofstream sink0("/dev/null");
    std::cout.rdbuf(sink0.rdbuf());
    CMolContact::readMolContact(contactfile.c_str(), moltype, molcontactlist);
    std::cout.rdbuf(keep0);
    if (moltype != 0) return 2;
    CBDnam::addMolContact(moltype, molcontactlist);
  }
  std::vector<char *> f1, f2;
  for (int k = 0; k < 4; k++) {
    f1.push_back(const_cast<char *>(types[0][k].c_str()));
    f2.push_back(const_cast<char *>(types[1][k].c_str()));
  }
  std::streambuf *keep = std::cout.rdbuf();
  std::ofstream sink("/dev/null");
  std::cout.rdbuf(sink.rdbuf());                 // the constructor's progress messages
  CBDnam bd(f1, f2, idiel);
  std::cout.rdbuf(keep);
  srand48(seed);
  for (int i = 0; i < 2; i++) {
    const std::vector<double> &v = poses[i];
    bd.m_mols[i]->setPos(CPnt(v[0], v[1], v[2]));
    bd.m_mols[i]->setOrient(CQuat(v[3], CPnt(v[4], v[5], v[6])));
  }
  FILE *out = fopen(argv[2], "w");
  if (!out) return 2;
  std::vector<CPnt> force(2), torque(2);
  CPnt dR2, dO1, dO2;
  CBDnam::STATUS status = CBDnam::RUNNING;
  int fevals = 0;
  double time = 0.0;
  const int map_status[4] = {1, 3, 0, 2};       // ESCAPED, DOCKED, RUNNING, STUCK
  double t_start = 0.0;                         // wall time of the steps after the first
  int n_done = 0;
  for (int k = 0; k < nsteps && status == CBDnam::RUNNING; k++, n_done++) {
    if (k == 1) t_start = read_timer();
    // CBDnam::compute_dt is an inline member of BDnam.cpp, not linkable: its body
    // (src/BDnam.cpp:409-417) on the same members
    const REAL dsep = CMolecule::getSepDist(bd.m_mols[0], bd.m_mols[1]);
    const REAL dt = (dsep - 5 > 0) ? 2.0 + (dsep - 5) / 15 : 2.0;
    const REAL dist = CMolecule::getC2CDist(bd.m_mols[0], bd.m_mols[1]);
    if (dist < f_DIST) {
      if (!CMolecule::computeForces(bd.m_mols, force, torque)) { fclose(out); return 4; }
      fevals++;
      dR2 = (bd.m_Dtr * dt * FACT2) * force[1];
      dO1 = (bd.m_Dr1 * dt * IKbT * COUL_K) * torque[0];
      dO2 = (bd.m_Dr2 * dt * IKbT * COUL_K) * torque[1];
    } else {
      dR2.zero(); dO1.zero(); dO2.zero();
    }
    status = bd.makeMove(dR2, dO1, dO2, dt);
    time += dt;
    fprintf(out, "BDSTEP %d %d %d %.17e\n", k + 1, map_status[status], fevals, time);
    for (int i = 0; i < 2; i++) {
      const CPnt p = bd.m_mols[i]->getRCen();
      const CQuat q = bd.m_mols[i]->getOrient();
      fprintf(out, "POSE %d %.17e %.17e %.17e %.17e %.17e %.17e %.17e\n", i, p.x(), p.y(), p.z(), q.real(),
              q.imag().x(), q.imag().y(), q.imag().z());
    }
  }
  if (n_done > 1) fprintf(out, "TIME %.6e %d\n", read_timer() - t_start, n_done - 1);
  fclose(out);
  return 0;
}
