// Force/energy harness around the reference PB-SAM classes (test oracle only).
//
// Builds molecule types exactly as the reference BD driver does
// (CBDnam::CBDnam, src/BDnam.cpp:48-150): read PQR, IMats and self-polarized
// F/H expansions, generate exposed surface points, self surface charges,
// intra-molecular pol lists and moltype self local expansions, then construct
// one CMolecule per placed copy and call CMolecule::initMutualConstants(mols,
// 10, 100, true).  For every frame of the spec it sets poses
// (setPos/setOrient, src/molecule.h:325-326), calls CMolecule::computeForces
// (src/moldynamics.cpp:553-587) and CMolecule::computeTotalIntEnergy
// (src/moldynamics.cpp:358-386), and writes the results with 17 significant
// digits.  Frames run in order in one process, so the reference's state carried
// between calls is reproduced as a BD run would see it.
//
// spec file (whitespace separated):
//   salt <mol/L>          idiel <eps_in>        dump <0|1>       energy <0|1>
//   moltype <pqr> <imat dir> <exp dir> <exp name>      (repeat per type)
//   frame                                               (starts a frame)
//   mol <type> <x> <y> <z> <qw> <qx> <qy> <qz>          (one per molecule)
//   box <L>                                             (optional: a cubic periodic box,
//                                                       CSystem::initConstants(..., true, L))
//   potpoint <x> <y> <z>                                (optional, repeat: after each
//                                                       frame, CMolecule::computePotInSpace
//                                                       at the point, src/moldynamics.cpp:470-506)
// The molecule list (types and count) must be the same in every frame.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include "molecule.h"
#include "system.h"
#include "readutil.h"

struct MolTypeData {
  std::vector<CPnt> scen, pos;
  std::vector<double> srad, chg;
  CPnt rcen;
  std::vector<REAL*> iMats;
  std::vector<CMulExpan*> iF, iH;
  std::vector<std::vector<CPnt> > SPxes;
  std::vector<int> nSPx;
  std::vector<std::vector<int> > neighs, near, far;
  std::vector<std::vector<double> > qF, qH;
  std::vector<double> tF, tH;
  std::vector<CLocalExpan*> LF, LH, LFfar, LHfar;
  std::vector<CMolCell> cells;
};

struct Pose { int type; double x, y, z, qw, qx, qy, qz; };

static void load_moltype(MolTypeData &m, const char *pqr, const char *imatdir,
                         const char *expdir, const char *expname, double idiel)
{
  readpqr(pqr, m.pos, m.chg, m.srad, m.scen);
  const int n = m.scen.size();
  m.rcen = CPnt(0, 0, 0);
  for (int i = 0; i < n; i++) m.rcen += m.scen[i];
  m.rcen /= n;
  readMats(m.iMats, N_POLES, const_cast<char*>(imatdir), n);
  REAL rc;
  readExpansionsP(m.iF, m.iH, N_POLES, const_cast<char*>(expdir), const_cast<char*>(expname), n, rc);
  const double intraRcutoff = 30;
  CMolecule::generateMolSPX(m.scen, m.srad, m.SPxes, m.nSPx, m.neighs);
  CMolecule::generateMolExposedChargesFH(m.iF, m.iH, m.scen, m.srad, m.SPxes, m.nSPx,
                                         m.qF, m.qH, m.tF, m.tH);
  CMolecule::generateMolTypeIntraPolLists(m.scen, m.srad, intraRcutoff, m.near, m.far);
  CMolecule::computeMolTypeValues(m.rcen, m.scen, m.srad, m.chg, m.pos, idiel, intraRcutoff,
                                  m.SPxes, m.nSPx, m.neighs, m.iF, m.iH, m.qF, m.qH, m.tF, m.tH,
                                  m.near, m.far, m.LF, m.LH, m.LFfar, m.LHfar);
}

static void dump_expan(FILE *f, const char *tag, int i, int ki, const CExpan &E)
{
  const std::vector<REAL> &v = E.getVector();
  fprintf(f, "%s %d %d %d", tag, i, ki, (int)v.size());
  for (size_t k = 0; k < v.size(); k++) fprintf(f, " %.17e", v[k]);
  fprintf(f, "\n");
}

int main(int argc, char **argv)
{
  if (argc < 3) { fprintf(stderr, "usage: harness <spec> <out>\n"); return 2; }
  std::ifstream in(argv[1]);
  if (!in) { fprintf(stderr, "cannot open spec\n"); return 2; }
  double salt = 0.05, idiel = 4.0, box = 0.0;
  int dump = 0, energy = 1;
  std::vector<std::vector<std::string> > types;
  std::vector<std::vector<Pose> > frames;
  std::vector<CPnt> potpts;
  std::string tok;
  while (in >> tok) {
    if (tok == "salt") in >> salt;
    else if (tok == "idiel") in >> idiel;
    else if (tok == "dump") in >> dump;
    else if (tok == "energy") in >> energy;
    else if (tok == "moltype") {
      std::vector<std::string> t(4);
      in >> t[0] >> t[1] >> t[2] >> t[3];
      types.push_back(t);
    } else if (tok == "frame") frames.push_back(std::vector<Pose>());
    else if (tok == "mol") {
      Pose p; in >> p.type >> p.x >> p.y >> p.z >> p.qw >> p.qx >> p.qy >> p.qz;
      frames.back().push_back(p);
    } else if (tok == "box") {
      in >> box;
    } else if (tok == "potpoint") {
      double x, y, z; in >> x >> y >> z;
      potpts.push_back(CPnt(x, y, z));
    } else { fprintf(stderr, "bad token %s\n", tok.c_str()); return 2; }
  }
  // constants as in the reference BD driver (src/BDnam_main.cpp:49-58)
  const double sdiel = 78.0, temperature = 298.15;
  const double AVO = 6.0221415e23, ECHG = 1.60217646e-19, EPS0 = 8.854187817e-12;
  const double KBOLTZ = 1.3806503e-23, ANG = 1e-10, LIT = 1e-3;
  const double kappa = ANG * sqrt((2 * salt * AVO / LIT * ECHG * ECHG) /
                                  (sdiel * EPS0 * KBOLTZ * temperature));
  if (box > 0) CSystem::initConstants(kappa, sdiel, temperature, true, box);   // periodic box (bdm)
  else CSystem::initConstants(kappa, sdiel, temperature);

  std::vector<MolTypeData> mt(types.size());
  for (size_t t = 0; t < types.size(); t++)
    load_moltype(mt[t], types[t][0].c_str(), types[t][1].c_str(), types[t][2].c_str(),
                 types[t][3].c_str(), idiel);

  FILE *out = fopen(argv[2], "w");
  fprintf(out, "KAPPA %.17e\n", kappa);
  std::vector<CMolecule*> mols;
  for (size_t i = 0; i < frames[0].size(); i++) {
    MolTypeData &m = mt[frames[0][i].type];
    mols.push_back(new CMolecule(frames[0][i].type, m.rcen, m.scen, m.srad, m.chg, m.pos, idiel,
                                 m.iMats, 30.0, m.SPxes, m.nSPx, m.neighs, m.near,
                                 m.iF, m.iH, m.LF, m.LH, m.LFfar, m.LHfar,
                                 m.qF, m.qH, m.tF, m.tH, m.cells));
  }
  CMolecule::initMutualConstants(mols, 10, 100, true);

  for (size_t f = 0; f < frames.size(); f++) {
    for (size_t i = 0; i < mols.size(); i++) {
      const Pose &p = frames[f][i];
      mols[i]->setPos(CPnt(p.x, p.y, p.z));
      mols[i]->setOrient(CQuat(p.qw, CPnt(p.qx, p.qy, p.qz)));
    }
    std::vector<CPnt> force, torque;
    double t0 = read_timer();
    bool ok = CMolecule::computeForces(mols, force, torque);
    double t1 = read_timer();
    fprintf(out, "FRAME %d %d %.6e\n", (int)f, ok ? 1 : 0, t1 - t0);
    if (!ok) continue;
    for (size_t i = 0; i < mols.size(); i++) {
      fprintf(out, "FORCE %d %.17e %.17e %.17e\n", (int)i, force[i].x(), force[i].y(), force[i].z());
      fprintf(out, "TORQUE %d %.17e %.17e %.17e\n", (int)i, torque[i].x(), torque[i].y(), torque[i].z());
    }
    if (energy) {
      double e = CMolecule::computeTotalIntEnergy(mols);
      fprintf(out, "ENERGY %.17e\n", e);
    }
    for (size_t k = 0; k < potpts.size(); k++)
      fprintf(out, "POT %d %.17e\n", (int)k, CMolecule::computePotInSpace(mols, potpts[k]));
    if (dump) {
      for (size_t i = 0; i < mols.size(); i++)
        for (int ki = 0; ki < mols[i]->getNKS(); ki++) {
          CSolExpCenter &K = mols[i]->getKS(ki);
          dump_expan(out, "F", i, ki, K.getF());
          dump_expan(out, "H", i, ki, K.getH());
          dump_expan(out, "LS", i, ki, K.getLS());
          const CGradExpan &g = K.getgLHN();
          for (int c = 0; c < 3; c++) {
            char tag[16]; sprintf(tag, "GLHN%d", c);
            dump_expan(out, tag, i, ki, g[c]);
          }
          const CGradExpan &gh = K.getGH();
          for (int c = 0; c < 3; c++) {
            char tag[16]; sprintf(tag, "GH%d", c);
            dump_expan(out, tag, i, ki, gh[c]);
          }
        }
    }
    fflush(out);
  }
  fclose(out);
  return 0;
}
