// The expansion classes of pb-sam_b200/cpp/pbsam_b200.hpp (CExpan, CGradExpan,
// CRotCoeff, CTransCoeff, CXFormA) driven the way the reference's code drives its own:
// one operation per line of the input, results one line each (the test compares them
// with the oracle's restatement of the reference's classes).
//
// input lines:
//   init <poles> <kappa> <sdiel> <temperature>
//   rotate <theta> <phi> <xi> <p> <with_xi> <forward> <poles^2 coefficients>
//   rotateq <w> <x> <y> <z> <p> <forward> <poles^2 coefficients>      (CRotCoeff::reset(CQuat))
//   translate <rho> <kappa or 0> <scale in> <scale out> <p> <deriv> <poles^2 coefficients>
//   xform <Px> <Py> <Pz> <r source> <r target> <p> <screened> <grad> <poles^2 coefficients>
//   batch <n>, then n lines "<theta> <phi> <xi> <poles^2 coefficients>" (rotateBatch, forward)
//   inprod <M scale> <L scale> <poles^2 M> <poles^2 L>
// output lines: "kappa <k>", "out <scale> <poles^2>", "grad <3 poles^2>", "inprod <v>".
// Exit status 0, or 2 on bad input, 3 when a library call fails.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "pbsam_b200.hpp"

static std::vector<double> read_coeffs(std::istream &in, int n)
{
  std::vector<double> v(n);
  for (int i = 0; i < n; i++) in >> v[i];
  return v;
}

static void put(FILE *out, const CExpan &e, int NP)
{
  const std::vector<double> v = e.padded(NP);
  std::fprintf(out, "out %.17g", e.getScale());
  for (double x : v) std::fprintf(out, " %.17g", x);
  std::fprintf(out, "\n");
}

int main(int argc, char **argv)
{
  if (argc < 3) return 2;
  std::ifstream in(argv[1]);
  FILE *out = std::fopen(argv[2], "w");
  if (!in || !out) return 2;
  int NP = 0;
  std::string tok;
  while (in >> tok) {
    if (tok == "init") {
      double kappa, sdiel, temp;
      in >> NP >> kappa >> sdiel >> temp;
      if (!CSystem::initConstants(kappa, sdiel, temp, NP)) return 3;
      std::fprintf(out, "kappa %.17g\n", CSystem::getKappa());
      continue;
    }
    if (NP == 0) return 2;
    const int NP2 = NP * NP;
    if (tok == "rotate" || tok == "rotateq") {
      CRotCoeff R;
      int p, withXi = 0, fwd;
      if (tok == "rotate") {
        double th, ph, xi;
        in >> th >> ph >> xi >> p >> withXi >> fwd;
        R.reset(th, ph, xi, p);
      } else {
        double w, x, y, z;
        in >> w >> x >> y >> z >> p >> fwd;
        R.reset(CQuat(w, CPnt(x, y, z)), p);
      }
      const CExpan M(read_coeffs(in, NP2), 0.25);
      CExpan O;
      const bool ok = withXi ? R.rotateWithXi(M, O, fwd != 0) : R.rotate(M, O, fwd != 0);
      if (!ok) return 3;
      put(out, O, NP);
    } else if (tok == "translate") {
      double rho, kap, si, so;
      int p, deriv;
      in >> rho >> kap >> si >> so >> p >> deriv;
      CTransCoeff T;
      if (!T.reset(rho, kap, p, si, so)) return 3;
      const CMulExpan M(read_coeffs(in, NP2), 1.0 / si);
      CLocalExpan L;
      if (!(deriv ? T.dTranslate(M, L) : T.translate(M, L))) return 3;
      put(out, L, NP);
    } else if (tok == "xform") {
      double px, py, pz, rs, rt;
      int p, screened, grad;
      in >> px >> py >> pz >> rs >> rt >> p >> screened >> grad;
      CXFormA X(rs, rt);
      X.reset(CPnt(px, py, pz), p);
      const CMulExpan M(read_coeffs(in, NP2), 1.0 / rs);
      CLocalExpan L;
      CGradExpan G;
      bool ok;
      if (!screened) ok = X.xformF(M, L);
      else if (grad) ok = X.xformH(M, L, G);
      else ok = X.xformH(M, L);
      if (!ok) return 3;
      put(out, L, NP);
      if (screened && grad) {
        std::fprintf(out, "grad");
        for (int c = 0; c < 3; c++)
          for (double x : G[c].padded(NP)) std::fprintf(out, " %.17g", x);
        std::fprintf(out, "\n");
      }
    } else if (tok == "batch") {
      int n;
      in >> n;
      std::vector<CRotCoeff> R(n);
      std::vector<CExpan> M(n), O;
      for (int i = 0; i < n; i++) {
        double th, ph, xi;
        in >> th >> ph >> xi;
        R[i].reset(th, ph, xi, NP);
        M[i] = CExpan(read_coeffs(in, NP2), 1.0);
      }
      if (!CRotCoeff::rotateBatch(R, M, O, true)) return 3;
      for (int i = 0; i < n; i++) put(out, O[i], NP);
    } else if (tok == "inprod") {
      double ms, ls;
      in >> ms >> ls;
      const CMulExpan M(read_coeffs(in, NP2), ms);
      const CLocalExpan L(read_coeffs(in, NP2), ls);
      std::fprintf(out, "inprod %.17g\n", inprod(M, L));
    } else {
      return 2;
    }
  }
  std::fclose(out);
  CSystem::clear();
  return 0;
}
