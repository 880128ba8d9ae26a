// Multi-threaded CPU preparation of molecule-type inputs (test infrastructure).
//
// The restated oracle (pbsam_oracle.cpp) compiled a second time with OpenMP, plus
// two entry points that make the inputs of the force path without a GPU:
//
//   pbsam_prep_imat     the surface-integral matrices of `pbsam mat`
//                       (CMolecule IMat constructor, src/molecule.cpp:279-346;
//                       build_IMatE, computeIntegralE / computeIntegralB,
//                       src/expcenter.cpp:666-1033; sphere points,
//                       src/molecule.cpp:902-939, 2272-2294)
//   pbsam_prep_selfpol  the self-polarized expansions of `pbsam spol`
//                       (CMolecule::polarize_self, src/molecule.cpp:1898-1979,
//                       as driven by main_selfPolarize, src/selfp_makemat.cpp:37-118)
//
// They serve the CPU arm of the benchmark, which must time the reference without
// loading the CUDA library, and are pinned to the reference's own `pbsam mat` /
// `pbsam spol` output files in tests/test_oracle_prep.py.  The arithmetic is the
// oracle's; only the order of a few sums differs (threads over rows of the
// Gram matrix, over IMat rows, over neighbours), so results agree with the serial
// oracle to rounding.  Built with OpenMP by oracle.build_prep().
#define PBSAM_PREP 1
#include "pbsam_oracle.cpp"

#include <immintrin.h>
#include <omp.h>

using namespace orc;

namespace {

// unit-sphere spiral of n points (src/molecule.cpp:2272-2294)
void unit_spiral(int n, std::vector<P3> &q)
{
  std::vector<double> th, ph;
  sphere_pts(n, th, ph);
  q.resize(n);
  for (int i = 0; i < n; i++) q[i] = P3(1 * sin(th[i]) * cos(ph[i]), 1 * sin(th[i]) * sin(ph[i]), 1 * cos(th[i]));
}

// real spherical-harmonic components (packed layout) of a point, into y[N]
void sh_row(const Tables &T, const P3 &pt, int P, double *y)
{
  Sph s = cart2sph(pt);
  vec Y;
  sph_harm(T, s.theta, s.phi, P, Y);
  for (int i = 0; i < P * P; i++) y[i] = Y[i];
}

// IMat of one sphere: the Gram of the harmonics over the exposed (or buried) points,
// the Simpson-weighted m = 0 pairs, and the scaling of build_IMatE
void imat_one(const Tables &T, int P, int k, int n_sph, const double *cen, const double *rad,
              const std::vector<P3> &unit, double *IM)
{
  const int N = P * P, n_points = unit.size();
  std::vector<int> neigh;
  for (int j = 0; j < n_sph; j++) {
    if (j == k) continue;
    const double sr = rad[k] + rad[j];
    const double dx = cen[3 * k] - cen[3 * j], dy = cen[3 * k + 1] - cen[3 * j + 1], dz = cen[3 * k + 2] - cen[3 * j + 2];
    if (dx * dx + dy * dy + dz * dz < sr * sr) neigh.push_back(j);
  }
  std::vector<P3> E, B;
  for (int i = 0; i < n_points; i++) {
    const P3 p = rad[k] * unit[i];
    bool buried = false;
    for (int j : neigh) {
      const double dx = (p.x + cen[3 * k]) - cen[3 * j], dy = (p.y + cen[3 * k + 1]) - cen[3 * j + 1],
                   dz = (p.z + cen[3 * k + 2]) - cen[3 * j + 2];
      if (dx * dx + dy * dy + dz * dz < rad[j] * rad[j] * 1.0) { buried = true; break; }
    }
    (buried ? B : E).push_back(p);
  }
  const bool use_buried = !(E.size() <= B.size());
  const std::vector<P3> &pts = use_buried ? B : E;
  const int K = pts.size();
  std::vector<double> G((size_t)N * N, 0.0), Gs((size_t)P * P, 0.0);
  const int HC = 128;                 // points per chunk (the chunk's harmonics stay in L2)
  std::vector<double> Y((size_t)HC * N);
  for (int h0 = 0; h0 < K; h0 += HC) {
    const int hc = K - h0 < HC ? K - h0 : HC;
    for (int h = 0; h < hc; h++) sh_row(T, pts[h0 + h], P, Y.data() + (size_t)h * N);
    // upper triangle of the Gram in 4 x 8 register tiles
    for (int i0 = 0; i0 < N; i0 += 4) {
      const int ni = N - i0 < 4 ? N - i0 : 4;
      for (int j0 = i0 - i0 % 8; j0 < N; j0 += 8) {
        const int nj = N - j0 < 8 ? N - j0 : 8;
        double acc[4][8] = {};
        if (ni == 4 && nj == 8) {
          // 4 x 8 outer products held in eight 4-wide registers
          __m256d c00 = _mm256_setzero_pd(), c01 = c00, c10 = c00, c11 = c00, c20 = c00, c21 = c00, c30 = c00,
                  c31 = c00;
          const double *y = Y.data();
          for (int h = 0; h < hc; h++, y += N) {
            const __m256d b0 = _mm256_loadu_pd(y + j0), b1 = _mm256_loadu_pd(y + j0 + 4);
            __m256d a = _mm256_broadcast_sd(y + i0);
            c00 = _mm256_fmadd_pd(a, b0, c00); c01 = _mm256_fmadd_pd(a, b1, c01);
            a = _mm256_broadcast_sd(y + i0 + 1);
            c10 = _mm256_fmadd_pd(a, b0, c10); c11 = _mm256_fmadd_pd(a, b1, c11);
            a = _mm256_broadcast_sd(y + i0 + 2);
            c20 = _mm256_fmadd_pd(a, b0, c20); c21 = _mm256_fmadd_pd(a, b1, c21);
            a = _mm256_broadcast_sd(y + i0 + 3);
            c30 = _mm256_fmadd_pd(a, b0, c30); c31 = _mm256_fmadd_pd(a, b1, c31);
          }
          _mm256_storeu_pd(acc[0], c00); _mm256_storeu_pd(acc[0] + 4, c01);
          _mm256_storeu_pd(acc[1], c10); _mm256_storeu_pd(acc[1] + 4, c11);
          _mm256_storeu_pd(acc[2], c20); _mm256_storeu_pd(acc[2] + 4, c21);
          _mm256_storeu_pd(acc[3], c30); _mm256_storeu_pd(acc[3] + 4, c31);
        } else {
          for (int h = 0; h < hc; h++) {
            const double *y = Y.data() + (size_t)h * N;
            for (int a = 0; a < ni; a++)
              for (int b = 0; b < nj; b++) acc[a][b] += y[i0 + a] * y[j0 + b];
          }
        }
        for (int a = 0; a < ni; a++)
          for (int b = 0; b < nj; b++) G[(size_t)(i0 + a) * N + j0 + b] += acc[a][b];
      }
    }
    // Simpson-weighted m = 0 pairs: 1/3 at the first point, then 2/3 (even) / 4/3 (odd)
    for (int h = 0; h < hc; h++) {
      const long hh = h0 + h;
      const double w = (hh > 0) ? ((hh % 2 == 0) ? 2.0 / 3.0 : 4.0 / 3.0) : 1.0 / 3.0;
      const double *y = Y.data() + (size_t)h * N;
      for (int n = 0; n < P; n++)
        for (int l = 0; l < P; l++) Gs[n * P + l] += w * y[IDX(n)] * y[IDX(l)];
    }
  }
  const double dA = 4 * M_PI / (double)(n_points - 1);
  for (int col = 0; col < N; col++)
    for (int row = 0; row < N; row++) {
      int n = (int)sqrt((double)row);
      while (n * n > row) n--;
      while ((n + 1) * (n + 1) <= row) n++;
      int l = (int)sqrt((double)col);
      while (l * l > col) l--;
      while ((l + 1) * (l + 1) <= col) l++;
      const int mr = row - n * n, mc = col - l * l;
      const int m = (mr + 1) / 2, s = (mc + 1) / 2;
      const bool rim = (mr > 0 && mr % 2 == 0), cim = (mc > 0 && mc % 2 == 0);
      // the Gram is kept in its upper triangle (and the 8-wide tiles that cross it)
      double v = (col >= row - row % 8) ? G[(size_t)row * N + col] : G[(size_t)col * N + row];
      if (m == 0 && s == 0 && (n + l) % 2 == 0) v = Gs[n * P + l];
      double y;
      if (!use_buried) y = v * dA;
      else if (n == l && m == s) {
        const double delta = 1.0 / T.CONST2[l];
        if (rim == cim) y = ((m == 0) ? delta : 0.5 * delta) - dA * v;
        else y = v * (-dA);
      } else y = v * (-dA);
      const double c = (s == 0) ? 1.0 : 2.0;
      IM[(size_t)col * N + row] = (c * T.CONST2[n]) * y;
    }
}

double round8(double x)   // 8 significant digits as the reference writes .exp files
{
  if (fabs(x) < 1e-15) return 0.0;
  char buf[64];
  snprintf(buf, sizeof buf, "%.8g", x);
  return atof(buf);
}

}  // namespace

// IMats of a molecule's spheres: imats[n_sph][p^2 * p^2] column-major, the content
// of imat.sp<k>.out.bin.  Spheres are spread over the threads.
extern "C" int pbsam_prep_imat(int poles, int n_sph, const double *centres, const double *radii, int n_points,
                               double *imats)
{
  if (poles < 1 || n_sph < 1 || n_points < 3) return -1;
  Tables T;
  T.init(poles, 0.0);
  std::vector<double> cr(3 * n_sph), rc(3, 0.0);
  for (int k = 0; k < n_sph; k++) for (int d = 0; d < 3; d++) rc[d] += centres[3 * k + d];
  for (int d = 0; d < 3; d++) rc[d] *= 1.0 / n_sph;
  for (int k = 0; k < n_sph; k++) for (int d = 0; d < 3; d++) cr[3 * k + d] = centres[3 * k + d] - rc[d];
  std::vector<P3> unit;
  unit_spiral(n_points, unit);
  const size_t N2 = (size_t)poles * poles * poles * poles;
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < n_sph; k++) imat_one(T, poles, k, n_sph, cr.data(), radii, unit, imats + (size_t)k * N2);
  return 0;
}

// Self-polarization of one molecule from its charges and IMats; outputs rounded as
// the .exp files are written: fself/hself[n_sph][p^2], hself_scale[n_sph].
extern "C" int pbsam_prep_selfpol(int poles, double salt, double idiel, int n_sph, const double *centres,
                                  const double *radii, int n_chg, const double *chg_pos, const double *chg,
                                  const double *imats, int max_rounds, double *fself, double *hself,
                                  double *hself_scale, int *rounds)
{
  if (poles < 1 || n_sph < 1 || max_rounds < 1) return -1;
  System sys;
  sys.prm.salt = salt;
  sys.prm.idiel = idiel;
  sys.NP = poles;
  sys.T.init(poles, kappa_of_salt(salt, sys.prm.sdiel, sys.prm.temperature));
  const Tables &T = sys.T;
  const int NP = poles, NP2 = NP * NP;
  std::vector<P3> pos(n_chg), cen(n_sph);
  std::vector<double> ch(chg, chg + n_chg), rad(radii, radii + n_sph);
  for (int q = 0; q < n_chg; q++) pos[q] = P3(chg_pos[3 * q], chg_pos[3 * q + 1], chg_pos[3 * q + 2]);
  for (int k = 0; k < n_sph; k++) cen[k] = P3(centres[3 * k], centres[3 * k + 1], centres[3 * k + 2]);
  MolType mt;
  mt.ns = n_sph;
  mt.sph.assign(n_sph, SphType());
  for (int k = 0; k < n_sph; k++) {
    SphType &S = mt.sph[k];
    S.imat.assign(imats + (size_t)k * NP2 * NP2, imats + (size_t)(k + 1) * NP2 * NP2);
    S.Fself.assign(NP2, 0.0);
    S.Hself.assign(NP2, 0.0);
    S.hself_scale = 1.0 / rad[k];
  }
  init_moltype(T, sys.prm, mt, pos, ch, rad, cen, false);
  // multipole of the charges assigned to each sphere (the first sphere that contains
  // the charge, src/molecule.cpp:1001-1023; CExpCenter::setFixedCharges,
  // src/expcenter.cpp:88-103): the starting H of the self-polarization
  std::vector<vec> Eass(n_sph, vec(NP2, 0.0));
  for (int q = 0; q < n_chg; q++) {
    const P3 pr = pos[q] - mt.rcen;
    for (int k = 0; k < n_sph; k++) {
      const P3 ap = pr - mt.sph[k].cen;
      if (sqrt(ap.norm2()) + 0.0 <= mt.sph[k].rad) {
        if (ch[q] != 0.0) add_multipole_charge(T, Eass[k], ch[q] / idiel, ap, false, NP, mt.sph[k].rad);
        break;
      }
    }
  }
  sys.types.push_back(mt);
  sys.add_molecule(0);
  sys.set_pose(0, P3(0, 0, 0), Quat());
  Molecule &M = sys.mols[0];
  for (int k = 0; k < n_sph; k++) {
    SphState &Z = M.s[k];
    Z.H = Eass[k];
    Z.F.assign(NP2, 0.0);
    Z.LS.assign(NP2, 0.0);
    Z.qF.assign(sys.types[0].sph[k].spx.size(), 0.0);
    Z.qH.assign(sys.types[0].sph[k].spx.size(), 0.0);
    sys.surface_charges(0, k);
    Z.dev = 0.0;
  }
  // the sweeps of polarize_self: every sphere, then those whose last change was
  // above a tenth of the largest (all of them every fifth sweep)
  const double tol2 = sys.prm.max_polar_dev * sys.prm.max_polar_dev;
  double maxdev = 0.0;
  for (int k = 0; k < n_sph; k++) {
    sys.reexpand_intra_near(0, k);
    const vec F = M.s[k].F, H = M.s[k].H;
    const double d = sys.solve_surface(0, k, F, H, false);
    if (maxdev < d) maxdev = d;
  }
  int ct = 1;
  while (maxdev > tol2 && ct < max_rounds) {
    double mn = 0.0;
    for (int k = 0; k < n_sph; k++) {
      double d = M.s[k].dev;
      if (d > 0.1 * maxdev || ct % 5 == 0) {
        sys.reexpand_intra_near(0, k);
        const vec F = M.s[k].F, H = M.s[k].H;
        d = sys.solve_surface(0, k, F, H, false);
      }
      if (mn < d) mn = d;
    }
    maxdev = mn;
    ct++;
  }
  for (int k = 0; k < n_sph; k++) {
    const vec F = trunc_or_pad(M.s[k].F, NP), H = trunc_or_pad(M.s[k].H, NP);
    for (int i = 0; i < NP2; i++) { fself[(size_t)k * NP2 + i] = round8(F[i]); hself[(size_t)k * NP2 + i] = round8(H[i]); }
    hself_scale[k] = round8(1.0 / rad[k]);
  }
  if (rounds) *rounds = ct;
  return 0;
}
