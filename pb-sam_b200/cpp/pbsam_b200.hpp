// C++ host layer over the C ABI (include/pbsam_b200.h) with the names and
// argument meaning of the reference's classes on the force path, so a driver
// written against PB-SAM's CSystem / CMolecule (src/system.h, src/molecule.h)
// runs its force calls on the GPU with the same calls:
//
//   CSystem::initConstants(kappa, sdiel, temp)          src/system.h:19-20
//   CMolecule::loadMolType(pqr, imatdir, expdir, name)   the per-species set-up of
//                                                        CBDnam::CBDnam, src/BDnam.cpp:59-119
//   new CMolecule(type, pos, orient)                     src/molecule.h:67-77
//   CMolecule::initMutualConstants(mols, 10, 100, true)  src/molecule.h:87-88
//   mol->setPos / setOrient / translate / rotate         src/molecule.h:325-329
//   CMolecule::computeForces(mols, force, torque)        src/molecule.h:179 (false on overlap)
//   CMolecule::computeTotalIntEnergy(mols)               src/molecule.h:180
//
// and the expansion classes a driver uses around them: CExpan / CMulExpan /
// CLocalExpan (src/expansion.h:96-494), CGradExpan (src/triexpan.h:253), CRotCoeff
// (src/rotcoeff.h:10-266), CTransCoeff (src/transcoeff.h:9-182) and CXFormA
// (src/xforms.h:58-104): host containers of packed expansions whose rotations,
// translations and re-expansions run on the GPU through pbsam_expan_* (each call one
// item; the *Batch functions send many at once).
// Header-only; link with pb-sam_b200/lib/libpbsam_b200.so.  The solver state the
// reference keeps in its molecules lives in one device system per list of
// molecules (created by initMutualConstants, or by the first computeForces on
// that list), so repeated calls on the same list carry the state between calls as
// the reference does.  Errors are reported the reference's way (false / -1), with
// the library's message on stderr; nothing exits the process.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <vector>

#include "pbsam_b200.h"

class CPnt {
 public:
  CPnt() : m_x(0), m_y(0), m_z(0) {}
  CPnt(double x, double y, double z) : m_x(x), m_y(y), m_z(z) {}
  double x() const { return m_x; }
  double y() const { return m_y; }
  double z() const { return m_z; }
  double norm() const { return std::sqrt(m_x * m_x + m_y * m_y + m_z * m_z); }
  CPnt operator+(const CPnt &o) const { return CPnt(m_x + o.m_x, m_y + o.m_y, m_z + o.m_z); }
  CPnt operator-(const CPnt &o) const { return CPnt(m_x - o.m_x, m_y - o.m_y, m_z - o.m_z); }
  friend CPnt operator*(double s, const CPnt &p) { return CPnt(s * p.m_x, s * p.m_y, s * p.m_z); }

 private:
  double m_x, m_y, m_z;
};

// unit quaternion (real, imag) as CQuat (src/util.h:205-298)
class CQuat {
 public:
  CQuat() : m_real(1.0), m_imag() {}
  CQuat(double real, const CPnt &imag) : m_real(real), m_imag(imag)
  {
    const double in = 1.0 / std::sqrt(imag.x() * imag.x() + imag.y() * imag.y() + imag.z() * imag.z() + real * real);
    m_real *= in;
    m_imag = in * m_imag;
  }
  double real() const { return m_real; }
  const CPnt &imag() const { return m_imag; }
  // q1 * q2 (src/util.h:254-262), no normalization
  friend CQuat operator*(const CQuat &a, const CQuat &b)
  {
    CQuat q;
    const CPnt &u = a.m_imag, &v = b.m_imag;
    q.m_real = a.m_real * b.m_real - (u.x() * v.x() + u.y() * v.y() + u.z() * v.z());
    q.m_imag = CPnt(a.m_real * v.x() + b.m_real * u.x() + (u.y() * v.z() - u.z() * v.y()),
                    a.m_real * v.y() + b.m_real * u.y() + (u.z() * v.x() - u.x() * v.z()),
                    a.m_real * v.z() + b.m_real * u.z() + (u.x() * v.y() - u.y() * v.x()));
    return q;
  }

 private:
  double m_real;
  CPnt m_imag;
};

// The solver context: CSystem's constants (kappa, solvent dielectric,
// temperature) plus what the reference fixes at compile time (pole order,
// tolerances) or per molecule (interior dielectric).
class CSystem {
 public:
  // kappa in 1/A as the reference's drivers compute it from the salt concentration
  // (src/BDnam_main.cpp:53-55); the context is created from the equivalent salt.
  static bool initConstants(double kappa, double sdiel, double temp, int poles = 10, double idiel = 4.0,
                            int device = 0)
  {
    clear();
    pbsam_params prm;
    pbsam_params_default(&prm);
    const double AVO = 6.0221415e23, ECHG = 1.60217646e-19, EPS0 = 8.854187817e-12;
    const double KBOLTZ = 1.3806503e-23, ANG = 1e-10, LIT = 1e-3;
    const double k = kappa / ANG;
    prm.salt = k * k * (sdiel * EPS0 * KBOLTZ * temp) / (2 * AVO / LIT * ECHG * ECHG);
    prm.sdiel = sdiel;
    prm.temperature = temp;
    prm.poles = poles;
    prm.idiel = idiel;
    const double *t = tolerances();
    prm.max_polar_dev = t[0]; prm.solve_tol = t[1]; prm.solve_max_ct = (int)t[2]; prm.max_pol_rounds = (int)t[3];
    polesRef() = poles;
    return check(pbsam_context_create(&prm, device, &ctx()));
  }
  // the context's pole order (the reference's N_POLES)
  static int poles() { return polesRef(); }
  static int &polesRef()
  {
    static int p = 10;
    return p;
  }
  // The reference's compile-time tolerances MAX_POLAR_DEV, SOLVE_TOL, SOLVE_MAX_CT,
  // MAX_POL_ROUNDS (src/molecule.cpp:6-13, src/expcenter.cpp:16-22); set before initConstants.
  static void setTolerances(double max_polar_dev, double solve_tol, int solve_max_ct, int max_pol_rounds)
  {
    double *t = tolerances();
    t[0] = max_polar_dev; t[1] = solve_tol; t[2] = solve_max_ct; t[3] = max_pol_rounds;
  }
  static double *tolerances()
  {
    static double t[4] = {1e-2, 1e-8, 100, 1000};
    return t;
  }
  static double getKappa()
  {
    double k = 0.0;
    check(pbsam_context_kappa(ctx(), &k));
    return k;
  }
  static pbsam_context *&ctx()
  {
    static pbsam_context *c = nullptr;
    return c;
  }
  static void clear();
  static bool check(int rc)
  {
    if (rc == PBSAM_OK) return true;
    std::fprintf(stderr, "pbsam-b200: %s\n", pbsam_last_error());
    return false;
  }
};

class CMolecule {
 public:
  // the per-species set-up of the BD driver: PQR, imat.sp<k>.out.bin, <name>.<k>.{F,H}.exp
  static int loadMolType(const char *pqr, const char *imatdir, const char *expdir, const char *expname)
  {
    int t = -1;
    return CSystem::check(pbsam_moltype_load(CSystem::ctx(), pqr, imatdir, expdir, expname, &t)) ? t : -1;
  }

  explicit CMolecule(int moltype, const CPnt &pos = CPnt(), const CQuat &orient = CQuat())
      : m_type(moltype), m_rcen(pos), m_orient(orient) {}

  int getMolType() const { return m_type; }
  const CPnt &getRCen() const { return m_rcen; }
  const CQuat &getOrient() const { return m_orient; }
  void setPos(const CPnt &p) { m_rcen = p; }
  void setOrient(const CQuat &q) { m_orient = q; }
  void translate(const CPnt &d) { m_undo = m_rcen; m_rcen = m_rcen + d; }
  void untranslate() { m_rcen = m_undo; }
  // m_orient *= dQ (src/moldynamics.cpp:666-679): dQ applied after the current orientation
  void rotate(const CQuat &dQ) { m_orient = dQ * m_orient; }

  // The reference sets its cutoff statics here; the context carries them, so the
  // call checks they agree and prepares the device system of this list.
  static bool initMutualConstants(std::vector<CMolecule *> &mols, double interRCutoff, double interactRCutoff,
                                  bool bGrad)
  {
    if (!bGrad || interRCutoff != 10.0 || interactRCutoff != 100.0) {
      std::fprintf(stderr, "pbsam-b200: the context was created with cutoffs 10 / 100 and gradients on\n");
      return false;
    }
    return system_of(mols) != nullptr;
  }

  // CMolecule::computeForces: false when two molecules overlap (src/molecule.cpp:1090-1097)
  // or the evaluation is not finite; a sweep loop that stopped at its cap returns true
  // with the forces, as the reference does after printing its warning
  static bool computeForces(std::vector<CMolecule *> &mols, std::vector<CPnt> &force, std::vector<CPnt> &torque)
  {
    pbsam_system *s = system_of(mols);
    if (!s || !set_poses(s, mols)) return false;
    const size_t n = mols.size();
    std::vector<double> f(3 * n), t(3 * n);
    int status = 0;
    if (!CSystem::check(pbsam_system_compute_forces(s, f.data(), t.data(), &status, 0))) return false;
    force.assign(n, CPnt());
    torque.assign(n, CPnt());
    if (status != PBSAM_SYS_OK && status != PBSAM_SYS_NOT_CONVERGED) return false;
    for (size_t i = 0; i < n; i++) {
      force[i] = CPnt(f[3 * i], f[3 * i + 1], f[3 * i + 2]);
      torque[i] = CPnt(t[3 * i], t[3 * i + 1], t[3 * i + 2]);
    }
    return true;
  }

  // CMolecule::computeTotalIntEnergy on the state of the last computeForces of this list
  static double computeTotalIntEnergy(std::vector<CMolecule *> &mols)
  {
    pbsam_system *s = system_of(mols);
    double e = 0.0;
    if (!s || !CSystem::check(pbsam_system_compute_energy(s, &e, 0))) return NAN;
    return e;
  }

  static std::map<std::vector<const CMolecule *>, pbsam_system *> &systems()
  {
    static std::map<std::vector<const CMolecule *>, pbsam_system *> m;
    return m;
  }

 private:
  static pbsam_system *system_of(const std::vector<CMolecule *> &mols)
  {
    std::vector<const CMolecule *> key(mols.begin(), mols.end());
    auto it = systems().find(key);
    if (it != systems().end()) return it->second;
    std::vector<int> types;
    for (const CMolecule *m : mols) types.push_back(m->m_type);
    pbsam_system *s = nullptr;
    if (!CSystem::check(pbsam_system_create(CSystem::ctx(), 1, (int)types.size(), types.data(), &s))) return nullptr;
    systems()[key] = s;
    return s;
  }
  static bool set_poses(pbsam_system *s, const std::vector<CMolecule *> &mols)
  {
    std::vector<double> pos, quat;
    for (const CMolecule *m : mols) {
      pos.push_back(m->m_rcen.x()); pos.push_back(m->m_rcen.y()); pos.push_back(m->m_rcen.z());
      quat.push_back(m->m_orient.real()); quat.push_back(m->m_orient.imag().x());
      quat.push_back(m->m_orient.imag().y()); quat.push_back(m->m_orient.imag().z());
    }
    return CSystem::check(pbsam_system_set_poses(s, pos.data(), quat.data(), 0));
  }

  int m_type;
  CPnt m_rcen, m_undo;
  CQuat m_orient;
};

// releases every device system and the context
inline void CSystem::clear()
{
  for (auto &kv : CMolecule::systems()) pbsam_system_destroy(kv.second);
  CMolecule::systems().clear();
  if (ctx()) pbsam_context_destroy(ctx());
  ctx() = nullptr;
}

// ---------------------------------------------------------------- expansions
// Packed real expansion of degrees < p (entries n^2, n^2 + 2m - 1, n^2 + 2m: the
// m = 0 term, then Re and Im of m = 1..n) with its scale, as CExpan.
class CExpan {
 public:
  explicit CExpan(int p = 0, double scale = 1.0) : m_scale(scale), m_c((size_t)p * p, 0.0) {}
  CExpan(const std::vector<double> &c, double scale) : m_scale(scale), m_c(c)
  {
    const int p = order();
    m_c.resize((size_t)p * p, 0.0);
  }
  int order() const { return (int)std::lround(std::sqrt((double)m_c.size())); }   // getRange().p2()
  double getScale() const { return m_scale; }
  void setScale(double s) { m_scale = s; }
  void setOrder(int p) { m_c.resize((size_t)p * p, 0.0); }                        // setRange(p)
  double &operator[](int i) { return m_c[i]; }
  double operator[](int i) const { return m_c[i]; }
  const std::vector<double> &coeffs() const { return m_c; }
  // range union, as CExpan::operator+= (src/expansion.h:509-560)
  CExpan &operator+=(const CExpan &o)
  {
    if (o.m_c.size() > m_c.size()) m_c.resize(o.m_c.size(), 0.0);
    for (size_t i = 0; i < o.m_c.size(); i++) m_c[i] += o.m_c[i];
    return *this;
  }
  CExpan &operator-=(const CExpan &o)
  {
    if (o.m_c.size() > m_c.size()) m_c.resize(o.m_c.size(), 0.0);
    for (size_t i = 0; i < o.m_c.size(); i++) m_c[i] -= o.m_c[i];
    return *this;
  }
  CExpan &operator*=(double s)
  {
    for (double &v : m_c) v *= s;
    return *this;
  }
  // the coefficients zero-padded to the context's pole order (the C ABI's layout)
  std::vector<double> padded(int NP) const
  {
    std::vector<double> v((size_t)NP * NP, 0.0);
    for (size_t i = 0; i < m_c.size() && i < v.size(); i++) v[i] = m_c[i];
    return v;
  }
  void assign(const double *v, int p, double scale)
  {
    m_c.assign(v, v + (size_t)p * p);
    m_scale = scale;
  }

 protected:
  double m_scale;
  std::vector<double> m_c;
};
class CMulExpan : public CExpan {   // multipole: M-scale
 public:
  using CExpan::CExpan;
};
class CLocalExpan : public CExpan {  // local: L-scale
 public:
  using CExpan::CExpan;
};
// x, y, z derivatives of an expansion (CGradExpan)
class CGradExpan {
 public:
  CExpan &operator[](int c) { return m_e[c]; }
  const CExpan &operator[](int c) const { return m_e[c]; }

 private:
  CExpan m_e[3];
};

// <M, L> with the scales of a multipole and a local expansion: sum over n of
// (1 / (M scale * L scale))^n times the degree-n products, the m > 0 terms twice
// (inprod, src/expansion.h:706-741)
inline double inprod(const CExpan &M, const CExpan &L)
{
  const int p = std::min(M.order(), L.order());
  const double fact = 1.0 / (M.getScale() * L.getScale());
  double sum = 0.0, scale = 1.0;
  for (int n = 0; n < p; n++) {
    double s = 0.0;
    for (int mm = 1; mm < 2 * n + 1; mm++) s += M[n * n + mm] * L[n * n + mm];
    sum += scale * (2.0 * s + M[n * n] * L[n * n]);
    scale *= fact;
  }
  return sum;
}


// Rotation of expansions by Euler angles (theta, phi, xi).
class CRotCoeff {
 public:
  CRotCoeff() : m_p(0), m_a{0.0, 0.0, 0.0} {}
  void reset(double theta, double phi, double xi, int p) { m_a[0] = theta; m_a[1] = phi; m_a[2] = xi; m_p = p; }
  void reset(const CQuat &Q, int p)
  {
    const double q[4] = {Q.real(), Q.imag().x(), Q.imag().y(), Q.imag().z()};
    CSystem::check(pbsam_quat_angles(q, m_a));
    m_p = p;
  }
  int getOrder() const { return m_p; }
  // rotate (src/rotcoeff.cpp:357-441); the output keeps the input's scale
  bool rotate(const CExpan &Min, CExpan &Mout, bool bFor) const { return apply(Min, Mout, bFor, 0); }
  // rotateWithXi (src/rotcoeff.cpp:250-350), for molecule rotations
  bool rotateWithXi(const CExpan &Min, CExpan &Mout, bool bFor) const { return apply(Min, Mout, bFor, 1); }
  // many expansions, each with its own rotation
  static bool rotateBatch(const std::vector<CRotCoeff> &rot, const std::vector<CExpan> &in, std::vector<CExpan> &out,
                          bool bFor, bool withXi = false)
  {
    const int NP = CSystem::poles(), n = (int)in.size();
    if ((int)rot.size() != n || n == 0) return n == 0;
    int p = NP;
    std::vector<double> a, x, y((size_t)n * NP * NP);
    for (int i = 0; i < n; i++) {
      p = std::min(p, std::min(rot[i].m_p, in[i].order()));
      a.insert(a.end(), rot[i].m_a, rot[i].m_a + 3);
      const std::vector<double> v = in[i].padded(NP);
      x.insert(x.end(), v.begin(), v.end());
    }
    if (!CSystem::check(pbsam_expan_rotate(CSystem::ctx(), n, a.data(), p, withXi, bFor, x.data(), y.data(), 0)))
      return false;
    out.assign(n, CExpan());
    for (int i = 0; i < n; i++) out[i].assign(y.data() + (size_t)i * NP * NP, p, in[i].getScale());
    return true;
  }

 private:
  bool apply(const CExpan &Min, CExpan &Mout, bool bFor, int withXi) const
  {
    const int NP = CSystem::poles(), p = std::min(m_p, Min.order());
    const std::vector<double> x = Min.padded(NP);
    std::vector<double> y((size_t)NP * NP);
    if (!CSystem::check(pbsam_expan_rotate(CSystem::ctx(), 1, m_a, p, withXi, bFor, x.data(), y.data(), 0)))
      return false;
    Mout.assign(y.data(), p, Min.getScale());
    return true;
  }
  int m_p;
  double m_a[3];
};

// Coaxial translation along z by rho: screened by the context's kappa or unscreened
// (kappa = 0), from scale_in to scale_out.
class CTransCoeff {
 public:
  CTransCoeff() : m_rho(0.0), m_screened(1), m_p(0), m_si(1.0), m_so(1.0) {}
  // reset(rho, kappa, p, scalei, scaleo): kappa must be the context's or 0
  bool reset(double rho, double kappa, int p, double scalei, double scaleo)
  {
    const double k = CSystem::getKappa();
    if (kappa != 0.0 && std::fabs(kappa - k) > 1e-12 * k) {
      std::fprintf(stderr, "pbsam-b200: translations are screened by the context's kappa or not at all\n");
      return false;
    }
    m_rho = rho; m_screened = kappa != 0.0; m_p = p; m_si = scalei; m_so = scaleo;
    return true;
  }
  // translate (src/transcoeff.cpp:211-286; tpose is not supported there either)
  bool translate(const CExpan &Min, CExpan &Mout, bool tpose = false) const { return apply(Min, Mout, tpose, 0); }
  // dTranslate (src/transcoeff.cpp:294-364)
  bool dTranslate(const CExpan &Min, CExpan &Mout, bool tpose = false) const { return apply(Min, Mout, tpose, 1); }

 private:
  bool apply(const CExpan &Min, CExpan &Mout, bool tpose, int deriv) const
  {
    if (tpose) {
      std::fprintf(stderr, "pbsam-b200: transposed translation is not supported (src/transcoeff.cpp:216-218)\n");
      return false;
    }
    const int NP = CSystem::poles(), p = std::min(m_p, Min.order());
    const double a[3] = {m_rho, m_si, m_so};
    const std::vector<double> x = Min.padded(NP);
    std::vector<double> y((size_t)NP * NP);
    if (!CSystem::check(pbsam_expan_translate(CSystem::ctx(), 1, a, p, m_screened, deriv, x.data(), y.data(), 0)))
      return false;
    Mout.assign(y.data(), p, m_so);
    return true;
  }
  double m_rho;
  int m_screened, m_p;
  double m_si, m_so;
};

// Re-expansion of a source sphere's multipole into a local expansion about a target
// sphere (CXFormA(source, target)): the spheres' radii are the scales.
class CXFormA {
 public:
  CXFormA(double radSource, double radTarget) : m_rs(radSource), m_rt(radTarget), m_P(), m_p(0) {}
  // reset(P, p), P = target centre - source centre
  void reset(const CPnt &P, int p) { m_P = P; m_p = p; }
  // xformH (screened; src/xforms.cpp:122-132)
  bool xformH(const CExpan &Min, CExpan &Mout) const { return apply(Min, Mout, nullptr, 1); }
  // xformH with its gradient w.r.t. the target position (src/xforms.cpp:85-115)
  bool xformH(const CExpan &Min, CExpan &Mout, CGradExpan &G) const { return apply(Min, Mout, &G, 1); }
  // xformF (unscreened; src/xforms.cpp:260-270)
  bool xformF(const CExpan &Min, CExpan &Mout) const { return apply(Min, Mout, nullptr, 0); }

 private:
  bool apply(const CExpan &Min, CExpan &Mout, CGradExpan *G, int screened) const
  {
    const int NP = CSystem::poles(), p = std::min(m_p, Min.order());
    const double a[5] = {m_P.x(), m_P.y(), m_P.z(), m_rs, m_rt};
    const std::vector<double> x = Min.padded(NP);
    std::vector<double> y((size_t)NP * NP), g(G ? 3 * (size_t)NP * NP : 0);
    if (!CSystem::check(pbsam_expan_reexpand(CSystem::ctx(), 1, a, p, screened, x.data(), y.data(),
                                             G ? g.data() : nullptr, 0)))
      return false;
    Mout.assign(y.data(), p, m_rt);
    if (G)
      for (int c = 0; c < 3; c++) (*G)[c].assign(g.data() + (size_t)c * NP * NP, p, m_rt);
    return true;
  }
  double m_rs, m_rt;
  CPnt m_P;
  int m_p;
};
