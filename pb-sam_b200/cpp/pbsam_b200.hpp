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
// Header-only; link with pb-sam_b200/lib/libpbsam_b200.so.  The solver state the
// reference keeps in its molecules lives in one device system per list of
// molecules (created by initMutualConstants, or by the first computeForces on
// that list), so repeated calls on the same list carry the state between calls as
// the reference does.  Errors are reported the reference's way (false / -1), with
// the library's message on stderr; nothing exits the process.
#pragma once
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
    return check(pbsam_context_create(&prm, device, &ctx()));
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
