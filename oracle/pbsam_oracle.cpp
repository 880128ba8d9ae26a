// CPU restatement of PB-SAM's mutual-polarization solve and force/torque
// evaluation -- TEST ORACLE ONLY.
//
// This file is test infrastructure: only tests/, the smoke check and the
// bench's CPU-baseline leg may load it, and only to check or time the CUDA
// drop-in.  It restates, in plain FP64 C++, the algorithm of the reference's
// CMolecule::computeForces (src/moldynamics.cpp:553-587) including its
// Gauss-Seidel sweep schedule, selective re-polarization and stopping rules, so
// that at the reference's tolerances it reproduces the reference's output.  It
// is pinned against outputs of the reference itself (tests/golden/*/ref_*),
// produced by oracle/ref_harness.cpp built with oracle/build_ref.py.
//
// Layout conventions (src/expansion.h:509-553): an expansion of p degrees is a
// packed real array of p*p doubles; degree n occupies [n*n, n*n + 2n], entry
// 0 is the m=0 coefficient and entries 2m-1, 2m are Re and Im of m>0.
// All arithmetic is FP64.  The pole order p is a runtime value here (a
// compile-time macro N_POLES in the reference, src/expansion.h:5-9).
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <array>
#include <algorithm>
#include <string>
#include <vector>

namespace orc {

typedef std::complex<double> cplx;
typedef std::vector<double> vec;

struct P3 {
  double x, y, z;
  P3() : x(0), y(0), z(0) {}
  P3(double a, double b, double c) : x(a), y(b), z(c) {}
  P3 operator+(const P3 &o) const { return P3(x + o.x, y + o.y, z + o.z); }
  P3 operator-(const P3 &o) const { return P3(x - o.x, y - o.y, z - o.z); }
  P3 operator-() const { return P3(-x, -y, -z); }
  double norm2() const { return x * x + y * y + z * z; }
  double norm() const { return sqrt(norm2()); }
};
static inline P3 operator*(double s, const P3 &p) { return P3(s * p.x, s * p.y, s * p.z); }
static inline double dot(const P3 &a, const P3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline P3 cross(const P3 &a, const P3 &b)
{ return P3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

// quaternion (src/util.h:199-298, 442-476)
struct Quat {
  double w; P3 v;
  Quat() : w(1), v() {}
  Quat(double w_, P3 v_) : w(w_), v(v_) { double in = 1.0 / sqrt(v.norm2() + w * w); v = in * v; w *= in; }
};
static inline P3 qrot(const Quat &q, const P3 &r)   // CQuat * CPnt (src/util.h:463-468)
{ P3 qr = cross(q.v, r); return r + 2 * (q.w * qr + cross(q.v, qr)); }
static inline Quat qconj(const Quat &q) { return Quat(q.w, -q.v); }

struct Sph { double rho, theta, phi; };
static inline Sph cart2sph(const P3 &c)             // src/util.h:418-438
{
  Sph s;
  s.rho = sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
  if (s.rho < fabs(c.z)) s.rho = fabs(c.z);
  s.theta = (s.rho == 0.0) ? 0.0 : acos(c.z / s.rho);
  s.phi = (c.x == 0.0 && c.y == 0.0) ? 0.0 : atan2(c.y, c.x);
  return s;
}

// ---------------------------------------------------------------------------
// Constant tables (src/expansion.cpp:39-96, src/rotcoeff.cpp:15-33,
// src/transcoeff.cpp:15-38, src/expcenter.cpp:186-210).  NP = pole order.
struct Tables {
  int NP;
  double kappa;                 // global inverse Debye length
  std::vector<double> C1, C2, C3, C5, C6, C4;   // [2NP][2NP] flattened for C1..C3
  std::vector<double> zeta, eta;               // zeta[n][m] (m<=2NP), eta[n][m+2NP-1]
  std::vector<double> alpha, beta, gam, del;   // [2NP][NP], [2NP][2NP-1]
  std::vector<double> Q;                       // m_Q[2NP-1][NP][2]
  std::vector<double> CONST2, CONST3;          // (2l+1)/4pi, 1/(2l+1)
  double c1(int n, int m) const { return C1[n * 2 * NP + m]; }
  double c2(int n, int m) const { return C2[n * 2 * NP + m]; }
  double c3(int n, int m) const { return C3[n * 2 * NP + m]; }
  double &ZETA(int n, int m) { return zeta[n * (2 * NP) + m]; }
  double ZETA(int n, int m) const { return zeta[n * (2 * NP) + m]; }
  double &ETA(int n, int m) { return eta[n * (4 * NP - 1) + 2 * NP - 1 + m]; }
  double ETA(int n, int m) const { return eta[n * (4 * NP - 1) + 2 * NP - 1 + m]; }
  double &ALPHA(int n, int m) { return alpha[n * NP + m]; }
  double ALPHA(int n, int m) const { return alpha[n * NP + m]; }
  double &BETA(int n, int m) { return beta[n * NP + m]; }
  double BETA(int n, int m) const { return beta[n * NP + m]; }
  double &GAMMA(int n, int m) { return gam[n * (2 * NP - 1) + NP - 1 + m]; }
  double GAMMA(int n, int m) const { return gam[n * (2 * NP - 1) + NP - 1 + m]; }
  double &DELTA(int n, int m) { return del[n * (2 * NP - 1) + NP - 1 + m]; }
  double DELTA(int n, int m) const { return del[n * (2 * NP - 1) + NP - 1 + m]; }
  double &MQ(int n, int m, int k) { return Q[(n * NP + m) * 2 + k]; }
  double MQ(int n, int m, int k) const { return Q[(n * NP + m) * 2 + k]; }

  void init(int np, double kap);
};

static void specialSH(const Tables &T, std::vector<double> &SH, int n, double val)  // src/expansion.cpp:527-546
{
  SH.assign(n, 0.0);
  if (n > 0) SH[0] = 0;
  if (n > 1) SH[1] = -1;
  if (n > 2) SH[2] = -val * 3;
  for (int l = 3; l < n; l++) SH[l] = (val * (2 * l - 1) * SH[l - 1] - l * SH[l - 2]) / (l - 1);
  for (int l = 1; l < n; l++) SH[l] *= (-T.c3(l, 1));
}

void Tables::init(int np, double kap)
{
  NP = np; kappa = kap;
  const int N2 = 2 * NP;
  C1.assign(N2 * N2, 0.0); C2.assign(N2 * N2, 0.0); C3.assign(N2 * N2, 0.0);
  C5.assign(N2, 0.0); C6.assign(N2, 0.0); C4.assign(N2, 0.0);
  std::vector<double> temp(4 * NP);
  temp[0] = 1.0;
  for (int i = 1; i < 4 * NP; i++) temp[i] = temp[i - 1] * sqrt((double)i);
  for (int n = 0; n < N2; n++) {
    for (int m = 0; m <= n; m++) {
      C1[n * N2 + m] = (2 * n - 1) / (double)(n - m);
      C2[n * N2 + m] = (n + m - 1) / (double)(n - m);
      C3[n * N2 + m] = temp[n - m] / temp[n + m];
    }
    C5[n] = (double)((2 * n + 1) * (2 * n + 3));
  }
  C6[0] = 1.0; C6[1] = 1.0;
  for (int n = 2; n < N2; n++) C6[n] = C6[n - 1] * (2 * n - 1);
  for (int n = 0; n < N2; n++) C4[n] = 1.0 / ((2 * n - 1) * (2 * n - 3));
  // rotation constants (src/rotcoeff.cpp:15-33); zeta padded to 2NP columns
  zeta.assign(N2 * N2, 0.0); eta.assign(N2 * (4 * NP - 1), 0.0);
  for (int n = 0; n < N2; n++)
    for (int m = 0; m <= n; m++) ZETA(n, m) = sqrt((double)(n + m + 1) * (n - m + 1) / ((2 * n + 1) * (2 * n + 3)));
  for (int n = 0; n < N2; n++)
    for (int m = 0; m <= n; m++) {
      ETA(n, m) = sqrt((double)(n - m - 1) * (n - m) / ((2 * n + 1) * (2 * n - 1)));
      if (m != 0) ETA(n, -m) = -sqrt((double)(n + m - 1) * (n + m) / ((2 * n + 1) * (2 * n - 1)));
    }
  // Q coefficients for singular dR (src/rotcoeff.cpp:949-983)
  Q.assign((2 * NP - 1) * NP * 2, 0.0);
  {
    std::vector<double> SH;
    specialSH(*this, SH, 2 * NP - 1, 1.0);
    for (int n = 1; n < 2 * NP - 1; n++) { MQ(n, 0, 0) = 0.0; MQ(n, 0, 1) = SH[n]; }
    for (int n = 2; n < 2 * NP - 1; n++) {
      MQ(n - 1, 1, 0) = (ETA(n, -1) * MQ(n, 0, 1) + ZETA(n - 1, 0)) / ETA(n, 0);
      MQ(n - 1, 1, 1) = (n > 2) ? (ETA(n, 1) / ETA(n, 0)) * MQ(n, 0, 1) : 0.0;
    }
    for (int m = 1; m < NP - 1; m++)
      for (int n = m + 2; n < 2 * NP - m - 1; n++) {
        MQ(n - 1, m + 1, 0) = (ETA(n, m - 1) * MQ(n, m, 0) + ZETA(n - 1, m)) / ETA(n, m);
        MQ(n - 1, m + 1, 1) = (n > m + 2) ? (ETA(n, m + 1) / ETA(n, m)) * MQ(n, m, 1) : 0.0;
      }
  }
  // translation constants (src/transcoeff.cpp:15-38)
  alpha.assign(N2 * NP, 0.0); beta.assign(N2 * NP, 0.0);
  gam.assign(N2 * (2 * NP - 1), 0.0); del.assign(N2 * (2 * NP - 1), 0.0);
  const double kapsqr = (kappa == 0 ? 0 : 1.0);
  for (int n = 0; n < N2; n++)
    for (int m = 0; m < NP; m++) {
      ALPHA(n, m) = sqrt((double)(n + m + 1) * (n - m + 1));
      BETA(n, m) = kapsqr * ALPHA(n, m) / ((2 * n + 1) * (2 * n + 3));
      GAMMA(n, m) = sqrt((double)(n - m - 1) * (n - m));
      DELTA(n, m) = kapsqr * GAMMA(n, m) / ((2 * n + 1) * (2 * n - 1));
      if (m != 0) {
        GAMMA(n, -m) = -sqrt((double)(n + m - 1) * (n + m));
        DELTA(n, -m) = kapsqr * GAMMA(n, -m) / ((2 * n + 1) * (2 * n - 1));
      }
    }
  CONST2.assign(NP, 0.0); CONST3.assign(NP, 0.0);
  for (int l = 0; l < NP; l++) { CONST2[l] = (2 * l + 1) / (4.0 * M_PI); CONST3[l] = 1 / (double)(2 * l + 1); }
}

static inline int IDX(int n) { return n * n; }

// ---------------------------------------------------------------------------
// Spherical harmonics (src/expansion.cpp:482-518, 634-675): P degrees.
static void sph_harm(const Tables &T, double theta, double phi, int P, vec &M)
{
  M.assign(P * P, 0.0);
  double negterm = 1.0;
  const double cost = cos(theta), sint = sin(theta);
  double sqrtterm = 1.0;
  M[0] = T.C6[0];
  negterm = -negterm;
  sqrtterm *= sint;
  if (P > 1) {
    M[IDX(1)] = cost * M[0];
    for (int n = 2; n < P; n++)
      M[IDX(n)] = cost * T.c1(n, 0) * M[IDX(n - 1)] - T.c2(n, 0) * M[IDX(n - 2)];
  }
  for (int m = 1, k = 1; m < P; m++, k += 2) {
    M[IDX(m) + k] = negterm * T.C6[m] * sqrtterm;
    M[IDX(m) + k + 1] = M[IDX(m) + k];
    negterm = -negterm;
    sqrtterm *= sint;
    if (m < P - 1) {
      M[IDX(m + 1) + k] = cost * (2 * m + 1) * M[IDX(m) + k];
      M[IDX(m + 1) + k + 1] = M[IDX(m + 1) + k];
      for (int n = m + 2; n < P; n++) {
        M[IDX(n) + k] = cost * T.c1(n, m) * M[IDX(n - 1) + k] - T.c2(n, m) * M[IDX(n - 2) + k];
        M[IDX(n) + k + 1] = M[IDX(n) + k];
      }
    }
  }
  std::vector<double> cosp(P), sinp(P);
  double ang = 0;
  for (int m = 0; m < P; m++, ang += phi) { cosp[m] = cos(ang); sinp[m] = sin(ang); }
  int it = 0;
  for (int n = 0; n < P; n++) {
    M[it++] *= T.c3(n, 0);
    double s = -1.0;
    for (int m = 1; m <= n; m++, s = -s) {
      M[it++] *= s * T.c3(n, m) * cosp[m];
      M[it++] *= s * T.c3(n, m) * sinp[m];
    }
  }
}

static inline cplx comp(const vec &M, int n, int m)   // src/expansion.h:521-536 (ISQRT2 = 1)
{
  if (m == 0) return cplx(M[IDX(n)], 0.0);
  int i = IDX(n) + 2 * abs(m) - 1;
  return (m > 0) ? cplx(M[i], M[i + 1]) : cplx(M[i], -M[i + 1]);
}

// modified spherical Bessel k-hat by upward recurrence (src/expansion.cpp:421-436)
static void bessel_k(const Tables &T, std::vector<double> &K, double val)
{
  if (val != 0.0 && K.size() > 1) {
    K[1] += val;
    const double valsqr = val * val;
    for (size_t n = 2; n < K.size(); n++) K[n] = K[n - 1] + valsqr * K[n - 2] * T.C4[n];
  }
}
// modified spherical Bessel i-hat by series (src/expansion.cpp:347-365)
static void bessel_i(std::vector<double> &K, double val)
{
  if (val != 0.0) {
    const double z = 0.5 * val * val;
    for (size_t n = 0; n < K.size(); n++) {
      double t = z / (2 * n + 3);
      for (int j = 1; j <= 20; j++) {
        K[n] += t;
        t *= (z / ((j + 1) * (2 * (n + j) + 3)));
        if (t < 1e-20) break;
      }
    }
  }
}

// single-charge local expansion added into L (CLExpan, src/expansion.h:467-494,
// src/expansion.cpp:289-316, 409-436); L holds P degrees.
static void add_local_charge(const Tables &T, vec &L, double ch, const P3 &pos, bool bKappa, int P,
                             double scale, double weight = 1.0)
{
  Sph s = cart2sph(pos);
  vec Y; sph_harm(T, s.theta, s.phi, P, Y);
  double val = bKappa ? s.rho * T.kappa : 0.0;
  std::vector<double> bes(P + 1, 1.0);
  bessel_k(T, bes, val);
  double r = 1.0 / s.rho;
  double k = ch * r * (bKappa ? exp(-val) : 1.0);
  r *= scale;
  int it = 0;
  for (int n = 0; n < P; n++) {
    for (int m = 0; m < 2 * n + 1; m++, it++) Y[it] *= (bes[n] * k);
    k *= r;
  }
  if ((int)L.size() < P * P) L.resize(P * P, 0.0);
  for (int i = 0; i < P * P; i++) L[i] += weight * Y[i];
}
// single-charge multipole expansion (CMExpan, src/expansion.cpp:323-365)
static void add_multipole_charge(const Tables &T, vec &M, double ch, const P3 &pos, bool bKappa, int P,
                                 double scale)
{
  Sph s = cart2sph(pos);
  vec Y; sph_harm(T, s.theta, s.phi, P, Y);
  double val = bKappa ? s.rho * T.kappa : 0.0;
  std::vector<double> bes(P + 1, 1.0);
  bessel_i(bes, val);
  double mscale = 1.0 / scale;
  double r = s.rho * mscale;
  double k = ch;
  int it = 0;
  for (int n = 0; n < P; n++) {
    for (int m = 0; m < 2 * n + 1; m++, it++) Y[it] *= (bes[n] * k);
    k *= r;
  }
  if ((int)M.size() < P * P) M.resize(P * P, 0.0);
  for (int i = 0; i < P * P; i++) M[i] += Y[i];
}

static void add_into(vec &a, const vec &b)     // CExpan::operator+= (range union)
{
  if (a.size() < b.size()) a.resize(b.size(), 0.0);
  for (size_t i = 0; i < b.size(); i++) a[i] += b[i];
}
static inline int degs(const vec &a) { return (int)lround(sqrt((double)a.size())); }

// inner product without scale factors (src/expansion.h:783-803)
static double inprod_unit(const vec &E1, const vec &E2)
{
  int P = std::min(degs(E1), degs(E2));
  double sum = 0.0;
  for (int n = 0; n < P; n++) {
    double s = 0.0;
    for (int mm = 1; mm < 2 * n + 1; mm++) s += E1[IDX(n) + mm] * E2[IDX(n) + mm];
    s *= 2.0;
    s += E1[IDX(n)] * E2[IDX(n)];
    sum += s;
  }
  return sum;
}
// multipole-local inner product with scale bookkeeping (src/expansion.h:705-741)
static double inprod_ml(const vec &M, double mscale, const vec &L, double lscale)
{
  int P = std::min(degs(M), degs(L));
  double sum = 0.0, fact = 1 / (mscale * lscale), scale = 1.0;
  for (int n = 0; n < P; n++) {
    double s = 0.0;
    for (int mm = 1; mm < 2 * n + 1; mm++) s += M[IDX(n) + mm] * L[IDX(n) + mm];
    s *= 2.0;
    s += M[IDX(n)] * L[IDX(n)];
    sum += scale * s;
    scale *= fact;
  }
  return sum;
}

// ---------------------------------------------------------------------------
// Rotation coefficients (src/rotcoeff.cpp:154-244, 779-850)
struct Rot {
  const Tables *T;
  int p;
  bool grad, sing;
  double theta, phi, xi, sint, cost, cott;
  cplx exphi, exiphi, exxi;
  std::vector<cplx> R, dR;       // [n][n+s][m], n < 2p-1, m <= n
  std::vector<int> off;
  int at(int n, int s, int m) const { return off[n] + (n + s) * (n + 1) + m; }
  const cplx &ROT(int n, int s, int m) const { return R[at(n, s, m)]; }
  const cplx &dROT(int n, int s, int m) const { return dR[at(n, s, m)]; }

  void reset(const Tables &TT, double th, double ph, double x, int pp, bool bGrad)
  {
    T = &TT; p = pp; grad = bGrad;
    theta = th; phi = ph; xi = x;
    sint = sin(theta);
    if (sint < 1e-12) {
      sing = true;
      if (theta < M_PI / 2) { theta = 0.0; phi = 0.0; sint = 0.0; cost = 1.0; exphi = cplx(1.0, 0.0); }
      else { theta = M_PI; phi = 0.0; sint = 0.0; cost = -1.0; exphi = cplx(1.0, 0.0); }
    } else {
      sing = false;
      cost = cos(theta);
      cott = cost / sint;
      exphi = cplx(cos(ph), sin(ph));
    }
    exiphi = std::conj(exphi);
    exxi = cplx(cos(x), sin(x));
    const int NN = 2 * p - 1;
    off.assign(NN + 1, 0);
    for (int n = 0; n < NN; n++) off[n + 1] = off[n] + (2 * n + 1) * (n + 1);
    R.assign(off[NN], cplx(0, 0));
    if (grad) dR.assign(off[NN], cplx(0, 0));
    if (sing) return;
    vec SH; sph_harm(TT, theta, phi, NN, SH);
    // computeCoeff
    R[at(0, 0, 0)] = comp(SH, 0, 0);
    for (int n = 1; n < NN; n++) {
      R[at(n, 0, 0)] = comp(SH, n, 0);
      for (int s = 1; s <= n; s++) { R[at(n, s, 0)] = comp(SH, n, -s); R[at(n, -s, 0)] = comp(SH, n, s); }
    }
    const double r1 = -0.5 * (1 + cost), r2 = 0.5 * (1 - cost), r3 = -sint;
    for (int m = 0; m < p - 1; m++)
      for (int n = m + 2; n < 2 * p - m - 1; n++)
        for (int s = -n + 1; s < n; s++) {
          cplx d1 = (r1 * TT.ETA(n, s - 1)) * R[at(n, s - 1, m)];
          cplx d2 = (r2 * TT.ETA(n, -s - 1)) * R[at(n, s + 1, m)];
          cplx d3 = (r3 * TT.ZETA(n - 1, abs(s))) * R[at(n, s, m)];
          R[at(n - 1, s, m + 1)] = exxi * (d1 * exiphi + d2 * exphi + d3) / TT.ETA(n, m);
        }
    if (!grad) return;
    // computeGradCoeff
    dR[at(0, 0, 0)] = cplx(0.0, 0.0);
    for (int n = 1; n < NN; n++) {
      dR[at(n, 0, 0)] = -sqrt((double)n * (n + 1)) * exiphi * comp(SH, n, 1);
      for (int s = 1; s < n; s++) {
        dR[at(n, -s, 0)] = (s * cott) * comp(SH, n, s) - sqrt((double)(n - s) * (n + s + 1)) * exiphi * comp(SH, n, s + 1);
        dR[at(n, s, 0)] = std::conj(dR[at(n, -s, 0)]);
      }
      dR[at(n, -n, 0)] = (n * cott) * comp(SH, n, n);
      dR[at(n, n, 0)] = std::conj(dR[at(n, -n, 0)]);
    }
    const double dr1 = 0.5 * sint, dr2 = dr1, dr3 = -cost;
    for (int m = 0; m < p - 1; m++)
      for (int n = m + 2; n < 2 * p - m - 1; n++)
        for (int s = -n + 1; s < n; s++) {
          cplx d1 = TT.ETA(n, s - 1) * (r1 * dR[at(n, s - 1, m)] + dr1 * R[at(n, s - 1, m)]);
          cplx d2 = TT.ETA(n, -s - 1) * (r2 * dR[at(n, s + 1, m)] + dr2 * R[at(n, s + 1, m)]);
          cplx d3 = TT.ZETA(n - 1, abs(s)) * (r3 * dR[at(n, s, m)] + dr3 * R[at(n, s, m)]);
          dR[at(n - 1, s, m + 1)] = exxi * (d1 * exiphi + d2 * exphi + d3) / TT.ETA(n, m);
        }
  }
  // molecule rotation from a quaternion (src/rotcoeff.cpp:180-201)
  void reset_quat(const Tables &TT, const Quat &Qt, int pp)
  {
    double th = acos(1.0 - 2 * Qt.v.x * Qt.v.x - 2 * Qt.v.y * Qt.v.y);
    double ph, x;
    if (fabs(th) > 1e-12) {
      ph = atan2(Qt.v.y * Qt.v.z + Qt.w * Qt.v.x, Qt.v.x * Qt.v.z - Qt.w * Qt.v.y);
      x = atan2(Qt.v.y * Qt.v.z - Qt.w * Qt.v.x, Qt.v.x * Qt.v.z + Qt.w * Qt.v.y);
    } else { th = 0.0; ph = 0.0; x = 2 * acos(Qt.w); }
    reset(TT, th, ph, x, pp, false);
  }

  // rotate (src/rotcoeff.cpp:356-441): out has p2 degrees
  void rotate(const vec &Min, vec &Mout, int p2, bool bFor) const
  {
    Mout.assign(p2 * p2, 0.0);
    if (sing) {
      if (cost == -1.0) {
        for (int n = 0; n < p2; n++) {
          Mout[IDX(n)] = (n % 2 == 0 ? Min[IDX(n)] : -Min[IDX(n)]);
          int s = (n % 2 == 0 ? 1 : -1);
          for (int m = 1; m < 2 * n + 1; m++, s = -s) Mout[IDX(n) + m] = s * Min[IDX(n) + m];
        }
      } else {
        for (int n = 0; n < p2; n++)
          for (int m = 0; m < 2 * n + 1; m++) Mout[IDX(n) + m] = Min[IDX(n) + m];
      }
      return;
    }
    if (bFor) {
      for (int n = 0; n < p2; n++)
        for (int m = 0; m <= n; m++) {
          cplx inc(Min[IDX(n)], 0.0);
          cplx out = ROT(n, 0, m) * inc;
          for (int s = 1; s <= n; s++) {
            inc = cplx(Min[IDX(n) + 2 * s - 1], Min[IDX(n) + 2 * s]);
            out += (ROT(n, s, m) * inc + ROT(n, -s, m) * std::conj(inc));
          }
          if (m == 0) Mout[IDX(n)] = out.real();
          else { Mout[IDX(n) + 2 * m - 1] = out.real(); Mout[IDX(n) + 2 * m] = out.imag(); }
        }
    } else {
      for (int n = 0; n < p2; n++)
        for (int s = 0; s <= n; s++) {
          cplx inc(Min[IDX(n)], 0.0);
          cplx out = ROT(n, -s, 0) * inc;
          for (int m = 1; m <= n; m++) {
            inc = cplx(Min[IDX(n) + 2 * m - 1], Min[IDX(n) + 2 * m]);
            out += std::conj(ROT(n, s, m)) * inc + ROT(n, -s, m) * std::conj(inc);
          }
          if (s == 0) Mout[IDX(n)] = out.real();
          else { Mout[IDX(n) + 2 * s - 1] = out.real(); Mout[IDX(n) + 2 * s] = out.imag(); }
        }
    }
  }
  // rotateWithXi (src/rotcoeff.cpp:249-350)
  void rotate_xi(const vec &Min, vec &Mout, int p2, bool bFor) const
  {
    if (!sing) { rotate(Min, Mout, p2, bFor); return; }
    Mout.assign(p2 * p2, 0.0);
    const double x = bFor ? xi : -xi;
    if (cost == -1.0) {
      for (int n = 0; n < p2; n++) {
        Mout[IDX(n)] = (n % 2 == 0 ? Min[IDX(n)] : -Min[IDX(n)]);
        int s = (n % 2 == 0 ? 1 : -1);
        for (int m = 1; m <= n; m++) {
          cplx inc(Min[IDX(n) + 2 * m - 1], Min[IDX(n) + 2 * m]);
          cplx e(cos(m * x), sin(m * x));
          cplx out = e * inc;
          Mout[IDX(n) + 2 * m - 1] = s * out.real();
          Mout[IDX(n) + 2 * m] = -s * out.imag();
        }
      }
    } else {
      for (int n = 0; n < p2; n++) {
        Mout[IDX(n)] = Min[IDX(n)];
        for (int m = 1; m <= n; m++) {
          cplx inc(Min[IDX(n) + 2 * m - 1], Min[IDX(n) + 2 * m]);
          cplx e(cos(m * x), sin(m * x));
          cplx out = e * inc;
          Mout[IDX(n) + 2 * m - 1] = out.real();
          Mout[IDX(n) + 2 * m] = out.imag();
        }
      }
    }
  }
  static cplx derv(const cplx &c, int s) { return cplx(-s * c.imag(), s * c.real()); }
  // singular dR/dtheta (src/rotcoeff.cpp:616-691)
  void dRotTSing(const vec &Min, vec &Mout, int p2) const
  {
    int p1 = 1;
    Mout[0] = 0.0; p1++;
    if (cost == 1.0) {
      for (int n = p1 - 1; n < p2; n++) {
        Mout[IDX(n)] = 2.0 * T->MQ(n, 0, 1) * Min[IDX(n) + 1];
        for (int m = 1; m < n; m++) {
          cplx i0 = (m == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (m - 1) - 1], Min[IDX(n) + 2 * (m - 1)]);
          cplx i1(Min[IDX(n) + 2 * (m + 1) - 1], Min[IDX(n) + 2 * (m + 1)]);
          cplx o = T->MQ(n, m, 0) * i0 + T->MQ(n, m, 1) * i1;
          Mout[IDX(n) + 2 * m - 1] = o.real(); Mout[IDX(n) + 2 * m] = o.imag();
        }
        cplx i0 = (n == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (n - 1) - 1], Min[IDX(n) + 2 * (n - 1)]);
        cplx o = T->MQ(n, n, 0) * i0;
        Mout[IDX(n) + 2 * n - 1] = o.real(); Mout[IDX(n) + 2 * n] = o.imag();
      }
    } else {
      double s = -1.0;
      for (int n = p1 - 1; n < p2; n++, s = -s) {
        Mout[IDX(n)] = 2.0 * s * T->MQ(n, 0, 1) * Min[IDX(n) + 1];
        for (int m = 1; m < n; m++) {
          cplx i0 = (m == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (m - 1) - 1], Min[IDX(n) + 2 * (m - 1)]);
          cplx i1(Min[IDX(n) + 2 * (m + 1) - 1], Min[IDX(n) + 2 * (m + 1)]);
          cplx o = s * (T->MQ(n, m, 0) * std::conj(i0) + T->MQ(n, m, 1) * std::conj(i1));
          Mout[IDX(n) + 2 * m - 1] = o.real(); Mout[IDX(n) + 2 * m] = o.imag();
        }
        cplx i0 = (n == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (n - 1) - 1], Min[IDX(n) + 2 * (n - 1)]);
        cplx o = s * T->MQ(n, n, 0) * std::conj(i0);
        Mout[IDX(n) + 2 * n - 1] = o.real(); Mout[IDX(n) + 2 * n] = o.imag();
      }
    }
  }
  // singular dR/dphi (src/rotcoeff.cpp:703-771)
  void dRotPSing(const vec &Min, vec &Mout, int p2) const
  {
    int p1 = 1;
    Mout[0] = 0.0; p1++;
    if (cost == 1.0) {
      for (int n = p1 - 1; n < p2; n++) {
        Mout[IDX(n)] = 2.0 * T->MQ(n, 0, 1) * Min[IDX(n) + 2];
        for (int m = 1; m < n; m++) {
          cplx i0 = (m == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (m - 1) - 1], Min[IDX(n) + 2 * (m - 1)]);
          cplx i1(Min[IDX(n) + 2 * (m + 1) - 1], Min[IDX(n) + 2 * (m + 1)]);
          cplx o = cplx(0.0, T->MQ(n, m, 0)) * i0 - cplx(0.0, T->MQ(n, m, 1)) * i1;
          Mout[IDX(n) + 2 * m - 1] = o.real(); Mout[IDX(n) + 2 * m] = o.imag();
        }
        cplx i0 = (n == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (n - 1) - 1], Min[IDX(n) + 2 * (n - 1)]);
        cplx o = cplx(0.0, T->MQ(n, n, 0)) * i0;
        Mout[IDX(n) + 2 * n - 1] = o.real(); Mout[IDX(n) + 2 * n] = o.imag();
      }
    } else {
      double s = 1.0;
      for (int n = p1 - 1; n < p2; n++, s = -s) {
        Mout[IDX(n)] = s * 2 * T->MQ(n, 0, 1) * Min[IDX(n) + 2];
        for (int m = 1; m < n; m++) {
          cplx i0 = (m == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (m - 1) - 1], Min[IDX(n) + 2 * (m - 1)]);
          cplx i1(Min[IDX(n) + 2 * (m + 1) - 1], Min[IDX(n) + 2 * (m + 1)]);
          cplx o = s * (cplx(0.0, T->MQ(n, m, 1)) * std::conj(i1) - cplx(0.0, T->MQ(n, m, 0)) * std::conj(i0));
          Mout[IDX(n) + 2 * m - 1] = o.real(); Mout[IDX(n) + 2 * m] = o.imag();
        }
        cplx i0 = (n == 1) ? cplx(Min[IDX(n)], 0.0) : cplx(Min[IDX(n) + 2 * (n - 1) - 1], Min[IDX(n) + 2 * (n - 1)]);
        cplx o = cplx(0.0, -s * T->MQ(n, n, 0)) * std::conj(i0);
        Mout[IDX(n) + 2 * n - 1] = o.real(); Mout[IDX(n) + 2 * n] = o.imag();
      }
    }
  }
  // dRotateT (src/rotcoeff.cpp:449-522)
  void dRotT(const vec &Min, vec &Mout, int p2, bool bFor) const
  {
    Mout.assign(p2 * p2, 0.0);
    if (sing) {
      dRotTSing(Min, Mout, p2);
      if (!bFor) for (auto &v : Mout) v = -v;
      return;
    }
    if (bFor) {
      for (int n = 0; n < p2; n++)
        for (int m = 0; m <= n; m++) {
          cplx inc(Min[IDX(n)], 0.0);
          cplx out = dROT(n, 0, m) * inc;
          for (int s = 1; s <= n; s++) {
            inc = cplx(Min[IDX(n) + 2 * s - 1], Min[IDX(n) + 2 * s]);
            out += (dROT(n, s, m) * inc + dROT(n, -s, m) * std::conj(inc));
          }
          if (m == 0) Mout[IDX(n)] = out.real();
          else { Mout[IDX(n) + 2 * m - 1] = out.real(); Mout[IDX(n) + 2 * m] = out.imag(); }
        }
    } else {
      for (int n = 0; n < p2; n++)
        for (int s = 0; s <= n; s++) {
          cplx inc(Min[IDX(n)], 0.0);
          cplx out = dROT(n, -s, 0) * inc;
          for (int m = 1; m <= n; m++) {
            inc = cplx(Min[IDX(n) + 2 * m - 1], Min[IDX(n) + 2 * m]);
            out += std::conj(dROT(n, s, m)) * inc + dROT(n, -s, m) * std::conj(inc);
          }
          if (s == 0) Mout[IDX(n)] = out.real();
          else { Mout[IDX(n) + 2 * s - 1] = out.real(); Mout[IDX(n) + 2 * s] = out.imag(); }
        }
    }
  }
  // dRotateP (src/rotcoeff.cpp:530-606)
  void dRotP(const vec &Min, vec &Mout, int p2, bool bFor) const
  {
    Mout.assign(p2 * p2, 0.0);
    if (sing) {
      dRotPSing(Min, Mout, p2);
      if (!bFor && cost == 1.0) for (auto &v : Mout) v = -v;
      return;
    }
    if (bFor) {
      for (int n = 0; n < p2; n++)
        for (int m = 0; m <= n; m++) {
          cplx out(0.0, 0.0);
          for (int s = 1; s <= n; s++) {
            cplx inc(Min[IDX(n) + 2 * s - 1], Min[IDX(n) + 2 * s]);
            out -= (ROT(n, s, m) * derv(inc, s) + ROT(n, -s, m) * derv(std::conj(inc), -s));
          }
          if (m == 0) Mout[IDX(n)] = out.real();
          else { Mout[IDX(n) + 2 * m - 1] = out.real(); Mout[IDX(n) + 2 * m] = out.imag(); }
        }
    } else {
      for (int n = 0; n < p2; n++)
        for (int s = 0; s <= n; s++) {
          cplx inc(Min[IDX(n)], 0);
          cplx out = ROT(n, -s, 0) * derv(inc, s);
          for (int m = 1; m <= n; m++) {
            inc = cplx(Min[IDX(n) + 2 * m - 1], Min[IDX(n) + 2 * m]);
            out += std::conj(ROT(n, s, m)) * derv(inc, s) + ROT(n, -s, m) * derv(std::conj(inc), s);
          }
          if (s == 0) Mout[IDX(n)] = out.real();
          else { Mout[IDX(n) + 2 * s - 1] = out.real(); Mout[IDX(n) + 2 * s] = out.imag(); }
        }
    }
  }
};

// ---------------------------------------------------------------------------
// Coaxial translation coefficients (src/transcoeff.cpp:150-449)
struct Trans {
  int p;
  bool grad;
  double scalei, scaleo;
  std::vector<double> fact;
  std::vector<double> Tc, dTc;     // [l][n][m], n<=l, m<=l
  std::vector<int> off;
  int at(int l, int n, int m) const { return off[l] + n * (l + 1) + m; }
  double TR(int l, int n, int m) const { return Tc[at(l, n, m)]; }
  double dTR(int l, int n, int m) const { return dTc[at(l, n, m)]; }

  void init_scale(int NP, double si, double so)        // src/transcoeff.cpp:194-203
  {
    scalei = si; scaleo = so;
    fact.assign(NP, 0.0);
    fact[0] = 1.0;
    for (int n = 1; n < NP; n++) fact[n] = fact[n - 1] * (scaleo / scalei);
  }
  void recur(const Tables &TT, std::vector<double> &U)   // computeCoeff_ (src/transcoeff.cpp:402-449)
  {
    const double kappasqr = TT.kappa * TT.kappa;     // global kappa, also for kappa = 0 transforms
    const double kpio = kappasqr * scalei * scaleo;
    const double kpoo = kappasqr * scaleo * scaleo;
    const double o_i = scaleo / scalei;
    auto u = [&](int l, int n, int m) -> double & { return U[at(l, n, m)]; };
    for (int l = 1; l < 2 * p - 2; l++)
      u(l, 1, 0) = -(kpio * TT.BETA(l - 1, 0) * u(l - 1, 0, 0) + o_i * TT.ALPHA(l, 0) * u(l + 1, 0, 0)) / TT.ALPHA(0, 0);
    for (int n = 1; n < p - 1; n++)
      for (int l = n + 1; l < 2 * p - 2 - n; l++)
        u(l, n + 1, 0) = -(kpio * TT.BETA(l - 1, 0) * u(l - 1, n, 0) + kpoo * TT.BETA(n - 1, 0) * u(l, n - 1, 0) +
                           o_i * TT.ALPHA(l, 0) * u(l + 1, n, 0)) / TT.ALPHA(n, 0);
    for (int m = 1; m < p; m++) {
      for (int l = m; l < 2 * p - 1 - m; l++)
        u(l, m, m) = -(kpio * TT.DELTA(l, -m) * u(l - 1, m - 1, m - 1) + o_i * TT.GAMMA(l + 1, m - 1) * u(l + 1, m - 1, m - 1)) /
                     TT.GAMMA(m, -m);
      int n = m;
      for (int l = n + 1; l < 2 * p - 2 - n; l++)
        u(l, n + 1, m) = -(kpio * TT.BETA(l - 1, m) * u(l - 1, n, m) + o_i * TT.ALPHA(l, m) * u(l + 1, n, m)) / TT.ALPHA(n, m);
      for (n = m + 1; n < p - 1; n++)
        for (int l = n + 1; l < 2 * p - 2 - n; l++)
          u(l, n + 1, m) = -(kpio * TT.BETA(l - 1, m) * u(l - 1, n, m) + kpoo * TT.BETA(n - 1, m) * u(l, n - 1, m) +
                             o_i * TT.ALPHA(l, m) * u(l + 1, n, m)) / TT.ALPHA(n, m);
    }
  }
  void reset(const Tables &TT, double d, double kap, int pp, bool bGrad)   // src/transcoeff.cpp:150-185, 371-395
  {
    p = pp; grad = bGrad;
    const int NL = 2 * p - 1;
    off.assign(NL + 1, 0);
    for (int l = 0; l < NL; l++) off[l + 1] = off[l] + (l + 1) * (l + 1);
    Tc.assign(off[NL], 0.0);
    if (grad) dTc.assign(off[NL], 0.0);
    const double kd = kap * d;
    double ir = 0, exkid = 0;
    if (d > 0.0) { ir = 1.0 / d; exkid = exp(-kd) * ir; }
    std::vector<double> K(2 * p, 1.0);
    bessel_k(TT, K, kd);
    Tc[at(0, 0, 0)] = exkid * K[0];
    exkid *= ir;
    if (grad) dTc[at(0, 0, 0)] = -exkid * K[1];
    exkid *= scalei;
    for (int l = 1; l < 2 * p - 1; l++) {
      Tc[at(l, 0, 0)] = exkid * K[l];
      exkid *= ir;
      if (grad) dTc[at(l, 0, 0)] = exkid * (l * K[l] - (2 * l + 1) * K[l + 1]);
      exkid *= scalei;
    }
    recur(TT, Tc);
    if (grad) recur(TT, dTc);
  }
  // forward translate (src/transcoeff.cpp:210-286, tpose = false)
  void translate(const vec &Min, vec &Mout, bool deriv) const
  {
    auto C = [&](int l, int n, int m) { return deriv ? dTR(l, n, m) : TR(l, n, m); };
    Mout.assign(p * p, 0.0);
    for (int n = 0; n < p; n++) {
      int l;
      for (l = 0; l <= n; l++) {
        double t = ((n + l) % 2 == 0) ? C(n, l, 0) : -C(n, l, 0);
        Mout[IDX(n)] += fact[n - l] * t * Min[IDX(l)];
      }
      for (; l < p; l++) Mout[IDX(n)] += C(l, n, 0) * Min[IDX(l)];
      for (int m = 1; m <= n; m++) {
        for (l = m; l <= n; l++) {
          double t = ((n + l) % 2 == 0) ? C(n, l, m) : -C(n, l, m);
          Mout[IDX(n) + 2 * m - 1] += fact[n - l] * t * Min[IDX(l) + 2 * m - 1];
          Mout[IDX(n) + 2 * m] += fact[n - l] * t * Min[IDX(l) + 2 * m];
        }
        for (; l < p; l++) {
          Mout[IDX(n) + 2 * m - 1] += C(l, n, m) * Min[IDX(l) + 2 * m - 1];
          Mout[IDX(n) + 2 * m] += C(l, n, m) * Min[IDX(l) + 2 * m];
        }
      }
    }
  }
};

static inline vec trunc_or_pad(const vec &a, int P)
{
  vec b(P * P, 0.0);
  for (int i = 0; i < P * P && i < (int)a.size(); i++) b[i] = a[i];
  return b;
}

// per-pair truncation order (src/xforms.cpp:401-414), MAX_ERROR 1e-6
static int compute_order(int NP, double rho, double TQ, double scale)
{
  if (TQ < 1e-10) return 1;
  double c = rho / scale - 1;
  if (c <= 1) return NP;
  int p = int(log(TQ / (1e-6 * scale * (c - 1))) / log(c) - 1 + 0.5);
  if (p < 1) p = 1;
  if (p > NP) p = NP;
  return p;
}

// analytic re-expansion (CXFormA / CXFormAIntra, src/xforms.cpp:11-270)
struct XForm {
  Rot rot;
  Trans tH, tF;
  int pH, pF;
  P3 Rm[3];
  // CXFormA::reset (src/xforms.cpp:50-77)
  void reset(const Tables &TT, const P3 &P, int p, double scaleSrc, double scaleTgt, bool bGrad)
  {
    pH = p;
    Sph S = cart2sph(P);
    rot.reset(TT, S.theta, S.phi, M_PI, p, bGrad);
    tH.init_scale(TT.NP, scaleSrc, scaleTgt);
    tH.reset(TT, S.rho, TT.kappa, p, bGrad);
    double ir = 1.0 / S.rho;
    if (rot.sing) {
      Rm[0] = P3(0.0, ir * rot.cost, 0.0); Rm[1] = P3(0.0, 0.0, ir); Rm[2] = P3(rot.cost, 0.0, 0.0);
    } else {
      double sint = rot.sint, cost = rot.cost, sinp = rot.exphi.imag(), cosp = rot.exphi.real();
      double irst = ir / sint, irct = ir * cost;
      Rm[0] = P3(sint * cosp, irct * cosp, -irst * sinp);
      Rm[1] = P3(sint * sinp, irct * sinp, irst * cosp);
      Rm[2] = P3(cost, -ir * sint, 0.0);
    }
  }
  // CXFormAIntra::reset (src/xforms.cpp:213-227)
  void reset_intra(const Tables &TT, const P3 &P, int ph, int pf, double scaleSrc, double scaleTgt)
  {
    int maxp = ph > pf ? ph : pf;
    pH = ph; pF = pf;
    Sph S = cart2sph(P);
    rot.reset(TT, S.theta, S.phi, M_PI, maxp, false);
    tH.init_scale(TT.NP, scaleSrc, scaleTgt);
    tF.init_scale(TT.NP, scaleSrc, scaleTgt);
    tH.reset(TT, S.rho, TT.kappa, pH, false);
    tF.reset(TT, S.rho, 0.0, pF, false);
  }
  void xformH(const vec &Min, vec &Mout) const    // src/xforms.cpp:122-132
  {
    vec tM, tL;
    rot.rotate(Min, tM, pH, true);
    tH.translate(tM, tL, false);
    rot.rotate(tL, Mout, pH, false);
  }
  void xformF(const vec &Min, vec &Mout) const    // src/xforms.cpp:260-270
  {
    vec tM, tL;
    rot.rotate(Min, tM, pF, true);
    tF.translate(tM, tL, false);
    rot.rotate(tL, Mout, pF, false);
  }
  // gradient of the transformed expansion w.r.t. the target position (src/xforms.cpp:85-115, 164-192)
  void xformH_grad(const vec &Min, vec G[3]) const
  {
    const int p = pH;
    vec tM1, tL, tmp;
    rot.rotate(Min, tM1, p, true);
    tH.translate(tM1, tL, true);
    rot.rotate(tL, G[0], p, false);
    tH.translate(tM1, tL, false);
    rot.dRotT(tL, G[1], p, false);
    rot.dRotP(tL, G[2], p, false);
    rot.dRotT(Min, tM1, p, true);
    tH.translate(tM1, tL, false);
    rot.rotate(tL, tmp, p, false);
    add_into(G[1], tmp);
    rot.dRotP(Min, tM1, p, true);
    tH.translate(tM1, tL, false);
    rot.rotate(tL, tmp, p, false);
    add_into(G[2], tmp);
    for (int i = 0; i < p * p; i++) {
      P3 a(G[0][i], G[1][i], G[2][i]);
      double bx = dot(Rm[0], a), by = dot(Rm[1], a), bz = dot(Rm[2], a);
      G[0][i] = bx; G[1][i] = by; G[2][i] = bz;
    }
  }
};

// ---------------------------------------------------------------------------
// Molecule type data (moltype precompute, src/BDnam.cpp:59-136)
struct SphType {
  P3 cen;              // relative to molecule centre (molecule frame)
  double rad;
  std::vector<P3> spx; // exposed surface points relative to sphere centre
  int nspx;            // number of generated points (sets dA)
  vec Fself, Hself;    // self-polarized expansions read from .exp
  double hself_scale;  // scale value stored in the .exp file (1/rad to 8 digits)
  vec qFself, qHself;
  double tFself, tHself;
  vec LFintra, LHintra, LFfar, LHfar;
  std::vector<int> near;         // intra pol list (near)
  vec Efix, Lfix, Dfix, Vfix;
  // per-sphere constants (src/expcenter.cpp:469-505)
  vec cH1, cF1, cH2, cF2, cLH1, cLF1, cLH2, cLF2, cInvH, cChgH;
  std::vector<double> imat;      // NP^2 x NP^2 column-major
};
struct MolType {
  int ns;
  P3 rcen;
  double maxR;
  std::vector<SphType> sph;
};

// surface points: spiral (src/molecule.cpp:2272-2294), exposure test (src/molecule.cpp:948-994)
static void sphere_pts(int N, std::vector<double> &th, std::vector<double> &ph)
{
  th.assign(N, 0.0); ph.assign(N, 0.0);
  for (int i = 1; i <= N; i++) {
    double h = -1.0 + 2.0 * (i - 1.0) / (N - 1.0);
    th[i - 1] = acos(h);
    if (i == 1 || i == N) ph[i - 1] = 0;
    else ph[i - 1] = (ph[i - 2] + 3.6 / sqrt(N * (1.0 - h * h)));
    while (ph[i - 1] > 2 * M_PI) ph[i - 1] -= 2 * M_PI;
    while (ph[i - 1] < -2 * M_PI) ph[i - 1] += 2 * M_PI;
  }
}

struct Params {
  double salt = 0.05, idiel = 4.0, sdiel = 78.0, temperature = 298.15;
  double max_polar_dev = 1e-2;   // src/molecule.cpp:6
  double solve_tol = 1e-8;       // src/expcenter.cpp:17
  int solve_max_ct = 100;        // src/expcenter.cpp:18
  int max_pol_rounds = 1000;     // src/molecule.cpp:10
  double inter_cut = 10, interact_cut = 100, intra_cut = 30;
  int num_points_x = 10000;      // src/molecule.cpp:64
};

static double kappa_of_salt(double salt, double sdiel, double temp)   // src/BDnam_main.cpp:53-55
{
  const double AVO = 6.0221415e23, ECHG = 1.60217646e-19, EPS0 = 8.854187817e-12;
  const double KBOLTZ = 1.3806503e-23, ANG = 1e-10, LIT = 1e-3;
  return ANG * sqrt((2 * salt * AVO / LIT * ECHG * ECHG) / (sdiel * EPS0 * KBOLTZ * temp));
}

// ---------------------------------------------------------------------------
// file readers (formats of src/readutil.cpp:285-355, 399-435, 564-598)
static bool read_pqr(const char *fname, std::vector<P3> &pos, std::vector<double> &ch,
                     std::vector<double> &rad, std::vector<P3> &cen)
{
  FILE *f = fopen(fname, "r");
  if (!f) return false;
  char buf[512];
  while (fgets(buf, sizeof buf, f)) {
    if (strncmp(buf, "ATOM", 4) != 0) continue;
    double x, y, z, c, r;
    if (sscanf(buf + 31, "%lf %lf %lf %lf %lf", &x, &y, &z, &c, &r) != 5) continue;
    if (strncmp(buf + 18, "CEN", 3) == 0) { rad.push_back(r); cen.push_back(P3(x, y, z)); }
    else { pos.push_back(P3(x, y, z)); ch.push_back(c); }
  }
  fclose(f);
  return true;
}
static bool read_imat(const char *fname, int NP, std::vector<double> &mat)
{
  FILE *f = fopen(fname, "rb");
  if (!f) return false;
  int p = 0;
  if (fread(&p, sizeof(int), 1, f) != 1 || p < NP) { fclose(f); return false; }
  const int psq = NP * NP;
  mat.assign((size_t)psq * psq, 0.0);
  if (p == NP) {
    size_t n = fread(mat.data(), sizeof(double), (size_t)psq * psq, f);
    fclose(f);
    return n == (size_t)psq * psq;
  }
  const long matlen = (long)p * p;
  for (int j = 0; j < psq; j++) {
    if (fread(mat.data() + (size_t)j * psq, sizeof(double), psq, f) != (size_t)psq) { fclose(f); return false; }
    fseek(f, (matlen - psq) * sizeof(double), SEEK_CUR);
  }
  fclose(f);
  return true;
}
static bool read_exp(const char *fname, int NP, vec &V, double &scale)
{
  std::ifstream fin(fname);
  if (!fin) return false;
  int pr; double rcut;
  fin >> pr >> scale >> rcut;
  V.assign(NP * NP, 0.0);
  int n = (pr < NP) ? pr * pr : NP * NP;
  for (int k = 0; k < n; k++) fin >> V[k];
  return true;
}

// moltype precompute (src/molecule.cpp:501-696, 756-810, src/expcenter.cpp:469-552, 1042-1060)
static void init_moltype(const Tables &T, const Params &prm, MolType &mt, const std::vector<P3> &pos,
                         const std::vector<double> &ch, const std::vector<double> &rad, const std::vector<P3> &cen,
                         bool self_terms = true);

static bool build_moltype(const Tables &T, const Params &prm, MolType &mt, const char *pqr,
                          const char *imatdir, const char *expdir, const char *expname)
{
  const int NP = T.NP;
  std::vector<P3> pos, cen;
  std::vector<double> ch, rad;
  if (!read_pqr(pqr, pos, ch, rad, cen)) return false;
  const int ns = cen.size();
  mt.ns = ns;
  mt.sph.assign(ns, SphType());
  char fn[1024];
  for (int k = 0; k < ns; k++) {
    SphType &S = mt.sph[k];
    snprintf(fn, sizeof fn, "%s/imat.sp%d.out.bin", imatdir, k);
    if (!read_imat(fn, NP, S.imat)) return false;
    double sc;
    snprintf(fn, sizeof fn, "%s/%s.%d.F.exp", expdir, expname, k);
    if (!read_exp(fn, NP, S.Fself, sc)) return false;
    snprintf(fn, sizeof fn, "%s/%s.%d.H.exp", expdir, expname, k);
    if (!read_exp(fn, NP, S.Hself, S.hself_scale)) return false;
  }
  init_moltype(T, prm, mt, pos, ch, rad, cen);
  return true;
}

// the rest of the moltype precompute, from absolute charge positions and sphere
// centres, with each sphere's IMat and self expansions already in mt.sph;
// self_terms = false skips what depends on the self expansions (surface charges and
// intra local expansions of the self values), for a type about to be self-polarized
static void init_moltype(const Tables &T, const Params &prm, MolType &mt, const std::vector<P3> &pos,
                         const std::vector<double> &ch, const std::vector<double> &rad, const std::vector<P3> &cen,
                         bool self_terms)
{
  const int NP = T.NP;
  const int ns = cen.size();
  P3 rc;
  for (int i = 0; i < ns; i++) rc = rc + cen[i];
  rc = (1.0 / ns) * rc;
  mt.rcen = rc;
  std::vector<P3> cr(ns), posr(pos.size());
  for (int i = 0; i < ns; i++) cr[i] = cen[i] - rc;
  for (size_t i = 0; i < pos.size(); i++) posr[i] = pos[i] - rc;
  mt.maxR = 0;
  for (int i = 0; i < ns; i++) { double d = cr[i].norm() + rad[i]; if (d > mt.maxR) mt.maxR = d; }
  for (int k = 0; k < ns; k++) { mt.sph[k].cen = cr[k]; mt.sph[k].rad = rad[k]; }
  // exposed surface points (generateMolSPX / getXFormSpherePoints)
  for (int k = 0; k < ns; k++) {
    SphType &S = mt.sph[k];
    std::vector<int> neigh;
    for (int j = 0; j < ns; j++) {
      if (j == k) continue;
      double sr = rad[k] + rad[j];
      if ((cen[k] - cen[j]).norm2() < sr * sr) neigh.push_back(j);
    }
    const int Nin = prm.num_points_x;
    const double cutoff = 1.5, maxrad = 10, gradient = Nin / ((maxrad - cutoff) * (maxrad - cutoff));
    int N;
    if (rad[k] < cutoff) N = 200;
    else { N = int(200 + gradient * (rad[k] - cutoff) * (rad[k] - cutoff)); if (N > Nin) N = Nin; }
    std::vector<double> th, ph;
    sphere_pts(N, th, ph);
    S.spx.clear();
    for (int n = 0; n < N; n++) {
      P3 q(sin(th[n]) * cos(ph[n]), sin(th[n]) * sin(ph[n]), cos(th[n]));
      P3 pp = rad[k] * q;
      bool inside = false;
      for (size_t t = 0; t < neigh.size(); t++) {
        int j = neigh[t];
        if ((pp + cen[k] - cen[j]).norm2() < rad[j] * rad[j]) { inside = true; break; }
      }
      if (!inside) S.spx.push_back(pp);
    }
    S.nspx = N;
  }
  // per-sphere constants (initMyConstants)
  const double eps = prm.idiel / prm.sdiel;
  for (int k = 0; k < ns; k++) {
    SphType &S = mt.sph[k];
    std::vector<double> bK(NP + 1, 1.0), bI(NP + 1, 1.0);
    double val = T.kappa * S.rad, valsqr = val * val, exp_val = exp(-1.0 * val);
    bessel_k(T, bK, val);
    bessel_i(bI, val);
    S.cH1.assign(NP, 0); S.cF1.assign(NP, 0); S.cH2.assign(NP, 0); S.cF2.assign(NP, 0);
    S.cLH1.assign(NP, 0); S.cLF1.assign(NP, 0); S.cLH2.assign(NP, 0); S.cLF2.assign(NP, 0);
    S.cInvH.assign(NP, 0); S.cChgH.assign(NP, 0);
    for (int n = 0; n < NP; n++) {
      double DH = -exp_val * bK[n], DF = 1.0;
      double VH = exp_val * (n * bK[n] - (2 * n + 1) * bK[n + 1]), VF = -eps * n;
      S.cH1[n] = VH;
      S.cF1[n] = VF + (2 * n + 1);
      S.cLF1[n] = -S.rad * eps * n;
      S.cLH1[n] = S.rad * (n * bI[n] + valsqr * bI[n + 1] / double(2 * n + 3));
      S.cH2[n] = DH + (2 * n + 1) / bI[n];
      S.cF2[n] = DF;
      S.cLF2[n] = S.rad;
      S.cLH2[n] = -S.rad * bI[n];
      S.cInvH[n] = bI[n] * (T.CONST3[n]);
      S.cChgH[n] = T.CONST2[n] / bI[n];
    }
  }
  // self surface charges (generateMolExposedChargesFH)
  for (int k = 0; k < ns && self_terms; k++) {
    SphType &S = mt.sph[k];
    const double dA = 4.0 * M_PI / double(S.nspx);
    std::vector<double> bI(NP + 1, 1.0);
    bessel_i(bI, T.kappa * S.rad);
    std::vector<double> constH(NP);
    for (int n = 0; n < NP; n++) constH[n] = T.CONST2[n] / bI[n];
    S.qFself.assign(S.spx.size(), 0); S.qHself.assign(S.spx.size(), 0);
    S.tFself = 0; S.tHself = 0;
    for (size_t h = 0; h < S.spx.size(); h++) {
      Sph q = cart2sph(S.spx[h]);
      vec Y; sph_harm(T, q.theta, q.phi, NP, Y);
      vec YI = Y;
      for (int n = 0; n < NP; n++) for (int m = 0; m < 2 * n + 1; m++) YI[IDX(n) + m] = Y[IDX(n) + m] * T.CONST2[n];
      S.qFself[h] = inprod_unit(S.Fself, YI) * dA;
      S.tFself += fabs(S.qFself[h]);
      for (int n = 0; n < NP; n++) for (int m = 0; m < 2 * n + 1; m++) YI[IDX(n) + m] = Y[IDX(n) + m] * constH[n];
      S.qHself[h] = inprod_unit(S.Hself, YI) * dA;
      S.tHself += fabs(S.qHself[h]);
    }
  }
  // intra pol lists (generateMolTypeIntraPolLists)
  std::vector<std::vector<int> > far(ns);
  for (int kj = 0; kj < ns; kj++)
    for (int ki = 0; ki < kj; ki++) {
      double rho = (cr[ki] - cr[kj]).norm();
      if (rho < (rad[ki] + rad[kj] + prm.intra_cut)) { mt.sph[ki].near.push_back(kj); mt.sph[kj].near.push_back(ki); }
      else { far[ki].push_back(kj); far[kj].push_back(ki); }
    }
  // moltype self local expansions (computeMolTypeValues)
  for (int ki = 0; ki < ns && self_terms; ki++) {
    SphType &Si = mt.sph[ki];
    Si.LFfar.assign(NP * NP, 0); Si.LHfar.assign(NP * NP, 0);
    for (size_t t = 0; t < far[ki].size(); t++) {
      int kj = far[ki][t];
      const SphType &Sj = mt.sph[kj];
      P3 P = Si.cen - Sj.cen;
      XForm X; X.reset_intra(T, P, NP, NP, Sj.rad, Si.rad);
      vec a, b;
      X.xformF(Sj.Fself, a); X.xformH(Sj.Hself, b);
      add_into(Si.LFfar, a); add_into(Si.LHfar, b);
    }
    Si.LFintra = Si.LFfar; Si.LHintra = Si.LHfar;
    for (size_t t = 0; t < Si.near.size(); t++) {
      int kj = Si.near[t];
      const SphType &Sj = mt.sph[kj];
      P3 P = Si.cen - Sj.cen;
      double rho = P.norm(), sep = rho - Si.rad - Sj.rad;
      vec a, b;
      if (sep > 0 && !(sep < 5)) {
        XForm X; X.reset_intra(T, P, NP, NP, Sj.rad, Si.rad);
        X.xformF(Sj.Fself, a); X.xformH(Sj.Hself, b);
      } else {
        int pF = compute_order(NP, rho, Sj.tFself, Sj.rad), pH = compute_order(NP, rho, Sj.tHself, Sj.rad);
        for (size_t h = 0; h < Sj.spx.size(); h++) {
          P3 d = Sj.spx[h] - P;
          if (Sj.qFself[h] != 0.0) add_local_charge(T, a, Sj.qFself[h], d, false, pF, Si.rad);
        }
        if (a.empty()) a.assign(pF * pF, 0.0);
        for (size_t h = 0; h < Sj.spx.size(); h++) {
          P3 d = Sj.spx[h] - P;
          if (Sj.qHself[h] != 0.0) add_local_charge(T, b, Sj.qHself[h], d, true, pH, Si.rad);
        }
        if (b.empty()) b.assign(pH * pH, 0.0);
      }
      add_into(Si.LFintra, a); add_into(Si.LHintra, b);
    }
  }
  // fixed charges (setFixedCharges with m_bKappa = false) and Dirichlet/Neumann terms (cal_DVFixed)
  for (int k = 0; k < ns; k++) {
    SphType &S = mt.sph[k];
    S.Efix.assign(NP * NP, 0); S.Lfix.assign(NP * NP, 0);
    const double rsq = S.rad * S.rad;
    for (size_t i = 0; i < posr.size(); i++) {
      P3 ap = posr[i] - S.cen;
      double c = ch[i] / prm.idiel;
      if (c == 0.0) continue;
      if (ap.norm2() < rsq) add_multipole_charge(T, S.Efix, c, ap, false, NP, S.rad);
      else add_local_charge(T, S.Lfix, c, ap, false, NP, S.rad);
    }
    S.Dfix.assign(NP * NP, 0); S.Vfix.assign(NP * NP, 0);
    for (int n = 0, kk = 0; n < NP; n++) {
      const double DE = 1.0, DL = S.rad, VE = eps * (n + 1), VL = -eps * n * S.rad;
      for (int mm = 0; mm < 2 * n + 1; mm++, kk++) {
        S.Dfix[kk] = DE * S.Efix[kk] + DL * S.Lfix[kk];
        S.Vfix[kk] = VE * S.Efix[kk] + VL * S.Lfix[kk];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// per-sphere mutable state (CSolExpCenter members used on the force path)
struct SphState {
  vec F, H, Hrot, HselfRot, LS, LFS, LHS;
  double hscale;                    // scale carried by H (file scale until solved)
  vec qF, qH;
  double tF, tH;
  std::vector<P3> gF, gHp;          // gradient surface charges (m_gSolvedF/H)
  double maxgF, maxgH;
  double dev;
  vec gLHN[3], gH[3];
  P3 cenRot;
  std::vector<std::pair<int, int> > interPol, interact;
};

struct Molecule {
  int type;
  P3 rcen;
  Quat orient;
  Rot rot;
  bool interXForm;
  std::vector<SphState> s;
  std::vector<std::pair<int, int> > interMolPolList;
  std::vector<int> intraMolPolList, intraInteractOnly;
};

struct System {
  Tables T;
  Params prm;
  std::vector<MolType> types;
  std::vector<Molecule> mols;
  int NP;
  double MAXDEV = 0.0;

  const SphType &st(int i, int k) const { return types[mols[i].type].sph[k]; }

  // per-sphere constants solve (src/expcenter.cpp:1079-1328)
  static double compute_dev(const double *M1, const double *M2, int p, int D)
  {
    double sum = 0;
    int k = 0;
    for (int d = 0; d < D; d++)
      for (int n = 0; n < p; n++)
        for (int m = 0; m <= n; m++) {
          cplx a, b;
          if (m == 0) { a = cplx(M1[k], 0); b = cplx(M2[k], 0); k++; }
          else { a = cplx(M1[k], M1[k + 1]); b = cplx(M2[k], M2[k + 1]); k += 2; }
          double s;
          const double PL = 1e-30;
          if (fabs(a.real()) < PL && fabs(a.imag()) < PL) {
            if (fabs(b.real()) < PL && fabs(b.imag()) < PL) continue;
            s = 1.0;
          } else if (fabs(b.real()) < PL && fabs(b.imag()) < PL) s = 1.0;
          else {
            cplx diff = a - b;
            double top = diff.real() * diff.real() + diff.imag() * diff.imag();
            double bot = a.real() * a.real() + a.imag() * a.imag() + b.real() * b.real() + b.imag() * b.imag();
            s = (m != 0) ? 2 * top / bot : top / bot;
          }
          sum += s;
        }
    sum /= 4 * p * p;
    return sum;
  }
  static double compute_dev2(const double *M1, const double *M2, int p, int D)
  {
    double totdiff = 0, totsum = 0;
    for (int d = 0, k = 0; d < D; d++)
      for (int n = 0; n < p; n++) {
        cplx a(M1[k], 0), b(M2[k], 0);
        k++;
        cplx diff = a - b;
        totdiff += diff.real() * diff.real() + diff.imag() * diff.imag();
        totsum += a.real() * a.real() + a.imag() * a.imag() + b.real() * b.real() + b.imag() * b.imag();
        for (int m = 1; m <= n; m++) {
          a = cplx(M1[k], M1[k + 1]); b = cplx(M2[k], M2[k + 1]);
          k += 2;
          diff = a - b;
          totdiff += 2 * (diff.real() * diff.real() + diff.imag() * diff.imag());
          totsum += 2 * (a.real() * a.real() + a.imag() * a.imag() + b.real() * b.real() + b.imag() * b.imag());
        }
      }
    return totdiff / (4 * totsum) / double(D);
  }
  double solve_fh(const SphType &S, vec &F, vec &H, const vec &LF, const vec &LH, int D) const
  {
    const int p = NP, p2 = p * p, len = D * p2;
    vec hbase(len), fbase(len), hx(len), fx(len), oldH, outerOldH;
    for (int d = 0, k = 0; d < D; d++)
      for (int n = 0; n < p; n++)
        for (int mm = 0; mm < 2 * n + 1; mm++, k++) {
          if (D == 1) {
            fbase[k] = S.Vfix[k] + S.cLH1[n] * LH[k] + S.cLF1[n] * LF[k];
            hbase[k] = S.Dfix[k] + S.cLH2[n] * LH[k] + S.cLF2[n] * LF[k];
          } else {
            fbase[k] = S.cLH1[n] * LH[k] + S.cLF1[n] * LF[k];
            hbase[k] = S.cLH2[n] * LH[k] + S.cLF2[n] * LF[k];
          }
        }
    oldH = H; outerOldH = H;
    auto matmul = [&](const vec &X, vec &Y) {      // applyMMat: Y = IMat * X (column-major)
#ifdef PBSAM_PREP
      // the same sums, row blocks across threads, columns streamed in order
      for (int d = 0; d < D; d++) {
#pragma omp parallel for schedule(static)
        for (int i0 = 0; i0 < p2; i0 += 64) {
          const int i1 = i0 + 64 < p2 ? i0 + 64 : p2;
          double acc[64];
          for (int i = i0; i < i1; i++) acc[i - i0] = 0.0;
          for (int kk = 0; kk < p2; kk++) {
            const double x = X[d * p2 + kk];
            const double *a = S.imat.data() + (size_t)kk * p2;
            for (int i = i0; i < i1; i++) acc[i - i0] += a[i] * x;
          }
          for (int i = i0; i < i1; i++) Y[d * p2 + i] = acc[i - i0];
        }
      }
#else
      for (int d = 0; d < D; d++)
        for (int i = 0; i < p2; i++) {
          double s = 0.0;
          for (int kk = 0; kk < p2; kk++) s += S.imat[(size_t)kk * p2 + i] * X[d * p2 + kk];
          Y[d * p2 + i] = s;
        }
#endif
    };
    auto iterate = [&]() {
      for (int d = 0, k = 0; d < D; d++)
        for (int n = 0; n < p; n++)
          for (int mm = 0; mm < 2 * n + 1; mm++, k++) fx[k] = fbase[k] + S.cH1[n] * H[k] + S.cF1[n] * F[k];
      matmul(fx, F);
      for (int d = 0, k = 0; d < D; d++)
        for (int n = 0; n < p; n++)
          for (int mm = 0; mm < 2 * n + 1; mm++, k++) F[k] *= T.CONST3[n];
      for (int d = 0, k = 0; d < D; d++)
        for (int n = 0; n < p; n++)
          for (int mm = 0; mm < 2 * n + 1; mm++, k++) hx[k] = hbase[k] + S.cH2[n] * H[k] + S.cF2[n] * F[k];
      matmul(hx, H);
      for (int d = 0, k = 0; d < D; d++)
        for (int n = 0; n < p; n++)
          for (int mm = 0; mm < 2 * n + 1; mm++, k++) H[k] *= S.cInvH[n];
      double dv = compute_dev(oldH.data(), H.data(), p, D);
      oldH = H;
      return dv;
    };
    if (exact_inner) {
      // the fixed point of the iteration solved directly (Gaussian elimination with
      // partial pivoting): F = C3 M (fb + cH1 H + cF1 F), H = CI M (hb + cH2 H + cF2 F)
      const int n2 = 2 * p2;
      std::vector<int> deg(p2);
      for (int n = 0; n < p; n++) for (int k = n * n; k < (n + 1) * (n + 1); k++) deg[k] = n;
      std::vector<double> A((size_t)n2 * n2, 0.0);
      for (int i = 0; i < p2; i++) {
        const double c3 = T.CONST3[deg[i]], ci = S.cInvH[deg[i]];
        for (int kk = 0; kk < p2; kk++) {
          const double m = S.imat[(size_t)kk * p2 + i];
          A[(size_t)i * n2 + kk] -= c3 * m * S.cF1[deg[kk]];
          A[(size_t)i * n2 + p2 + kk] -= c3 * m * S.cH1[deg[kk]];
          A[(size_t)(p2 + i) * n2 + kk] -= ci * m * S.cF2[deg[kk]];
          A[(size_t)(p2 + i) * n2 + p2 + kk] -= ci * m * S.cH2[deg[kk]];
        }
        A[(size_t)i * n2 + i] += 1.0;
        A[(size_t)(p2 + i) * n2 + p2 + i] += 1.0;
      }
      for (int d = 0; d < D; d++) {
        std::vector<double> B = A, y(n2, 0.0);
        for (int i = 0; i < p2; i++) {
          double sf = 0.0, sh = 0.0;
          for (int kk = 0; kk < p2; kk++) {
            sf += S.imat[(size_t)kk * p2 + i] * fbase[d * p2 + kk];
            sh += S.imat[(size_t)kk * p2 + i] * hbase[d * p2 + kk];
          }
          y[i] = T.CONST3[deg[i]] * sf;
          y[p2 + i] = S.cInvH[deg[i]] * sh;
        }
        for (int c = 0; c < n2; c++) {
          int piv = c;
          for (int r = c + 1; r < n2; r++) if (fabs(B[(size_t)r * n2 + c]) > fabs(B[(size_t)piv * n2 + c])) piv = r;
          if (piv != c) { for (int k = 0; k < n2; k++) std::swap(B[(size_t)c * n2 + k], B[(size_t)piv * n2 + k]); std::swap(y[c], y[piv]); }
          for (int r = c + 1; r < n2; r++) {
            const double f = B[(size_t)r * n2 + c] / B[(size_t)c * n2 + c];
            if (f == 0.0) continue;
            for (int k = c; k < n2; k++) B[(size_t)r * n2 + k] -= f * B[(size_t)c * n2 + k];
            y[r] -= f * y[c];
          }
        }
        for (int c = n2 - 1; c >= 0; c--) {
          double sum = y[c];
          for (int k = c + 1; k < n2; k++) sum -= B[(size_t)c * n2 + k] * y[k];
          y[c] = sum / B[(size_t)c * n2 + c];
        }
        for (int i = 0; i < p2; i++) { F[d * p2 + i] = y[i]; H[d * p2 + i] = y[p2 + i]; }
      }
      n_inner += 1; n_solves++;
      return compute_dev2(outerOldH.data(), H.data(), p, D);
    }
    double dev = iterate();
    int ct = 1;
    while (dev > prm.solve_tol && ct < prm.solve_max_ct) { dev = iterate(); ct++; }
    n_inner += ct; n_solves++;
    return compute_dev2(outerOldH.data(), H.data(), p, D);
  }
  bool exact_inner = false;   // solve each sphere's F/H fixed point directly
  mutable long n_inner = 0, n_solves = 0;

  // exposed surface charges (src/expcenter.cpp:1419-1440)
  void surface_charges(int i, int k)
  {
    const SphType &S = st(i, k);
    SphState &Z = mols[i].s[k];
    const double dA = 4 * M_PI / double(S.nspx);
    Z.tF = 0.0; Z.tH = 0.0;
    for (size_t h = 0; h < S.spx.size(); h++) {
      Sph q = cart2sph(S.spx[h]);
      vec Y; sph_harm(T, q.theta, q.phi, NP, Y);
      vec YI = Y;
      for (int n = 0; n < NP; n++) for (int m = 0; m < 2 * n + 1; m++) YI[IDX(n) + m] = Y[IDX(n) + m] * T.CONST2[n];
      Z.qF[h] = inprod_unit(Z.F, YI) * dA;
      Z.tF += fabs(Z.qF[h]);
      for (int n = 0; n < NP; n++) for (int m = 0; m < 2 * n + 1; m++) YI[IDX(n) + m] = Y[IDX(n) + m] * S.cChgH[n];
      Z.qH[h] = inprod_unit(Z.H, YI) * dA;
      Z.tH += fabs(Z.qH[h]);
    }
  }
  // exposed gradient charges (src/expcenter.cpp:1377-1412)
  void surface_gradient(int i, int k, const vec gF[3], const vec gH[3])
  {
    const SphType &S = st(i, k);
    SphState &Z = mols[i].s[k];
    const double dA = 4 * M_PI / double(S.nspx);
    double tfx = 0, tfy = 0, tfz = 0, thx = 0, thy = 0, thz = 0;
    for (size_t h = 0; h < S.spx.size(); h++) {
      Sph q = cart2sph(S.spx[h]);
      vec Y; sph_harm(T, q.theta, q.phi, NP, Y);
      vec YI = Y;
      for (int n = 0; n < NP; n++) for (int m = 0; m < 2 * n + 1; m++) YI[IDX(n) + m] = Y[IDX(n) + m] * T.CONST2[n];
      double fx = inprod_unit(gF[0], YI) * dA, fy = inprod_unit(gF[1], YI) * dA, fz = inprod_unit(gF[2], YI) * dA;
      Z.gF[h] = P3(fx, fy, fz);
      tfx += fabs(fx); tfy += fabs(fy); tfz += fabs(fz);
      for (int n = 0; n < NP; n++) for (int m = 0; m < 2 * n + 1; m++) YI[IDX(n) + m] = Y[IDX(n) + m] * S.cChgH[n];
      double hx = inprod_unit(gH[0], YI) * dA, hy = inprod_unit(gH[1], YI) * dA, hz = inprod_unit(gH[2], YI) * dA;
      Z.gHp[h] = P3(hx, hy, hz);
      thx += fabs(hx); thy += fabs(hy); thz += fabs(hz);
    }
    Z.maxgF = (tfx > tfy ? tfx : tfy); if (tfz > Z.maxgF) Z.maxgF = tfz;
    Z.maxgH = (thx > thy ? thx : thy); if (thz > Z.maxgH) Z.maxgH = thz;
  }

  P3 cen_lab(int i, int k) const { return mols[i].rcen + mols[i].s[k].cenRot; }

  void add_molecule(int type)
  {
    Molecule M;
    M.type = type;
    M.rot.reset_quat(T, Quat(), NP);
    M.interXForm = false;
    const MolType &mt = types[type];
    M.s.assign(mt.ns, SphState());
    for (int k = 0; k < mt.ns; k++) {
      const SphType &S = mt.sph[k];
      SphState &Z = M.s[k];
      Z.F = S.Fself; Z.H = S.Hself; Z.Hrot = S.Hself; Z.hscale = S.hself_scale;
      Z.qF = S.qFself; Z.qH = S.qHself; Z.tF = S.tFself; Z.tH = S.tHself;   // initSurfaceCharges from self values
      Z.gF.assign(S.spx.size(), P3()); Z.gHp.assign(S.spx.size(), P3());
      Z.maxgF = 0; Z.maxgH = 0; Z.dev = 0;
      for (int c = 0; c < 3; c++) { Z.gLHN[c].assign(NP * NP, 0.0); Z.gH[c].assign(NP * NP, 0.0); }
      Z.LS.assign(NP * NP, 0); Z.LFS.assign(NP * NP, 0); Z.LHS.assign(NP * NP, 0);
      Z.cenRot = S.cen;
    }
    mols.push_back(M);
  }
  void set_pose(int i, const P3 &pos, const Quat &q)
  {
    Molecule &M = mols[i];
    M.rcen = pos;
    M.orient = q;
    for (size_t k = 0; k < M.s.size(); k++) M.s[k].cenRot = qrot(q, st(i, k).cen);
  }

  // pair lists (src/molecule.cpp:1035-1126, 122-166)
  bool pair_lists()
  {
    const int nmol = mols.size();
    if (nmol == 1) return true;
    for (int i = 0; i < nmol; i++) {
      mols[i].interXForm = false;
      for (auto &Z : mols[i].s) { Z.interPol.clear(); Z.interact.clear(); }
    }
    for (int j = 1; j < nmol; j++) {
      std::vector<int> neigh;
      for (int i = 0; i < j; i++) {
        double c2c = (mols[i].rcen - mols[j].rcen).norm();
        double sep = c2c - types[mols[i].type].maxR - types[mols[j].type].maxR;
        if (sep < prm.interact_cut) neigh.push_back(i);
      }
      if (neigh.empty()) continue;
      for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
        for (size_t ii = 0; ii < neigh.size(); ii++) {
          int i = neigh[ii];
          for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
            P3 P = cen_lab(i, ki) - cen_lab(j, kj);
            double sep = P.norm() - st(i, ki).rad - st(j, kj).rad;
            if (sep <= 0) return false;
            if (sep < prm.interact_cut) {
              if (sep > prm.inter_cut) {
                mols[i].s[ki].interact.push_back({j, (int)kj});
                mols[j].s[kj].interact.push_back({i, (int)ki});
              } else {
                mols[i].s[ki].interPol.push_back({j, (int)kj});
                mols[j].s[kj].interPol.push_back({i, (int)ki});
              }
              mols[i].interXForm = true;
              mols[j].interXForm = true;
            }
          }
        }
      }
    }
    for (int i = 0; i < nmol; i++) mols[i].interMolPolList.clear();
    for (int i = 0; i < nmol; i++)
      for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
        std::vector<bool> added(nmol, false);
        for (auto &e : mols[i].s[ki].interPol) {
          int j = e.first;
          if (added[j]) continue;
          mols[j].interMolPolList.push_back({i, (int)ki});
          added[j] = true;
        }
      }
    for (int j = 0; j < nmol; j++) {
      mols[j].intraMolPolList.clear(); mols[j].intraInteractOnly.clear();
      for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
        const SphState &Z = mols[j].s[kj];
        if (!Z.interPol.empty()) mols[j].intraMolPolList.push_back(kj);
        else if (!Z.interact.empty()) mols[j].intraInteractOnly.push_back(kj);
      }
    }
    return true;
  }

  // LS from neighbours' rotated H (src/molecule.cpp:1265-1358)
  void reexpand_LS(int i, int ki, bool fromSelf)
  {
    SphState &Z = mols[i].s[ki];
    const SphType &Si = st(i, ki);
    vec LSrot(NP * NP, 0.0);
    for (auto &e : Z.interPol) {
      int j = e.first, kj = e.second;
      const SphState &Zj = mols[j].s[kj];
      const SphType &Sj = st(j, kj);
      P3 P = cen_lab(i, ki) - cen_lab(j, kj);
      int pj2i = compute_order(NP, P.norm(), fromSelf ? Sj.tHself : Zj.tH, Sj.rad);
      XForm X; X.reset(T, P, pj2i, Sj.rad, Si.rad, false);
      vec tL; X.xformH(fromSelf ? Zj.HselfRot : Zj.Hrot, tL);
      add_into(LSrot, tL);
    }
    mols[i].rot.rotate_xi(LSrot, Z.LS, NP, false);
  }
  // intra near re-expansion with latest values (src/molecule.cpp:1413-1473)
  void reexpand_intra_near(int i, int ki)
  {
    SphState &Z = mols[i].s[ki];
    const SphType &Si = st(i, ki);
    Z.LFS.assign(NP * NP, 0.0);
    Z.LHS = Z.LS;
    const int nn = Si.near.size();
#ifdef PBSAM_PREP
    // neighbours' terms computed across threads, added in list order
    std::vector<vec> ta(nn), tb(nn);
#pragma omp parallel for schedule(dynamic)
    for (int t = 0; t < nn; t++) intra_near_term(i, ki, Si.near[t], ta[t], tb[t]);
    for (int t = 0; t < nn; t++) { add_into(Z.LFS, ta[t]); add_into(Z.LHS, tb[t]); }
#else
    for (int t = 0; t < nn; t++) {
      vec a, b;
      intra_near_term(i, ki, Si.near[t], a, b);
      add_into(Z.LFS, a); add_into(Z.LHS, b);
    }
#endif
  }
  // one near neighbour kj's F (a) and H (b) re-expanded into sphere ki
  void intra_near_term(int i, int ki, int kj, vec &a, vec &b) const
  {
    const SphType &Si = st(i, ki);
    const SphType &Sj = st(i, kj);
    const SphState &Zj = mols[i].s[kj];
    P3 P = Si.cen - Sj.cen;
    double rho = P.norm(), sep = rho - Si.rad - Sj.rad;
    if (sep > 0 && !(sep < 5)) {
      int pF = compute_order(NP, rho, Zj.tF, Sj.rad), pH = compute_order(NP, rho, Zj.tH, Sj.rad);
      XForm X; X.reset_intra(T, P, pH, pF, Sj.rad, Si.rad);
      X.xformF(Zj.F, a); X.xformH(Zj.H, b);
    } else {
      int pF = compute_order(NP, rho, Zj.tF, Sj.rad), pH = compute_order(NP, rho, Zj.tH, Sj.rad);
      a.assign(pF * pF, 0.0); b.assign(pH * pH, 0.0);
      for (size_t h = 0; h < Sj.spx.size(); h++) {
        P3 d = Sj.spx[h] - P;
        if (Zj.qF[h] != 0.0) add_local_charge(T, a, Zj.qF[h], d, false, pF, Si.rad);
        if (Zj.qH[h] != 0.0) add_local_charge(T, b, Zj.qH[h], d, true, pH, Si.rad);
      }
    }
  }
  double solve_surface(int i, int ki, const vec &Finit, const vec &Hinit, bool rotH)   // src/expcenter.cpp:608-629
  {
    const SphType &S = st(i, ki);
    SphState &Z = mols[i].s[ki];
    vec F = trunc_or_pad(Finit, NP), H = trunc_or_pad(Hinit, NP);
    double dv = solve_fh(S, F, H, trunc_or_pad(Z.LFS, NP), trunc_or_pad(Z.LHS, NP), 1);
    Z.F = F; Z.H = H; Z.hscale = 1.0 / S.rad;
    if (rotH) mols[i].rot.rotate_xi(Z.H, Z.Hrot, NP, true);
    Z.dev = dv;
    surface_charges(i, ki);
    return dv;
  }
  double recompute_from_self(int i, int ki)     // src/molecule.cpp:1136-1160, 1236-1246
  {
    SphState &Z = mols[i].s[ki];
    const SphType &S = st(i, ki);
    reexpand_LS(i, ki, true);
    Z.LHS = Z.LS; add_into(Z.LHS, S.LHintra);
    Z.LFS = S.LFintra;
    return solve_surface(i, ki, S.Fself, S.Hself, true);
  }
  double recompute(int i, int ki)               // src/molecule.cpp:1168-1229
  {
    SphState &Z = mols[i].s[ki];
    const SphType &S = st(i, ki);
    reexpand_LS(i, ki, false);
    reexpand_intra_near(i, ki);
    add_into(Z.LHS, S.LHfar);
    add_into(Z.LFS, S.LFfar);
    vec F = Z.F, H = Z.H;
    return solve_surface(i, ki, F, H, false);
  }

  // gradient pieces (src/molecule.cpp:1483-1628)
  void grad_xform_from(int i, int ki, int m, int km, bool self, vec acc[3], bool pbc_unused = false)
  {
    const SphState &Zm = mols[m].s[km];
    const SphType &Sm = st(m, km), &Si = st(i, ki);
    P3 P = cen_lab(i, ki) - cen_lab(m, km);
    int p = compute_order(NP, P.norm(), self ? Sm.tHself : Zm.tH, Sm.rad);
    XForm X; X.reset(T, P, p, Sm.rad, Si.rad, true);
    vec G[3];
    X.xformH_grad(self ? Zm.HselfRot : Zm.Hrot, G);
    for (int c = 0; c < 3; c++) add_into(acc[c], G[c]);
  }
  void prepare_dta(int j, std::vector<std::array<vec, 3> > &tG)
  {
    const Molecule &Mj = mols[j];
    size_t ni = Mj.interMolPolList.size(), na = Mj.intraMolPolList.size();
    tG.assign(ni + na, std::array<vec, 3>());
    size_t k = 0;
    for (; k < ni; k++) {
      int i = Mj.interMolPolList[k].first, ki = Mj.interMolPolList[k].second;
      for (int c = 0; c < 3; c++) tG[k][c].assign(NP * NP, 0.0);
      for (auto &e : mols[i].s[ki].interPol) {
        if (e.first != j) continue;
        grad_xform_from(i, ki, e.first, e.second, false, tG[k].data());
      }
    }
    for (size_t hh = 0; hh < na; hh++, k++) {
      int ki = Mj.intraMolPolList[hh];
      for (int c = 0; c < 3; c++) tG[k][c].assign(NP * NP, 0.0);
      for (auto &e : mols[j].s[ki].interPol) grad_xform_from(j, ki, e.first, e.second, false, tG[k].data());
      for (auto &e : mols[j].s[ki].interact) grad_xform_from(j, ki, e.first, e.second, false, tG[k].data());
    }
  }
  void prepare_dta_iself(int i, int ki)
  {
    vec acc[3];
    for (int c = 0; c < 3; c++) acc[c].assign(NP * NP, 0.0);
    for (auto &e : mols[i].s[ki].interPol) grad_xform_from(i, ki, e.first, e.second, true, acc);
    for (auto &e : mols[i].s[ki].interact) grad_xform_from(i, ki, e.first, e.second, true, acc);
    for (int c = 0; c < 3; c++) mols[i].s[ki].gLHN[c] = acc[c];
  }

  struct GradSet {
    std::vector<std::array<vec, 3> > gF, gH, gHrot;
    std::map<std::pair<int, int>, int> key;
  };

  double recompute_grad(int i, int ki, int j, const std::array<vec, 3> &tG_DTA, GradSet &G)   // src/molecule.cpp:1810-1843
  {
    SphState &Z = mols[i].s[ki];
    const SphType &Si = st(i, ki);
    // reexpandGrad (src/molecule.cpp:1680-1724)
    vec tGrot[3] = {tG_DTA[0], tG_DTA[1], tG_DTA[2]};
    for (auto &e : Z.interPol) {
      if (i != j && e.first != j) continue;
      int m = e.first, km = e.second;
      const SphState &Zm = mols[m].s[km];
      const SphType &Sm = st(m, km);
      P3 P = cen_lab(i, ki) - cen_lab(m, km);
      int p = compute_order(NP, P.norm(), Zm.maxgH, Sm.rad);
      XForm X; X.reset(T, P, p, Sm.rad, Si.rad, false);
      const std::array<vec, 3> &src = G.gHrot[G.key[{m, km}]];
      for (int c = 0; c < 3; c++) { vec o; X.xformH(src[c], o); add_into(tGrot[c], o); }
    }
    vec LGH[3];
    for (int c = 0; c < 3; c++) mols[i].rot.rotate_xi(tGrot[c], LGH[c], NP, false);
    if (j == i) for (int c = 0; c < 3; c++) Z.gLHN[c] = LGH[c];
    // reexpandIntraGrad (src/molecule.cpp:1730-1802)
    vec LGF[3], LGH2[3];
    for (int c = 0; c < 3; c++) { LGF[c].assign(NP * NP, 0.0); LGH2[c].assign(NP * NP, 0.0); }
    std::vector<int> plist;
    if (i == j) plist = mols[j].intraMolPolList;
    else for (auto &e : mols[j].interMolPolList) if (e.first == i) plist.push_back(e.second);
    for (int km : plist) {
      if (km == ki) continue;
      const SphType &Sm = st(i, km);
      const SphState &Zm = mols[i].s[km];
      P3 P = Si.cen - Sm.cen;
      double rho = P.norm(), sep = rho - Si.rad - Sm.rad;
      if (sep > 0 && !(sep < 5)) {
        int pF = compute_order(NP, rho, Zm.maxgF, Sm.rad), pH = compute_order(NP, rho, Zm.maxgH, Sm.rad);
        XForm X; X.reset_intra(T, P, pH, pF, Sm.rad, Si.rad);
        int key = G.key[{i, km}];
        for (int c = 0; c < 3; c++) {
          vec o; X.xformF(G.gF[key][c], o); add_into(LGF[c], o);
          X.xformH(G.gH[key][c], o); add_into(LGH2[c], o);
        }
      } else {
        int pF = compute_order(NP, rho, Zm.maxgF, Sm.rad), pH = compute_order(NP, rho, Zm.maxgH, Sm.rad);
        vec a[3], b[3];
        for (int c = 0; c < 3; c++) { a[c].assign(pF * pF, 0.0); b[c].assign(pH * pH, 0.0); }
        for (size_t h = 0; h < Sm.spx.size(); h++) {
          P3 d = Sm.spx[h] - P;
          const P3 &gf = Zm.gF[h], &gh = Zm.gHp[h];
          if (gf.norm2() >= 1e-15) {
            vec L; add_local_charge(T, L, 1.0, d, false, pF, Si.rad);
            for (int t = 0; t < pF * pF; t++) { a[0][t] += gf.x * L[t]; a[1][t] += gf.y * L[t]; a[2][t] += gf.z * L[t]; }
          }
          if (gh.norm2() >= 1e-15) {
            vec L; add_local_charge(T, L, 1.0, d, true, pH, Si.rad);
            for (int t = 0; t < pH * pH; t++) { b[0][t] += gh.x * L[t]; b[1][t] += gh.y * L[t]; b[2][t] += gh.z * L[t]; }
          }
        }
        for (int c = 0; c < 3; c++) { add_into(LGF[c], a[c]); add_into(LGH2[c], b[c]); }
      }
    }
    for (int c = 0; c < 3; c++) add_into(LGH[c], LGH2[c]);
    // solveSurfaceGradient (src/expcenter.cpp:639-659)
    int key = G.key[{i, ki}];
    vec gF(3 * NP * NP), gH(3 * NP * NP), LF1(3 * NP * NP), LH1(3 * NP * NP);
    for (int c = 0; c < 3; c++)
      for (int t = 0; t < NP * NP; t++) {
        gF[c * NP * NP + t] = G.gF[key][c][t];
        gH[c * NP * NP + t] = G.gH[key][c][t];
        LF1[c * NP * NP + t] = t < (int)LGF[c].size() ? LGF[c][t] : 0.0;
        LH1[c * NP * NP + t] = t < (int)LGH[c].size() ? LGH[c][t] : 0.0;
      }
    double dv = solve_fh(Si, gF, gH, LF1, LH1, 3);
    for (int c = 0; c < 3; c++)
      for (int t = 0; t < NP * NP; t++) { G.gF[key][c][t] = gF[c * NP * NP + t]; G.gH[key][c][t] = gH[c * NP * NP + t]; }
    for (int c = 0; c < 3; c++) mols[i].rot.rotate_xi(G.gH[key][c], G.gHrot[key][c], NP, true);
    Z.dev = dv;
    surface_gradient(i, ki, G.gF[key].data(), G.gH[key].data());
    return dv;
  }

  // polarize_mutual (src/molecule.cpp:1988-2263)
  void polarize_mutual()
  {
    const int nmol = mols.size();
    if (nmol == 1) return;
    for (int i = 0; i < nmol; i++) {
      if (!mols[i].interXForm) continue;
      mols[i].rot.reset_quat(T, mols[i].orient, NP);
      for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
        SphState &Z = mols[i].s[ki];
        if (!(Z.interPol.empty() && Z.interact.empty())) {
          mols[i].rot.rotate_xi(st(i, ki).Hself, Z.HselfRot, NP, true);
          Z.Hrot = Z.HselfRot;
        }
      }
    }
    double dev = 0.0;
    int mtotal = 0;
    std::vector<double> maxdevs(nmol, 0.0);
    for (int i = 0; i < nmol; i++) {
      double dmol = 0.0;
      if (mols[i].interXForm)
        for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
          if (mols[i].s[ki].interPol.empty()) continue;
          double d = recompute_from_self(i, ki);
          dmol += d;
          if (maxdevs[i] < d) maxdevs[i] = d;
          mtotal++;
        }
      dev += dmol;
    }
    MAXDEV = 0.0;
    for (int i = 0; i < nmol; i++) if (maxdevs[i] > MAXDEV) MAXDEV = maxdevs[i];
    int ct = 1;
    double itot = (mtotal > 0 ? 1.0 / mtotal : 0);
    const double tol2 = prm.max_polar_dev * prm.max_polar_dev;
    while (dev * itot > tol2 && ct < prm.max_pol_rounds) {
      dev = 0.0;
      maxdevs.assign(nmol, 0.0);
      for (int i = 0; i < nmol; i++) {
        double dmol = 0.0;
        if (mols[i].interXForm)
          for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
            if (mols[i].s[ki].interPol.empty()) continue;
            double d = mols[i].s[ki].dev;
            // the exact form sweeps every sphere until the fixed point: the selective
            // update can leave a sphere whose last change was small out of date
            if (exact_inner || d > 0.1 * MAXDEV) d = recompute(i, ki);
            if (maxdevs[i] < d) maxdevs[i] = d;
            dmol += d;
          }
        dev += dmol;
      }
      MAXDEV = 0.0;
      for (int i = 0; i < nmol; i++) if (maxdevs[i] > MAXDEV) MAXDEV = maxdevs[i];
      ct++;
    }
    n_sweeps = ct;
    if (skip_grad) return;
    // gradient phase
    for (int j = 0; j < nmol; j++) {
      Molecule &Mj = mols[j];
      const int ni = Mj.interMolPolList.size();
      if (ni == 0) {
        if (Mj.interXForm)
          for (size_t kj = 0; kj < Mj.s.size(); kj++)
            if (!(Mj.s[kj].interPol.empty() && Mj.s[kj].interact.empty())) prepare_dta_iself(j, kj);
        continue;
      }
      const int na = Mj.intraMolPolList.size(), jsize = ni + na;
      std::vector<double> d(jsize);
      const double itj = 1.0 / double(jsize);
      std::vector<std::array<vec, 3> > tG;
      prepare_dta(j, tG);
      GradSet G;
      G.gF.assign(jsize, std::array<vec, 3>()); G.gH = G.gF; G.gHrot = G.gF;
      std::vector<std::pair<int, int> > ids(jsize);
      for (int k = 0; k < jsize; k++) {
        ids[k] = (k < ni) ? Mj.interMolPolList[k] : std::make_pair(j, Mj.intraMolPolList[k - ni]);
        for (int c = 0; c < 3; c++) { G.gF[k][c].assign(NP * NP, 0.0); G.gH[k][c].assign(NP * NP, 0.0); G.gHrot[k][c].assign(NP * NP, 0.0); }
        G.key[ids[k]] = k;
      }
      double dv = 0.0;
      for (int k = 0; k < jsize; k++) { d[k] = recompute_grad(ids[k].first, ids[k].second, j, tG[k], G); dv += d[k]; }
      int gct = 1, k = 0;
      while (dv * itj > tol2 && gct < prm.max_pol_rounds) {
        dv -= d[k];
        d[k] = recompute_grad(ids[k].first, ids[k].second, j, tG[k], G);
        dv += d[k];
        k++;
        if (k == jsize) { k = 0; gct++; }
      }
      for (int h = 0; h < na; h++) {
        int kj = Mj.intraMolPolList[h];
        for (int c = 0; c < 3; c++) Mj.s[kj].gH[c] = G.gH[G.key[{j, kj}]][c];
      }
      for (int kj : Mj.intraInteractOnly) prepare_dta_iself(j, kj);
    }
  }
  int n_sweeps = 0;
  bool skip_grad = false;   // energies only: leave out the per-molecule gradient solves

  // forces (src/moldynamics.cpp:524-587, src/expcenter.cpp:123-149)
  bool compute_forces(std::vector<P3> &force, std::vector<P3> &torque)
  {
    const int nmol = mols.size();
    force.assign(nmol, P3()); torque.assign(nmol, P3());
    if (nmol == 1) return true;
    if (!pair_lists()) return false;
    polarize_mutual();
    for (int i = 0; i < nmol; i++) {
      P3 f, t;
      if (mols[i].interXForm) {
        for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
          const SphState &Z = mols[i].s[ki];
          const SphType &S = st(i, ki);
          if (Z.interPol.empty() && Z.interact.empty()) continue;
          P3 fk;
          if (!Z.interPol.empty()) {
            fk.x -= inprod_ml(Z.H, 1.0 / S.rad, Z.gLHN[0], S.rad);
            fk.y -= inprod_ml(Z.H, 1.0 / S.rad, Z.gLHN[1], S.rad);
            fk.z -= inprod_ml(Z.H, 1.0 / S.rad, Z.gLHN[2], S.rad);
            fk.x -= inprod_ml(Z.gH[0], 1.0 / S.rad, Z.LS, S.rad);
            fk.y -= inprod_ml(Z.gH[1], 1.0 / S.rad, Z.LS, S.rad);
            fk.z -= inprod_ml(Z.gH[2], 1.0 / S.rad, Z.LS, S.rad);
          } else {
            fk.x -= inprod_ml(S.Hself, S.hself_scale, Z.gLHN[0], S.rad);
            fk.y -= inprod_ml(S.Hself, S.hself_scale, Z.gLHN[1], S.rad);
            fk.z -= inprod_ml(S.Hself, S.hself_scale, Z.gLHN[2], S.rad);
          }
          f = f + fk;
          t = t + cross(S.cen, fk);
        }
      }
      Quat cq = qconj(mols[i].orient);
      force[i] = qrot(cq, f);
      torque[i] = qrot(cq, t);
    }
    return true;
  }

  // interaction energy (src/moldynamics.cpp:358-386, src/molecule.cpp:1850-1890)
  double total_energy() const
  {
    double pot = 0.0;
    const int nmol = mols.size();
    for (int i = 0; i < nmol; i++)
      for (int j = i + 1; j < nmol; j++) {
        double e = 0.0;
        for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
          const SphType &Si = st(i, ki);
          const SphState &Zi = mols[i].s[ki];
          vec Lki(1, 0.0);
          for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
            const SphType &Sj = st(j, kj);
            const SphState &Zj = mols[j].s[kj];
            P3 P = (mols[i].rcen + Si.cen) - (mols[j].rcen + Sj.cen);
            double rho = P.norm();
            int pi2j = compute_order(NP, rho, Zi.tH, Si.rad), pj2i = compute_order(NP, rho, Zj.tH, Sj.rad);
            int minp = pi2j < pj2i ? pi2j : pj2i;
            XForm X; X.reset(T, P, minp, Sj.rad, Si.rad, false);
            vec tL; X.xformH(Zj.H, tL);
            add_into(Lki, tL);
          }
          e += inprod_ml(Zi.H, Zi.hscale, Lki, Si.rad);
        }
        pot += e;
      }
    return pot;
  }

  // the same sum in the lab frame: centres rcen + q*cen and H rotated to the lab
  // frame by the molecule's orientation (the corrected form of
  // interactCenters_LowMemory, src/molecule.cpp:1850-1890)
  double total_energy_lab()
  {
    const int nmol = mols.size();
    std::vector<std::vector<vec> > Hl(nmol);
    for (int i = 0; i < nmol; i++) {
      Rot R;
      R.reset_quat(T, mols[i].orient, NP);
      Hl[i].resize(mols[i].s.size());
      for (size_t k = 0; k < mols[i].s.size(); k++) R.rotate_xi(mols[i].s[k].H, Hl[i][k], NP, true);
    }
    double pot = 0.0;
    for (int i = 0; i < nmol; i++)
      for (int j = i + 1; j < nmol; j++) {
        double e = 0.0;
        for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
          const SphType &Si = st(i, ki);
          const SphState &Zi = mols[i].s[ki];
          vec Lki(1, 0.0);
          for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
            const SphType &Sj = st(j, kj);
            const SphState &Zj = mols[j].s[kj];
            P3 P = (mols[i].rcen + qrot(mols[i].orient, Si.cen)) - (mols[j].rcen + qrot(mols[j].orient, Sj.cen));
            double rho = P.norm();
            int pi2j = compute_order(NP, rho, Zi.tH, Si.rad), pj2i = compute_order(NP, rho, Zj.tH, Sj.rad);
            int minp = pi2j < pj2i ? pi2j : pj2i;
            XForm X; X.reset(T, P, minp, Sj.rad, Si.rad, false);
            vec tL; X.xformH(Hl[j][kj], tL);
            add_into(Lki, tL);
          }
          e += inprod_ml(Hl[i][ki], Zi.hscale, Lki, Si.rad);
        }
        pot += e;
      }
    return pot;
  }

  // electrostatic potential at a point from every sphere's H (CMolecule::computePotInSpace,
  // src/moldynamics.cpp:470-506, molecules not aggregated): the reference's convention uses
  // the unrotated sphere centres and molecule-frame H; lab = true the rotated centres and
  // lab-frame H
  double potential(const P3 &P, bool lab) const
  {
    double pot = 0.0;
    for (size_t i = 0; i < mols.size(); i++) {
      Rot R;
      if (lab) R.reset_quat(T, mols[i].orient, NP);
      for (size_t k = 0; k < mols[i].s.size(); k++) {
        const SphType &S = st(i, k);
        const SphState &Z = mols[i].s[k];
        const P3 c = lab ? mols[i].s[k].cenRot : S.cen;
        const P3 d = P - mols[i].rcen - c;
        const int p = compute_order(NP, d.norm(), Z.tH, S.rad);
        vec L;
        add_local_charge(T, L, 1.0, d, true, p, S.rad);
        vec H = Z.H;
        if (lab) R.rotate_xi(Z.H, H, NP, true);
        pot += inprod_ml(H, Z.hscale, L, S.rad);
      }
    }
    return pot;
  }

  // ---------------------------------------------------------------- adjoint (pinning form)
  // Gradient of the lab-frame interaction energy (total_energy_lab) with respect to
  // every molecule's position and orientation, through the converged polarization
  // of the reference's procedure (polarize_mutual, src/molecule.cpp:1988-2263): the
  // first round from self values (recomputeFromSelfVal), its rotated H frozen for the
  // later rounds (solveSurfaceCharges() does not rotate, src/expcenter.cpp:594-598),
  // then the intra-molecular fixed point.  Every linear operator is made an explicit
  // matrix here and transposed exactly; truncation orders and surface point sets are
  // held at their converged values.  It is the checker of the CUDA backward pass,
  // itself checked against central differences of total_energy_lab.
  struct LinMat {
    int nin = 0, nout = 0;
    std::vector<double> a;   // row-major nout x nin
    vec apply(const vec &x) const
    {
      vec y(nout, 0.0);
      for (int r = 0; r < nout; r++) {
        double s = 0.0;
        for (int c = 0; c < nin && c < (int)x.size(); c++) s += a[(size_t)r * nin + c] * x[c];
        y[r] = s;
      }
      return y;
    }
    vec applyT(const vec &w) const
    {
      vec y(nin, 0.0);
      for (int r = 0; r < nout && r < (int)w.size(); r++)
        for (int c = 0; c < nin; c++) y[c] += a[(size_t)r * nin + c] * w[r];
      return y;
    }
  };
  template <class Fn>
  static LinMat lin_of(int nin, int nout, Fn f)
  {
    LinMat M;
    M.nin = nin; M.nout = nout;
    M.a.assign((size_t)nin * nout, 0.0);
    vec e(nin, 0.0), o;
    for (int c = 0; c < nin; c++) {
      e[c] = 1.0;
      o.clear();
      f(e, o);
      for (int r = 0; r < nout && r < (int)o.size(); r++) M.a[(size_t)r * nin + c] = o[r];
      e[c] = 0.0;
    }
    return M;
  }
  static double vdot(const vec &a, const vec &b)
  {
    double s = 0.0;
    for (size_t k = 0; k < a.size() && k < b.size(); k++) s += a[k] * b[k];
    return s;
  }
  static void vacc(vec &a, const vec &b, double w = 1.0)
  {
    if (a.size() < b.size()) a.resize(b.size(), 0.0);
    for (size_t k = 0; k < b.size(); k++) a[k] += w * b[k];
  }
  // molecule rotation matrix: forward (molecule -> lab) or back
  LinMat rot_mat(const Quat &q, bool fwd) const
  {
    Rot R;
    R.reset_quat(T, q, NP);
    const int p2 = NP * NP;
    return lin_of(p2, p2, [&](const vec &x, vec &y) { R.rotate_xi(x, y, NP, fwd); });
  }
  // generator of a lab-frame rotation about axis c acting on a packed expansion:
  // d/de [rotation by e about c] v at e = 0.  Within degree n it couples order m
  // to m +- 1 with half ladder coefficients c_m = sqrt((n - m)(n + m + 1)) / 2 (the
  // m = 0 entry, weighted 1 against 2 for the others, takes 2 c_0); about z it turns
  // (Re, Im) of order m by m.  Checked against differenced rotation coefficients.
  static void rot_generator(int c, const vec &v, vec &o, int P)
  {
    o.assign(P * P, 0.0);
    for (int n = 1; n < P; n++) {
      const int b = n * n;
      auto cm = [&](int m) { return 0.5 * sqrt((double)(n - m) * (n + m + 1)); };
      auto re = [&](int m) { return m == 0 ? b : b + 2 * m - 1; };
      auto im = [&](int m) { return b + 2 * m; };
      for (int m = 0; m <= n; m++) {
        if (c == 2) {
          if (m > 0) { o[re(m)] = -m * v[im(m)]; o[im(m)] = m * v[re(m)]; }
          continue;
        }
        if (m == 0) {
          if (n >= 1) o[b] = (c == 0 ? 2 * cm(0) * v[im(1)] : -2 * cm(0) * v[re(1)]);
          continue;
        }
        double r = 0.0, i = 0.0;
        if (c == 0) {
          if (m >= 2) r += cm(m - 1) * v[im(m - 1)];
          if (m < n) r += cm(m) * v[im(m + 1)];
          i -= cm(m - 1) * v[re(m - 1)];
          if (m < n) i -= cm(m) * v[re(m + 1)];
        } else {
          r += cm(m - 1) * v[re(m - 1)];
          if (m < n) r -= cm(m) * v[re(m + 1)];
          if (m >= 2) i += cm(m - 1) * v[im(m - 1)];
          if (m < n) i -= cm(m) * v[im(m + 1)];
        }
        o[re(m)] = r; o[im(m)] = i;
      }
    }
  }
  // inner solve transposed (src/expcenter.cpp:1079-1135 at its fixed point): given
  // dU/dF, dU/dH of the solved sphere, returns dU/dLF, dU/dLH (each NP^2)
  void solve_T(const SphType &S, const vec &gF, const vec &gH, vec &gLF, vec &gLH) const
  {
    const int p = NP, p2 = p * p, n2 = 2 * p2;
    std::vector<double> A((size_t)n2 * n2, 0.0);   // A x = rhs, x = (F, H)
    std::vector<int> deg(p2);
    for (int n = 0; n < p; n++) for (int k = n * n; k < (n + 1) * (n + 1); k++) deg[k] = n;
    auto M = [&](int i, int kk) { return S.imat[(size_t)kk * p2 + i]; };
    for (int i = 0; i < p2; i++) {
      const double c3 = T.CONST3[deg[i]], ci = S.cInvH[deg[i]];
      for (int kk = 0; kk < p2; kk++) {
        const double m = M(i, kk);
        A[(size_t)i * n2 + kk] -= c3 * m * S.cF1[deg[kk]];
        A[(size_t)i * n2 + p2 + kk] -= c3 * m * S.cH1[deg[kk]];
        A[(size_t)(p2 + i) * n2 + kk] -= ci * m * S.cF2[deg[kk]];
        A[(size_t)(p2 + i) * n2 + p2 + kk] -= ci * m * S.cH2[deg[kk]];
      }
      A[(size_t)i * n2 + i] += 1.0;
      A[(size_t)(p2 + i) * n2 + p2 + i] += 1.0;
    }
    // solve A^T y = g by Gaussian elimination with partial pivoting
    std::vector<double> B((size_t)n2 * n2), y(n2);
    for (int r = 0; r < n2; r++) for (int c = 0; c < n2; c++) B[(size_t)r * n2 + c] = A[(size_t)c * n2 + r];
    for (int k = 0; k < p2; k++) { y[k] = k < (int)gF.size() ? gF[k] : 0.0; y[p2 + k] = k < (int)gH.size() ? gH[k] : 0.0; }
    for (int c = 0; c < n2; c++) {
      int piv = c;
      for (int r = c + 1; r < n2; r++) if (fabs(B[(size_t)r * n2 + c]) > fabs(B[(size_t)piv * n2 + c])) piv = r;
      if (piv != c) { for (int k = 0; k < n2; k++) std::swap(B[(size_t)c * n2 + k], B[(size_t)piv * n2 + k]); std::swap(y[c], y[piv]); }
      for (int r = c + 1; r < n2; r++) {
        const double f = B[(size_t)r * n2 + c] / B[(size_t)c * n2 + c];
        if (f == 0.0) continue;
        for (int k = c; k < n2; k++) B[(size_t)r * n2 + k] -= f * B[(size_t)c * n2 + k];
        y[r] -= f * y[c];
      }
    }
    for (int c = n2 - 1; c >= 0; c--) {
      double s = y[c];
      for (int k = c + 1; k < n2; k++) s -= B[(size_t)c * n2 + k] * y[k];
      y[c] = s / B[(size_t)c * n2 + c];
    }
    // y = dU/d(C3 M fb) and dU/d(CI M hb): back through M and the diagonal scalings
    vec gfb(p2, 0.0), ghb(p2, 0.0);
    for (int i = 0; i < p2; i++) {
      const double yf = y[i] * T.CONST3[deg[i]], yh = y[p2 + i] * S.cInvH[deg[i]];
      for (int kk = 0; kk < p2; kk++) { gfb[kk] += M(i, kk) * yf; ghb[kk] += M(i, kk) * yh; }
    }
    gLF.assign(p2, 0.0); gLH.assign(p2, 0.0);
    for (int k = 0; k < p2; k++) {
      const int n = deg[k];
      gLH[k] = S.cLH1[n] * gfb[k] + S.cLH2[n] * ghb[k];
      gLF[k] = S.cLF1[n] * gfb[k] + S.cLF2[n] * ghb[k];
    }
  }
  // intra near coupling of sphere kj (F, H) into sphere ki (LF, LH) with frozen
  // orders: analytic (sep >= 5) or numeric through the surface charges (sep < 5)
  void intra_maps(int i, int ki, int kj, LinMat &AF, LinMat &AH) const
  {
    const SphType &Si = st(i, ki), &Sj = st(i, kj);
    const SphState &Zj = mols[i].s[kj];
    const int p2 = NP * NP;
    P3 P = Si.cen - Sj.cen;
    const double rho = P.norm(), sep = rho - Si.rad - Sj.rad;
    const int pF = compute_order(NP, rho, Zj.tF, Sj.rad), pH = compute_order(NP, rho, Zj.tH, Sj.rad);
    if (sep > 0 && !(sep < 5)) {
      XForm X; X.reset_intra(T, P, pH, pF, Sj.rad, Si.rad);
      AF = lin_of(p2, p2, [&](const vec &x, vec &y) { X.xformF(x, y); });
      AH = lin_of(p2, p2, [&](const vec &x, vec &y) { X.xformH(x, y); });
      return;
    }
    const double dA = 4 * M_PI / double(Sj.nspx);
    auto numeric = [&](const vec &v, vec &L, bool kap) {
      L.assign(p2, 0.0);
      for (size_t h = 0; h < Sj.spx.size(); h++) {
        Sph q = cart2sph(Sj.spx[h]);
        vec Y; sph_harm(T, q.theta, q.phi, NP, Y);
        for (int n = 0; n < NP; n++)
          for (int m = 0; m < 2 * n + 1; m++) Y[IDX(n) + m] *= kap ? Sj.cChgH[n] : T.CONST2[n];
        const double qh = inprod_unit(v, Y) * dA;
        if (qh == 0.0) continue;
        vec Lh;
        add_local_charge(T, Lh, qh, Sj.spx[h] - P, kap, kap ? pH : pF, Si.rad);
        vacc(L, Lh);
      }
    };
    AF = lin_of(p2, p2, [&](const vec &x, vec &y) { numeric(x, y, false); });
    AH = lin_of(p2, p2, [&](const vec &x, vec &y) { numeric(x, y, true); });
  }
  // geometric part of one inter-molecular pair transform: L_tgt += T(P) v with
  // P = c_tgt - c_src, weighted by g = dU/dL_tgt; adds dU/dv into gv and the pose terms
  void pair_adjoint(int it, int kt, int is, int ks, int p, const vec &v, const vec &g, vec &gv,
                    std::vector<P3> &dpos, std::vector<P3> &drot) const
  {
    const int p2 = NP * NP;
    P3 P = cen_lab(it, kt) - cen_lab(is, ks);
    XForm X; X.reset(T, P, p, st(is, ks).rad, st(it, kt).rad, true);
    LinMat Tm = lin_of(p2, p2, [&](const vec &x, vec &y) { X.xformH(x, y); });
    vacc(gv, Tm.applyT(g));
    vec G[3];
    X.xformH_grad(v, G);
    const P3 gP(vdot(g, G[0]), vdot(g, G[1]), vdot(g, G[2]));
    dpos[it] = dpos[it] + gP; dpos[is] = dpos[is] - gP;
    drot[it] = drot[it] + cross(mols[it].s[kt].cenRot, gP);
    drot[is] = drot[is] - cross(mols[is].s[ks].cenRot, gP);
  }
  // dU/dpos and dU/domega (lab frame) of total_energy_lab after compute_forces
  void backward(std::vector<P3> &dpos, std::vector<P3> &drot, int max_its = 2000) const
  {
    const int nmol = mols.size(), p2 = NP * NP;
    dpos.assign(nmol, P3()); drot.assign(nmol, P3());
    std::vector<LinMat> RF(nmol), RB(nmol);
    for (int i = 0; i < nmol; i++) { RF[i] = rot_mat(mols[i].orient, true); RB[i] = rot_mat(mols[i].orient, false); }
    // derivatives of the molecule rotations for a lab-frame turn about axis c:
    // d(RF v) = J_c RF v, d(RB v) = -RB J_c v
    auto dRFv = [&](int i, int c, const vec &v) { vec o; rot_generator(c, RF[i].apply(v), o, NP); return o; };
    auto dRBv = [&](int i, int c, const vec &v) {
      vec o; rot_generator(c, v, o, NP);
      vec r = RB[i].apply(o);
      for (double &x : r) x = -x;
      return r;
    };
    std::vector<std::vector<vec> > Hl(nmol), gHl(nmol), gH(nmol);
    for (int i = 0; i < nmol; i++) {
      Hl[i].resize(mols[i].s.size()); gHl[i].assign(mols[i].s.size(), vec(p2, 0.0)); gH[i] = gHl[i];
      for (size_t k = 0; k < mols[i].s.size(); k++) Hl[i][k] = RF[i].apply(trunc_or_pad(mols[i].s[k].H, NP));
    }
    // energy
    for (int i = 0; i < nmol; i++)
      for (int j = i + 1; j < nmol; j++)
        for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
          const SphType &Si = st(i, ki);
          const SphState &Zi = mols[i].s[ki];
          vec a(p2);
          const double fact = 1 / (Zi.hscale * Si.rad);
          double sc = 1.0;
          for (int n = 0; n < NP; n++, sc *= fact)
            for (int m = 0; m < 2 * n + 1; m++) a[IDX(n) + m] = (m == 0 ? 1.0 : 2.0) * sc;
          vec wi(p2);
          for (int k = 0; k < p2; k++) wi[k] = a[k] * Hl[i][ki][k];
          for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
            const SphType &Sj = st(j, kj);
            const SphState &Zj = mols[j].s[kj];
            P3 P = cen_lab(i, ki) - cen_lab(j, kj);
            const double rho = P.norm();
            int pi2j = compute_order(NP, rho, Zi.tH, Si.rad), pj2i = compute_order(NP, rho, Zj.tH, Sj.rad);
            const int minp = pi2j < pj2i ? pi2j : pj2i;
            XForm X; X.reset(T, P, minp, Sj.rad, Si.rad, false);
            vec L; X.xformH(Hl[j][kj], L);
            for (int k = 0; k < (int)L.size(); k++) gHl[i][ki][k] += a[k] * L[k];
            pair_adjoint(i, ki, j, kj, minp, Hl[j][kj], wi, gHl[j][kj], dpos, drot);
          }
        }
    // Hlab = RF H
    for (int i = 0; i < nmol; i++)
      for (size_t k = 0; k < mols[i].s.size(); k++) {
        const vec H = trunc_or_pad(mols[i].s[k].H, NP);
        for (int c = 0; c < 3; c++) {
          const double d = vdot(gHl[i][k], dRFv(i, c, H));
          if (c == 0) drot[i].x += d; else if (c == 1) drot[i].y += d; else drot[i].z += d;
        }
        gH[i][k] = RF[i].applyT(gHl[i][k]);
      }
    // the intra-molecular fixed point over the polarized spheres (stage 2)
    std::vector<std::pair<int, int> > P;
    std::map<std::pair<int, int>, int> idx;
    for (int i = 0; i < nmol; i++)
      if (mols[i].interXForm)
        for (size_t k = 0; k < mols[i].s.size(); k++)
          if (!mols[i].s[k].interPol.empty()) { idx[{i, (int)k}] = P.size(); P.push_back({i, (int)k}); }
    const int nP = P.size();
    std::vector<std::vector<std::pair<int, std::pair<LinMat, LinMat> > > > Ain(nP);   // s <- (s2, AF, AH)
    for (int u = 0; u < nP; u++) {
      const int i = P[u].first, ki = P[u].second;
      for (int kj : st(i, ki).near) {
        auto it = idx.find({i, kj});
        if (it == idx.end()) continue;
        LinMat AF, AH;
        intra_maps(i, ki, kj, AF, AH);
        Ain[u].push_back({it->second, {AF, AH}});
      }
    }
    // transposed fixed point lambda_v = g_v + sum_u A_uv^T S_u^T lambda_u, swept in the
    // reverse of the forward sphere order with the latest values (Gauss-Seidel on the
    // transposed system; the forward's splitting converges, Jacobi need not)
    std::vector<std::vector<std::pair<int, int> > > Aout(nP);   // v -> (u, index in Ain[u])
    for (int u = 0; u < nP; u++)
      for (size_t e = 0; e < Ain[u].size(); e++) Aout[Ain[u][e].first].push_back({u, (int)e});
    std::vector<vec> lF(nP, vec(p2, 0.0)), lH(nP), mF(nP), mH(nP);
    for (int u = 0; u < nP; u++) {
      lH[u] = gH[P[u].first][P[u].second];
      solve_T(st(P[u].first, P[u].second), lF[u], lH[u], mF[u], mH[u]);
    }
    for (int it = 0; it < max_its; it++) {
      double dn = 0.0, nn = 0.0;
      for (int v = nP - 1; v >= 0; v--) {
        vec nF(p2, 0.0), nH = gH[P[v].first][P[v].second];
        for (auto &ue : Aout[v]) {
          const auto &A = Ain[ue.first][ue.second].second;
          vacc(nF, A.first.applyT(mF[ue.first]));
          vacc(nH, A.second.applyT(mH[ue.first]));
        }
        for (int k = 0; k < p2; k++) {
          dn += (nF[k] - lF[v][k]) * (nF[k] - lF[v][k]) + (nH[k] - lH[v][k]) * (nH[k] - lH[v][k]);
          nn += nF[k] * nF[k] + nH[k] * nH[k];
        }
        lF[v] = nF; lH[v] = nH;
        solve_T(st(P[v].first, P[v].second), lF[v], lH[v], mF[v], mH[v]);
      }
      if (dn <= 1e-30 * nn) break;
    }
    // stage-2 LS: LS = RB(sum T(Hrot)); its dU/dLS is the LH part of mu
    std::vector<std::vector<vec> > gHrot(nmol);
    for (int i = 0; i < nmol; i++) gHrot[i].assign(mols[i].s.size(), vec(p2, 0.0));
    for (int u = 0; u < nP; u++) {
      const int i = P[u].first, ki = P[u].second;
      const SphState &Z = mols[i].s[ki];
      vec LSrot(p2, 0.0);
      for (auto &e : Z.interPol) {
        const SphState &Zm = mols[e.first].s[e.second];
        P3 Pv = cen_lab(i, ki) - cen_lab(e.first, e.second);
        const int p = compute_order(NP, Pv.norm(), Zm.tH, st(e.first, e.second).rad);
        XForm X; X.reset(T, Pv, p, st(e.first, e.second).rad, st(i, ki).rad, false);
        vec t; X.xformH(trunc_or_pad(Zm.Hrot, NP), t); vacc(LSrot, t);
      }
      const vec gLSrot = RB[i].applyT(mH[u]);
      for (int c = 0; c < 3; c++) {
        const double d = vdot(mH[u], dRBv(i, c, LSrot));
        if (c == 0) drot[i].x += d; else if (c == 1) drot[i].y += d; else drot[i].z += d;
      }
      for (auto &e : Z.interPol) {
        const SphState &Zm = mols[e.first].s[e.second];
        P3 Pv = cen_lab(i, ki) - cen_lab(e.first, e.second);
        const int p = compute_order(NP, Pv.norm(), Zm.tH, st(e.first, e.second).rad);
        pair_adjoint(i, ki, e.first, e.second, p, trunc_or_pad(Zm.Hrot, NP), gLSrot, gHrot[e.first][e.second], dpos, drot);
      }
    }
    // Hrot = RF H1 (stage 1), H1 = RB Hrot
    std::vector<std::vector<vec> > gHsr(nmol);
    for (int i = 0; i < nmol; i++) gHsr[i].assign(mols[i].s.size(), vec(p2, 0.0));
    for (int u = 0; u < nP; u++) {
      const int i = P[u].first, ki = P[u].second;
      const SphState &Z = mols[i].s[ki];
      const vec H1 = RB[i].apply(trunc_or_pad(Z.Hrot, NP));
      for (int c = 0; c < 3; c++) {
        const double d = vdot(gHrot[i][ki], dRFv(i, c, H1));
        if (c == 0) drot[i].x += d; else if (c == 1) drot[i].y += d; else drot[i].z += d;
      }
      const vec gH1 = RF[i].applyT(gHrot[i][ki]);
      vec g1F, g1H;
      solve_T(st(i, ki), vec(p2, 0.0), gH1, g1F, g1H);
      // stage-1 LS from the neighbours' rotated self H
      vec LSrot(p2, 0.0);
      for (auto &e : Z.interPol) {
        const SphType &Sm = st(e.first, e.second);
        P3 Pv = cen_lab(i, ki) - cen_lab(e.first, e.second);
        const int p = compute_order(NP, Pv.norm(), Sm.tHself, Sm.rad);
        XForm X; X.reset(T, Pv, p, Sm.rad, st(i, ki).rad, false);
        vec t; X.xformH(trunc_or_pad(mols[e.first].s[e.second].HselfRot, NP), t); vacc(LSrot, t);
      }
      const vec gLSrot = RB[i].applyT(g1H);
      for (int c = 0; c < 3; c++) {
        const double d = vdot(g1H, dRBv(i, c, LSrot));
        if (c == 0) drot[i].x += d; else if (c == 1) drot[i].y += d; else drot[i].z += d;
      }
      for (auto &e : Z.interPol) {
        const SphType &Sm = st(e.first, e.second);
        P3 Pv = cen_lab(i, ki) - cen_lab(e.first, e.second);
        const int p = compute_order(NP, Pv.norm(), Sm.tHself, Sm.rad);
        pair_adjoint(i, ki, e.first, e.second, p, trunc_or_pad(mols[e.first].s[e.second].HselfRot, NP), gLSrot,
                     gHsr[e.first][e.second], dpos, drot);
      }
    }
    // HselfRot = RF Hself
    for (int i = 0; i < nmol; i++)
      for (size_t k = 0; k < mols[i].s.size(); k++) {
        bool any = false;
        for (double x : gHsr[i][k]) if (x != 0.0) { any = true; break; }
        if (!any) continue;
        const vec Hs = trunc_or_pad(st(i, k).Hself, NP);
        for (int c = 0; c < 3; c++) {
          const double d = vdot(gHsr[i][k], dRFv(i, c, Hs));
          if (c == 0) drot[i].x += d; else if (c == 1) drot[i].y += d; else drot[i].z += d;
        }
      }
  }

  // ---------------------------------------------------------------- Brownian dynamics
  // The Ermak-McCammon step of the reference's drivers: CBDnam::run / makeMove /
  // compute_dt (src/BDnam.cpp:166-417) and CBDmulti::propagate / makeMove /
  // compute_dt / computeMinSepDist (src/BDmulti.cpp:396-566).  Noise: Philox4x64-10
  // (Salmon et al., SC 2011), key (seed, 0), counter (draw, system, 0, 0), four
  // uniforms ((x >> 11) + 0.5) 2^-53 and the Box-Muller transform give one random
  // vector (the reference draws from drand48 with the polar method).
  struct BD {
    int mode = 0, max_tries = 500;
    double force_dist = 100, escape_dist = 500, dt_min = 2, dt_max = 1e300, dt_ref = 5, dt_div = 15;
    double fact_tr = 5.604586e2, ikbt = 1.0 / (1.3806503e-23 * 298.15), coul_k = 2.30708e-18;
    unsigned long long seed = 0, ctr = 0;
    int sys = 0, status = 0, steps = 0, fevals = 0;
    double time = 0;
    std::vector<double> dtr, drot;
    std::vector<Quat> rot;
    // noise 0: Philox4x64-10 (the CUDA path's generator); noise 1: the reference's
    // own stream, drand48 seeded by srand48(seed) with the polar Box-Muller method
    // of normRand (src/util.h:489-539), the three deviates of a vector drawn in
    // argument order `order` (0: x first, 1: z first)
    int noise = 0, order = 0;
    unsigned long long lcg = 0;
    bool nr_saved = false;
    double nr_value = 0.0;
  } bd;

  // drand48 (POSIX): X <- (0x5DEECE66D X + 0xB) mod 2^48, returns X / 2^48
  double drand()
  {
    bd.lcg = (0x5DEECE66DULL * bd.lcg + 0xBULL) & ((1ULL << 48) - 1);
    return (double)bd.lcg / 281474976710656.0;
  }
  double norm_rand()   // normRand, src/util.h:515-539
  {
    if (!bd.nr_saved) {
      double v1, v2, rsq;
      do {
        v1 = 2.0 * drand() - 1.0;
        v2 = 2.0 * drand() - 1.0;
        rsq = v1 * v1 + v2 * v2;
      } while (rsq >= 1.0 || rsq == 0.0);
      const double fac = sqrt(-2.0 * log(rsq) / rsq);
      bd.nr_value = v1 * fac;
      bd.nr_saved = true;
      return fac * v2;
    }
    bd.nr_saved = false;
    return bd.nr_value;
  }

  static void philox(unsigned long long c[4], unsigned long long k0, unsigned long long k1)
  {
    const unsigned long long M0 = 0xD2E7470EE14C6C93ULL, M1 = 0xCA5A826395121157ULL;
    const unsigned long long W0 = 0x9E3779B97F4A7C15ULL, W1 = 0xBB67AE8584CAA73BULL;
    for (int r = 0; r < 10; r++) {
      if (r) { k0 += W0; k1 += W1; }
      unsigned __int128 p0 = (unsigned __int128)M0 * c[0], p1 = (unsigned __int128)M1 * c[2];
      unsigned long long hi0 = (unsigned long long)(p0 >> 64), lo0 = (unsigned long long)p0;
      unsigned long long hi1 = (unsigned long long)(p1 >> 64), lo1 = (unsigned long long)p1;
      unsigned long long n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
      c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
  }
  P3 rand_vec(double sd)   // CBDnam::getRandVec (src/BDnam.h:44-45)
  {
    if (bd.noise == 1) {
      double a, b, c;
      if (bd.order == 0) { a = norm_rand(); b = norm_rand(); c = norm_rand(); }
      else { c = norm_rand(); b = norm_rand(); a = norm_rand(); }
      return sd * P3(a, b, c);
    }
    unsigned long long c[4] = {bd.ctr++, (unsigned long long)bd.sys, 0ULL, 0ULL};
    philox(c, bd.seed, 0ULL);
    double u[4];
    for (int i = 0; i < 4; i++) u[i] = ((double)(c[i] >> 11) + 0.5) * 0x1p-53;
    const double r0 = sqrt(-2.0 * log(u[0])), r1 = sqrt(-2.0 * log(u[2]));
    return sd * P3(r0 * cos(2.0 * M_PI * u[1]), r0 * sin(2.0 * M_PI * u[1]), r1 * cos(2.0 * M_PI * u[3]));
  }
  static Quat qraw(double w, const P3 &v) { Quat q; q.w = w; q.v = v; return q; }
  static Quat qmul(const Quat &a, const Quat &b)   // a * b: b *= a (src/util.h:242-263)
  {
    return qraw(a.w * b.w - dot(a.v, b.v), (a.w * b.v + b.w * a.v) + cross(a.v, b.v));
  }
  static Quat axis_angle(const P3 &ax, double angle)   // CQuat(axis, angle), src/util.h:220-229
  {
    if (angle != 0.0 && ax.norm2() != 0.0) return Quat(cos(0.5 * angle), sin(0.5 * angle) * ((1.0 / ax.norm()) * ax));
    return Quat();
  }
  double c2c(int i, int j) const { return (mols[i].rcen - mols[j].rcen).norm(); }
  double mol_gap(int i, int j) const
  {
    return c2c(i, j) - types[mols[i].type].maxR - types[mols[j].type].maxR;
  }
  void rotate(int i, const Quat &dq)   // CMolecule::rotate (src/moldynamics.cpp:666-679)
  {
    Molecule &M = mols[i];
    M.orient = qmul(dq, M.orient);
    for (size_t k = 0; k < M.s.size(); k++) M.s[k].cenRot = qrot(M.orient, st(i, k).cen);
  }
  bool is_collided(int i) const   // src/moldynamics.cpp:167-193
  {
    for (size_t j = 0; j < mols.size(); j++) {
      if ((int)j == i || mol_gap(i, j) > 0) continue;
      for (size_t ki = 0; ki < mols[i].s.size(); ki++)
        for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
          P3 d = ((mols[i].rcen + mols[i].s[ki].cenRot) - mols[j].rcen) - mols[j].s[kj].cenRot;
          if ((d.norm() - st(i, ki).rad) - st(j, kj).rad < 0.0) return true;
        }
    }
    return false;
  }
  bool will_rot_collide(int i, const Quat &dq) const   // src/moldynamics.cpp:43-85
  {
    const Quat Q = qmul(dq, mols[i].orient);
    for (size_t j = 0; j < mols.size(); j++) {
      if ((int)j == i || mol_gap(i, j) > 0) continue;
      for (size_t ki = 0; ki < mols[i].s.size(); ki++) {
        const P3 cki = mols[i].rcen + qrot(Q, st(i, ki).cen);
        for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
          P3 d = (cki - mols[j].rcen) - mols[j].s[kj].cenRot;
          if ((st(i, ki).rad + st(j, kj).rad) - d.norm() > 0.0) return true;
        }
      }
    }
    return false;
  }
  double bd_dt(double d) const
  {
    double dt = (d - bd.dt_ref > 0) ? bd.dt_min + (d - bd.dt_ref) / bd.dt_div : bd.dt_min;
    return dt < bd.dt_max ? dt : bd.dt_max;
  }
  int translate_try(int i, const P3 &drift, double sd)
  {
    int c = 0;
    bool done = false;
    while (!done && c < bd.max_tries) {
      c++;
      const P3 old = mols[i].rcen;
      mols[i].rcen = mols[i].rcen + (drift + rand_vec(sd));
      if (is_collided(i)) mols[i].rcen = old;
      else done = true;
    }
    return c;
  }
  int rotate_try(int i, const P3 &drift, double sd, Quat &last)
  {
    int c = 0;
    bool done = false;
    while (!done && c < bd.max_tries) {
      c++;
      const P3 o = drift + rand_vec(sd);
      last = axis_angle(o, o.norm());
      if (!will_rot_collide(i, last)) { rotate(i, last); done = true; }
    }
    return c;
  }
  // one step; returns false when a needed force evaluation failed
  bool bd_step()
  {
    const int nmol = mols.size();
    if (bd.status != 0) return true;
    double dt, md = 0;
    bool need;
    if (bd.mode == 0) {
      dt = bd_dt(mol_gap(0, 1));
      need = c2c(0, 1) < bd.force_dist;
    } else {
      // as bdm runs it: CBDmulti::initConstants (src/BDmulti.cpp:26-38) runs before the
      // molecules set CMolecule::m_interactRcutoff (still DBL_MAX, src/molecule.cpp:26),
      // so every pair is tracked sphere by sphere, floored at DISTCUTOFF_TIME
      const double ic = prm.interact_cut;
      const double maxd = 1e300, mind = bd.dt_ref;
      double smin = 1e300, mmin = 1e300;
      bool track = false;
      for (int i = 0; i < nmol; i++)
        for (int j = i + 1; j < nmol; j++) {
          const double dm = mol_gap(i, j);
          if (dm < maxd) {
            track = true;
            for (size_t ki = 0; ki < mols[i].s.size(); ki++)
              for (size_t kj = 0; kj < mols[j].s.size(); kj++) {
                P3 d = ((mols[i].rcen + mols[i].s[ki].cenRot) - mols[j].rcen) - mols[j].s[kj].cenRot;
                const double g = (d.norm() - st(i, ki).rad) - st(j, kj).rad;
                if (g < smin) smin = g;
              }
          } else if (dm < mmin) mmin = dm;
        }
      md = track ? (smin < mind ? mind : smin) : (mmin > 0 ? mmin : 0);
      dt = bd_dt(md);
      need = md < ic;
    }
    std::vector<P3> F(nmol), T(nmol);
    if (need) {
      bd.fevals++;
      if (!compute_forces(F, T)) { bd.status = 4; return false; }
    }
    int status = 0;
    if (bd.mode == 0) {
      P3 dR, dO1, dO2;
      if (need) {
        dR = ((bd.dtr[1] * dt) * bd.fact_tr) * F[1];
        dO1 = (((bd.drot[0] * dt) * bd.ikbt) * bd.coul_k) * T[0];
        dO2 = (((bd.drot[1] * dt) * bd.ikbt) * bd.coul_k) * T[1];
      }
      const double bdist = c2c(0, 1);
      const int ct = translate_try(1, dR, sqrt(2 * dt * bd.dtr[1]));
      if (ct == bd.max_tries) status = 2;
      else if (c2c(0, 1) > bd.escape_dist) status = 1;
      if (status == 0) {
        const double s1 = sqrt(2 * dt * bd.drot[0]), s2 = sqrt(2 * dt * bd.drot[1]);
        const P3 o1 = dO1 + rand_vec(s1), o2 = dO2 + rand_vec(s2);
        const Quat Q1 = axis_angle(o1, o1.norm()), Q2 = axis_angle(o2, o2.norm());
        const double adist = c2c(0, 1);
        if (adist > bd.force_dist) {
          bd.rot[0] = qmul(Q1, bd.rot[0]);
          bd.rot[1] = qmul(Q2, bd.rot[1]);
        } else if (bdist > bd.force_dist) {
          rotate(0, bd.rot[0]);
          rotate(1, bd.rot[1]);
          bd.rot[0] = Quat(); bd.rot[1] = Quat();
        } else {
          for (int i = 0; i < 2 && status == 0; i++) {
            Quat last;
            if (rotate_try(i, i ? dO2 : dO1, i ? s2 : s1, last) == bd.max_tries) {
              bd.rot[i] = qmul(last, bd.rot[i]);
              status = 2;
            }
          }
        }
      }
    } else {
      for (int i = 0; i < nmol; i++) {
        P3 dR, dO;
        if (need) {
          dR = ((bd.dtr[i] * dt) * bd.fact_tr) * F[i];
          dO = (((bd.drot[i] * dt) * bd.ikbt) * bd.coul_k) * T[i];
        }
        translate_try(i, dR, sqrt(2 * dt * bd.dtr[i]));
        Quat last;
        rotate_try(i, dO, sqrt(2 * dt * bd.drot[i]), last);
      }
    }
    bd.status = status;
    bd.steps++;
    bd.time += dt;
    return true;
  }
};

}  // namespace orc

// ---------------------------------------------------------------------------
// entry point: same spec and output format as oracle/ref_harness.cpp, plus
//   poles <P>      tol <max_polar_dev> <solve_tol> <solve_max_ct> <max_pol_rounds>
extern "C" int pbsam_oracle_run(const char *spec_path, const char *out_path)
{
  using namespace orc;
  std::ifstream in(spec_path);
  if (!in) return 2;
  Params prm;
  int NP = 10, dump = 0, energy = 1, backward = 0, nograd = 0, exact = 0, potlab = 0;
  std::vector<P3> potpts;
  std::vector<std::vector<std::string> > types;
  struct PoseL { int type; double v[7]; };
  std::vector<std::vector<PoseL> > frames;
  int bdmode = -1, bdsteps = 0, bdsys = 0, bdnoise = 0, bdorder = 0;
  unsigned long long bdseed = 0;
  double bdp[7] = {500, 100, 500, 2, 1e300, 5, 15};   // max_tries, force, escape, dt_min, dt_max, dt_ref, dt_div
  std::vector<double> bddtr, bddrot;
  std::string tok;
  while (in >> tok) {
    if (tok == "salt") in >> prm.salt;
    else if (tok == "idiel") in >> prm.idiel;
    else if (tok == "dump") in >> dump;
    else if (tok == "energy") in >> energy;
    else if (tok == "backward") in >> backward;
    else if (tok == "nograd") in >> nograd;
    else if (tok == "exact") in >> exact;
    else if (tok == "potpoint") { double x, y, z; in >> x >> y >> z; potpts.push_back(P3(x, y, z)); }
    else if (tok == "potlab") in >> potlab;
    else if (tok == "poles") in >> NP;
    else if (tok == "tol") in >> prm.max_polar_dev >> prm.solve_tol >> prm.solve_max_ct >> prm.max_pol_rounds;
    else if (tok == "moltype") { std::vector<std::string> t(4); in >> t[0] >> t[1] >> t[2] >> t[3]; types.push_back(t); }
    else if (tok == "frame") frames.push_back(std::vector<PoseL>());
    else if (tok == "mol") { PoseL p; in >> p.type; for (int k = 0; k < 7; k++) in >> p.v[k]; frames.back().push_back(p); }
    else if (tok == "bd") in >> bdmode >> bdsteps >> bdseed >> bdsys;
    else if (tok == "bdp") in >> bdp[0] >> bdp[1] >> bdp[2] >> bdp[3] >> bdp[4] >> bdp[5] >> bdp[6];
    else if (tok == "bddiff") { double a, b; in >> a >> b; bddtr.push_back(a); bddrot.push_back(b); }
    else if (tok == "bdnoise") in >> bdnoise >> bdorder;
    else return 2;
  }
  System sys;
  sys.prm = prm;
  sys.NP = NP;
  sys.skip_grad = nograd != 0;
  sys.exact_inner = exact != 0;
  const double kappa = kappa_of_salt(prm.salt, prm.sdiel, prm.temperature);
  sys.T.init(NP, kappa);
  sys.types.resize(types.size());
  for (size_t t = 0; t < types.size(); t++)
    if (!build_moltype(sys.T, prm, sys.types[t], types[t][0].c_str(), types[t][1].c_str(), types[t][2].c_str(),
                       types[t][3].c_str())) return 3;
  FILE *out = fopen(out_path, "w");
  if (!out) return 2;
  fprintf(out, "KAPPA %.17e\n", kappa);
  for (auto &p : frames[0]) sys.add_molecule(p.type);
  if (bdmode >= 0) {
    // Brownian dynamics from the first frame's poses: one BDSTEP block per step
    for (size_t i = 0; i < frames[0].size(); i++) {
      const double *v = frames[0][i].v;
      sys.set_pose(i, P3(v[0], v[1], v[2]), Quat(v[3], P3(v[4], v[5], v[6])));
    }
    System::BD &B = sys.bd;
    B.mode = bdmode; B.seed = bdseed; B.sys = bdsys;
    B.noise = bdnoise; B.order = bdorder;
    B.lcg = (((unsigned long long)bdseed & 0xFFFFFFFFULL) << 16) | 0x330EULL;   // srand48(seed)
    B.max_tries = (int)bdp[0]; B.force_dist = bdp[1]; B.escape_dist = bdp[2];
    B.dt_min = bdp[3]; B.dt_max = bdp[4]; B.dt_ref = bdp[5]; B.dt_div = bdp[6];
    B.dtr = bddtr; B.drot = bddrot;
    B.rot.assign(sys.mols.size(), Quat());
    if (bddtr.size() != sys.mols.size()) { fclose(out); return 2; }
    for (int k = 0; k < bdsteps; k++) {
      sys.bd_step();
      fprintf(out, "BDSTEP %d %d %d %.17e\n", B.steps, B.status, B.fevals, B.time);
      for (size_t i = 0; i < sys.mols.size(); i++) {
        const Molecule &M = sys.mols[i];
        fprintf(out, "POSE %d %.17e %.17e %.17e %.17e %.17e %.17e %.17e\n", (int)i, M.rcen.x, M.rcen.y, M.rcen.z,
                M.orient.w, M.orient.v.x, M.orient.v.y, M.orient.v.z);
      }
    }
    fclose(out);
    return 0;
  }
  for (size_t f = 0; f < frames.size(); f++) {
    for (size_t i = 0; i < frames[f].size(); i++) {
      const double *v = frames[f][i].v;
      sys.set_pose(i, P3(v[0], v[1], v[2]), Quat(v[3], P3(v[4], v[5], v[6])));
    }
    std::vector<P3> force, torque;
    bool ok = sys.compute_forces(force, torque);
    fprintf(out, "FRAME %d %d 0 sweeps %d inner %ld solves %ld\n", (int)f, ok ? 1 : 0, sys.n_sweeps, sys.n_inner, sys.n_solves);
    if (!ok) continue;
    for (size_t i = 0; i < force.size(); i++) {
      fprintf(out, "FORCE %d %.17e %.17e %.17e\n", (int)i, force[i].x, force[i].y, force[i].z);
      fprintf(out, "TORQUE %d %.17e %.17e %.17e\n", (int)i, torque[i].x, torque[i].y, torque[i].z);
    }
    if (energy) fprintf(out, "ENERGY %.17e\n", sys.total_energy());
    if (energy > 1) fprintf(out, "ENERGYLAB %.17e\n", sys.total_energy_lab());
    for (size_t k = 0; k < potpts.size(); k++)
      fprintf(out, "POT %d %.17e\n", (int)k, sys.potential(potpts[k], potlab != 0));
    if (backward) {
      std::vector<P3> dpos, drot;
      sys.backward(dpos, drot);
      for (size_t i = 0; i < dpos.size(); i++) {
        fprintf(out, "DPOS %d %.17e %.17e %.17e\n", (int)i, dpos[i].x, dpos[i].y, dpos[i].z);
        fprintf(out, "DROT %d %.17e %.17e %.17e\n", (int)i, drot[i].x, drot[i].y, drot[i].z);
      }
    }
    if (dump)
      for (size_t i = 0; i < sys.mols.size(); i++)
        for (size_t ki = 0; ki < sys.mols[i].s.size(); ki++) {
          const SphState &Z = sys.mols[i].s[ki];
          auto pr = [&](const char *tag, const vec &v) {
            fprintf(out, "%s %d %d %d", tag, (int)i, (int)ki, (int)v.size());
            for (double x : v) fprintf(out, " %.17e", x);
            fprintf(out, "\n");
          };
          pr("F", Z.F); pr("H", Z.H); pr("LS", Z.LS);
          pr("GLHN0", Z.gLHN[0]); pr("GLHN1", Z.gLHN[1]); pr("GLHN2", Z.gLHN[2]);
          pr("GH0", Z.gH[0]); pr("GH1", Z.gH[1]); pr("GH2", Z.gH[2]);
        }
    fflush(out);
  }
  fclose(out);
  return 0;
}

// one Philox4x64-10 block in place (pins the noise generator against an
// independent implementation in the tests)
extern "C" void pbsam_oracle_philox(unsigned long long *c, unsigned long long k0, unsigned long long k1)
{
  orc::System::philox(c, k0, k1);
}

// Single-expansion operations (the tests of the CUDA pbsam_expan_* entry points):
// op 0 rotate (Rot::reset(theta, phi, xi) + rotate, or rotate_xi when f1; forward when f2;
// src/rotcoeff.cpp:155-171, 250-441), op 1 translate (Trans::reset with kappa or 0 when
// f1 is 0, translate or its derivative when f2; src/transcoeff.cpp:172-364), op 2
// re-expand (XForm::reset + xformH, or reset_intra + xformF when f1 is 0, with the
// gradient xformH_grad when grad is given; src/xforms.cpp:50-132, 213-270).  args as
// the CUDA entry points; in, out [n][np^2], grad [n][3][np^2].
extern "C" int pbsam_oracle_expan(int np, double kappa, int op, int n, const double *args, int p, int f1, int f2,
                                  const double *in, double *out, double *grad)
{
  using namespace orc;
  if (np < 1 || p < 1 || p > np || op < 0 || op > 2) return 1;
  Tables T;
  T.init(np, kappa);
  const int NP2 = np * np;
  auto put = [&](const vec &v, double *dst) {
    for (int k = 0; k < NP2; k++) dst[k] = k < (int)v.size() ? v[k] : 0.0;
  };
  for (int i = 0; i < n; i++) {
    const vec x(in + (size_t)i * NP2, in + (size_t)(i + 1) * NP2);
    vec y;
    if (op == 0) {
      const double *a = args + 3 * (size_t)i;
      Rot R;
      R.reset(T, a[0], a[1], a[2], p, false);
      if (f1) R.rotate_xi(x, y, p, f2 != 0);
      else R.rotate(x, y, p, f2 != 0);
    } else if (op == 1) {
      const double *a = args + 3 * (size_t)i;
      Trans Tr;
      Tr.init_scale(np, a[1], a[2]);
      Tr.reset(T, a[0], f1 ? T.kappa : 0.0, p, f2 != 0);
      Tr.translate(x, y, f2 != 0);
    } else {
      const double *a = args + 5 * (size_t)i;
      const P3 P(a[0], a[1], a[2]);
      XForm X;
      if (f1) {
        X.reset(T, P, p, a[3], a[4], grad != nullptr);
        X.xformH(x, y);
        if (grad) {
          vec G[3];
          X.xformH_grad(x, G);
          for (int c = 0; c < 3; c++) put(G[c], grad + ((size_t)i * 3 + c) * NP2);
        }
      } else {
        X.reset_intra(T, P, p, p, a[3], a[4]);
        X.xformF(x, y);
      }
    }
    put(y, out + (size_t)i * NP2);
  }
  return 0;
}
