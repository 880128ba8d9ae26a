// Device math for the PB-SAM mutual-polarization drop-in (sm_100a, FP64).
//
// Every routine here is executed cooperatively by a Team (the threads that own
// one independent system).  Intermediate tables live in per-team global scratch
// (L2-resident); team.sync() orders all global/shared accesses of the team.
//
// Expansion layout (the reference's packed real layout, src/expansion.h:509-553):
// degree n occupies [n*n, n*n + 2n]; entry 0 of a degree is m = 0, entries
// 2m-1 / 2m hold Re / Im of order m > 0.  NP = pole order of the context.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pbsam {

#define PB_PI 3.14159265358979323846

struct Team {
  int rank, size;
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};
// one warp working alone on an object (rank = lane, size = 32): the functions
// templated on the team type run with either
struct WarpTeam {
  int rank, size;
  __device__ __forceinline__ void sync() const { __syncwarp(); }
};

// Constant tables of one context (built on the host by the same formulas as
// src/expansion.cpp:39-96, src/rotcoeff.cpp:15-33, 949-983,
// src/transcoeff.cpp:15-38, src/expcenter.cpp:186-210).
struct Tab {
  int NP;
  double kappa;
  const double *C1, *C2, *C3;   // [2NP][2NP]  Legendre recurrence / SH normalisation
  const double *C4, *C6;        // [2NP]       k-hat recurrence 1/((2n-1)(2n-3)); (2n-1)!!
  const double *zeta;           // [2NP][2NP]
  const double *eta;            // [2NP][4NP-1], column 2NP-1+m
  const double *alpha, *beta;   // [2NP][NP]
  const double *gam, *del;      // [2NP][2NP-1], column NP-1+m
  const double *Q;              // [2NP-1][NP][2]
  const double *CONST2, *CONST3;// [NP]: (2l+1)/4pi, 1/(2l+1)
  __device__ __forceinline__ double c1(int n, int m) const { return C1[n * 2 * NP + m]; }
  __device__ __forceinline__ double c2(int n, int m) const { return C2[n * 2 * NP + m]; }
  __device__ __forceinline__ double c3(int n, int m) const { return C3[n * 2 * NP + m]; }
  __device__ __forceinline__ double ZETA(int n, int m) const { return zeta[n * 2 * NP + m]; }
  __device__ __forceinline__ double ETA(int n, int m) const { return eta[n * (4 * NP - 1) + 2 * NP - 1 + m]; }
  __device__ __forceinline__ double ALPHA(int n, int m) const { return alpha[n * NP + m]; }
  __device__ __forceinline__ double BETA(int n, int m) const { return beta[n * NP + m]; }
  __device__ __forceinline__ double GAMMA(int n, int m) const { return gam[n * (2 * NP - 1) + NP - 1 + m]; }
  __device__ __forceinline__ double DELTA(int n, int m) const { return del[n * (2 * NP - 1) + NP - 1 + m]; }
  __device__ __forceinline__ double MQ(int n, int m, int k) const { return Q[(n * NP + m) * 2 + k]; }
};

__device__ __forceinline__ int IDX(int n) { return n * n; }

// ---------------------------------------------------------------- complex
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
// complex division a / r for real r (std::complex operator/ with a real divisor)
__device__ __forceinline__ double2 cdivr(double2 a, double r) { return make_double2(a.x / r, a.y / r); }

// ---------------------------------------------------------------- geometry
struct Sph { double rho, theta, phi; };
__device__ __forceinline__ Sph cart2sph(double x, double y, double z)   // src/util.h:418-438
{
  Sph s;
  s.rho = sqrt(x * x + y * y + z * z);
  if (s.rho < fabs(z)) s.rho = fabs(z);
  s.theta = (s.rho == 0.0) ? 0.0 : acos(z / s.rho);
  s.phi = (x == 0.0 && y == 0.0) ? 0.0 : atan2(y, x);
  return s;
}

// rotate v by unit quaternion (w, qx, qy, qz) (src/util.h:463-468)
__device__ __forceinline__ void qrot(const double *q, const double *r, double *o)
{
  double qr0 = q[2] * r[2] - q[3] * r[1], qr1 = q[3] * r[0] - q[1] * r[2], qr2 = q[1] * r[1] - q[2] * r[0];
  double c0 = q[2] * qr2 - q[3] * qr1, c1 = q[3] * qr0 - q[1] * qr2, c2 = q[1] * qr1 - q[2] * qr0;
  o[0] = r[0] + 2 * (q[0] * qr0 + c0);
  o[1] = r[1] + 2 * (q[0] * qr1 + c1);
  o[2] = r[2] + 2 * (q[0] * qr2 + c2);
}

// ---------------------------------------------------------------- Bessel
// k-hat_n by upward recurrence; K[0..len) initialised to 1 (src/expansion.cpp:421-436)
__device__ __forceinline__ void bessel_k(const Tab &T, double *K, int len, double val)
{
  for (int n = 0; n < len; n++) K[n] = 1.0;
  if (val != 0.0 && len > 1) {
    K[1] += val;
    const double vs = val * val;
    for (int n = 2; n < len; n++) K[n] = K[n - 1] + vs * K[n - 2] * T.C4[n];
  }
}
// i-hat_n by its power series (src/expansion.cpp:347-365)
__device__ __forceinline__ void bessel_i(double *K, int len, double val)
{
  for (int n = 0; n < len; n++) K[n] = 1.0;
  if (val != 0.0) {
    const double z = 0.5 * val * val;
    for (int n = 0; n < len; n++) {
      double t = z / (2 * n + 3);
      for (int j = 1; j <= 20; j++) {
        K[n] += t;
        t *= (z / ((j + 1) * (2 * (n + j) + 3)));
        if (t < 1e-20) break;
      }
    }
  }
}

// ---------------------------------------------------------------- spherical harmonics
// Column m (degrees m..P-1) of the normalised real spherical harmonics at
// (cos t, sin t, phi): associated Legendre recurrence of src/expansion.cpp:634-675
// and the normalisation of src/expansion.cpp:482-518.  Calls f(n, re, im) in
// increasing n (im = 0 for m = 0).
template <class Fn>
__device__ __forceinline__ void sh_column(const Tab &T, double cost, double sint, double phi, int m, int P, Fn f)
{
  if (m >= P) return;
  double cp = 1.0, sp = 0.0;
  if (m > 0) {
    double ang = 0.0;
    for (int k = 0; k < m; k++) ang += phi;
    sincos(ang, &sp, &cp);
  }
  double pm2 = 0.0, pm1 = 0.0;
  if (m == 0) {
    double p0 = T.C6[0];
    f(0, p0 * T.c3(0, 0), 0.0);
    if (P > 1) {
      double p1 = cost * p0;
      f(1, p1 * T.c3(1, 0), 0.0);
      pm2 = p0; pm1 = p1;
      for (int n = 2; n < P; n++) {
        double pn = cost * T.c1(n, 0) * pm1 - T.c2(n, 0) * pm2;
        f(n, pn * T.c3(n, 0), 0.0);
        pm2 = pm1; pm1 = pn;
      }
    }
    return;
  }
  double sq = 1.0;
  for (int k = 0; k < m; k++) sq *= sint;
  const double neg = (m & 1) ? -1.0 : 1.0;
  const double s = (m & 1) ? -1.0 : 1.0;
  double pmm = neg * T.C6[m] * sq;
  {
    double sc = s * T.c3(m, m);
    f(m, pmm * (sc * cp), pmm * (sc * sp));
  }
  if (m + 1 < P) {
    double p1 = cost * (2 * m + 1) * pmm;
    double sc = s * T.c3(m + 1, m);
    f(m + 1, p1 * (sc * cp), p1 * (sc * sp));
    pm2 = pmm; pm1 = p1;
    for (int n = m + 2; n < P; n++) {
      double pn = cost * T.c1(n, m) * pm1 - T.c2(n, m) * pm2;
      double sc2 = s * T.c3(n, m);
      f(n, pn * (sc2 * cp), pn * (sc2 * sp));
      pm2 = pm1; pm1 = pn;
    }
  }
}

// sh_column with the column's (cos m phi, sin m phi) = (cp, sp) and sint^m = sq given
// by the caller (the same recurrence and normalisation)
template <class Fn>
__device__ __forceinline__ void sh_column_cs(const Tab &T, double cost, double cp, double sp, double sq, int m, int P,
                                             Fn f)
{
  if (m >= P) return;
  if (m == 0) {
    double p0 = T.C6[0];
    f(0, p0 * T.c3(0, 0), 0.0);
    if (P > 1) {
      double p1 = cost * p0;
      f(1, p1 * T.c3(1, 0), 0.0);
      double pm2 = p0, pm1 = p1;
      for (int n = 2; n < P; n++) {
        double pn = cost * T.c1(n, 0) * pm1 - T.c2(n, 0) * pm2;
        f(n, pn * T.c3(n, 0), 0.0);
        pm2 = pm1; pm1 = pn;
      }
    }
    return;
  }
  const double neg = (m & 1) ? -1.0 : 1.0;
  const double s = (m & 1) ? -1.0 : 1.0;
  double pmm = neg * T.C6[m] * sq;
  {
    double sc = s * T.c3(m, m);
    f(m, pmm * (sc * cp), pmm * (sc * sp));
  }
  if (m + 1 < P) {
    double p1 = cost * (2 * m + 1) * pmm;
    double sc = s * T.c3(m + 1, m);
    f(m + 1, p1 * (sc * cp), p1 * (sc * sp));
    double pm2 = pmm, pm1 = p1;
    for (int n = m + 2; n < P; n++) {
      double pn = cost * T.c1(n, m) * pm1 - T.c2(n, m) * pm2;
      double sc2 = s * T.c3(n, m);
      f(n, pn * (sc2 * cp), pn * (sc2 * sp));
      pm2 = pm1; pm1 = pn;
    }
  }
}

// team: full SH expansion of P degrees at (theta, phi) into out[P*P]
template <class TM>
__device__ void sh_full(const TM &tm, const Tab &T, double theta, double phi, int P, double *out)
{
  const double cost = cos(theta), sint = sin(theta);
  for (int m = tm.rank; m < P; m += tm.size) {
    sh_column(T, cost, sint, phi, m, P, [&](int n, double re, double im) {
      if (m == 0) out[IDX(n)] = re;
      else { out[IDX(n) + 2 * m - 1] = re; out[IDX(n) + 2 * m] = im; }
    });
  }
}

__device__ __forceinline__ double2 comp(const double *M, int n, int m)   // src/expansion.h:521-536
{
  if (m == 0) return make_double2(M[IDX(n)], 0.0);
  int am = m < 0 ? -m : m;
  int i = IDX(n) + 2 * am - 1;
  return (m > 0) ? make_double2(M[i], M[i + 1]) : make_double2(M[i], -M[i + 1]);
}

// ---------------------------------------------------------------- rotation coefficients
// R(n,s,m), n < 2p-1, |s| <= n, 0 <= m <= n, stored [n][n+s][m] (src/rotcoeff.h:241-242)
__host__ __device__ __forceinline__ int rot_off(int n)
{
  return ((n - 1) * n * (2 * n - 1)) / 3 + (3 * (n - 1) * n) / 2 + n;
}
__device__ __forceinline__ int rot_at(int n, int s, int m) { return rot_off(n) + (n + s) * (n + 1) + m; }

struct RotState {
  int p;
  bool sing;
  double cost, sint, cott, xi;
  double2 exphi, exiphi, exxi;
  double2 *R, *dR;
};

// CRotCoeff::initParams + computeCoeff + computeGradCoeff (src/rotcoeff.cpp:154-244, 779-850).
// The recursion in m runs level by level in two shared-memory buffers lvA/lvB of
// (2p-1)^2 complex entries (level entry (n, s) at n*n + n + s); R receives the
// entries with n < min(p, nout) in the [n][n+s][m] layout (a prefix of the full
// layout), which is all the rotation apply reads.  With grad, dR (full layout,
// n < 2p-1, global) is computed alongside.  shbuf: (2p-1)^2 doubles of scratch.
template <class TM>
__device__ void rot_compute(const TM &tm, const Tab &T, double theta, double phi, double xi, int p, bool grad,
                            RotState &rs, double2 *R, double2 *dR, double *shbuf, double2 *lvA, double2 *lvB,
                            int nout = 1 << 20)
{
  rs.p = p; rs.R = R; rs.dR = dR; rs.xi = xi;
  double sint = sin(theta);
  if (sint < 1e-12) {
    rs.sing = true;
    if (theta < PB_PI / 2) { theta = 0.0; rs.cost = 1.0; }
    else { theta = PB_PI; rs.cost = -1.0; }
    phi = 0.0; rs.sint = 0.0; rs.cott = 0.0;
    rs.exphi = make_double2(1.0, 0.0);
  } else {
    rs.sing = false;
    rs.sint = sint;
    rs.cost = cos(theta);
    rs.cott = rs.cost / sint;
    double sp, cp; sincos(phi, &sp, &cp);
    rs.exphi = make_double2(cp, sp);
  }
  rs.exiphi = cconj(rs.exphi);
  { double sx, cx; sincos(xi, &sx, &cx); rs.exxi = make_double2(cx, sx); }
  if (rs.sing) return;
  const int NN = 2 * p - 1;
  const int pout = p < nout ? p : nout;
  sh_full(tm, T, theta, phi, NN, shbuf);
  tm.sync();
  // level m = 0 from the spherical harmonics
  for (int idx = tm.rank; idx < NN * NN; idx += tm.size) {
    int n = (int)sqrt((double)idx);
    while (n * n > idx) n--;
    while ((n + 1) * (n + 1) <= idx) n++;
    const int s = idx - n * n - n;
    const double2 v = comp(shbuf, n, -s);
    lvA[idx] = v;
    if (n < pout) R[rot_at(n, s, 0)] = v;
    if (grad) {
      double2 w;
      const int as = s < 0 ? -s : s;
      if (n == 0) w = make_double2(0.0, 0.0);
      else if (as == 0) w = cscale(-sqrt((double)n * (n + 1)), cmul(rs.exiphi, comp(shbuf, n, 1)));
      else if (as < n)
        w = csub(cscale(as * rs.cott, comp(shbuf, n, as)),
                 cscale(sqrt((double)(n - as) * (n + as + 1)), cmul(rs.exiphi, comp(shbuf, n, as + 1))));
      else w = cscale(n * rs.cott, comp(shbuf, n, n));
      // w = dROT(n, -|s|, 0); dROT(n, |s|, 0) = conj(w)
      dR[rot_at(n, s, 0)] = (s <= 0) ? w : cconj(w);
    }
  }
  tm.sync();
  const double r1 = -0.5 * (1 + rs.cost), r2 = 0.5 * (1 - rs.cost), r3 = -rs.sint;
  const double dr1 = 0.5 * rs.sint, dr2 = dr1, dr3 = -rs.cost;
  double2 *cur = lvA, *nxt = lvB;
  for (int m = 0; m < p - 1; m++) {
    const int n0 = m + 2, n1 = 2 * p - m - 1;          // n in [n0, n1)
    const int W = 2 * (n1 - 1) - 1;                     // widest s range
    const int cnt = (n1 - n0) * W;
    for (int idx = tm.rank; idx < cnt; idx += tm.size) {
      const int n = n0 + idx / W, s = idx % W - (W / 2);
      if (s <= -n || s >= n) continue;
      const int as = s < 0 ? -s : s;
      const double2 a = cur[n * n + n + s - 1], b = cur[n * n + n + s + 1], c = cur[n * n + n + s];
      const double2 d1 = cscale(r1 * T.ETA(n, s - 1), a);
      const double2 d2 = cscale(r2 * T.ETA(n, -s - 1), b);
      const double2 d3 = cscale(r3 * T.ZETA(n - 1, as), c);
      const double2 acc = cadd(cadd(cmul(d1, rs.exiphi), cmul(d2, rs.exphi)), d3);
      const double2 v = cdivr(cmul(rs.exxi, acc), T.ETA(n, m));
      nxt[(n - 1) * (n - 1) + (n - 1) + s] = v;
      if (n - 1 < pout) R[rot_at(n - 1, s, m + 1)] = v;
      if (grad) {
        const double2 e1 = cscale(T.ETA(n, s - 1), cadd(cscale(r1, dR[rot_at(n, s - 1, m)]), cscale(dr1, a)));
        const double2 e2 = cscale(T.ETA(n, -s - 1), cadd(cscale(r2, dR[rot_at(n, s + 1, m)]), cscale(dr2, b)));
        const double2 e3 = cscale(T.ZETA(n - 1, as), cadd(cscale(r3, dR[rot_at(n, s, m)]), cscale(dr3, c)));
        const double2 a2 = cadd(cadd(cmul(e1, rs.exiphi), cmul(e2, rs.exphi)), e3);
        dR[rot_at(n - 1, s, m + 1)] = cdivr(cmul(rs.exxi, a2), T.ETA(n, m));
      }
    }
    tm.sync();
    double2 *t = cur; cur = nxt; nxt = t;
  }
}

// Euler angles of a molecule orientation (src/rotcoeff.cpp:180-201)
__host__ __device__ __forceinline__ void quat_angles(const double *q, double &th, double &ph, double &xi)
{
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  th = acos(1.0 - 2 * x * x - 2 * y * y);
  if (fabs(th) > 1e-12) {
    ph = atan2(y * z + w * x, x * z - w * y);
    xi = atan2(y * z - w * x, x * z + w * y);
  } else { th = 0.0; ph = 0.0; xi = 2 * acos(w); }
}

// team: rotate Min -> Mout for degrees < p2 (src/rotcoeff.cpp:356-441);
// Mout is written for degrees < p2 and zeroed up to zero_to degrees.
template <class TM>
__device__ void rot_apply(const TM &tm, const RotState &rs, const double *Min, double *Mout, int p2, bool bFor,
                          int zero_to)
{
  for (int i = tm.rank + p2 * p2; i < zero_to * zero_to; i += tm.size) Mout[i] = 0.0;
  if (rs.sing) {
    for (int i = tm.rank; i < p2 * p2; i += tm.size) {
      int n = (int)sqrt((double)i);
      while (n * n > i) n--;
      while ((n + 1) * (n + 1) <= i) n++;
      int mm = i - n * n;
      double v = Min[i];
      if (rs.cost == -1.0) {
        // m = 0 sign (-1)^n, then alternating signs starting at (-1)^n for mm >= 1
        double sgn;
        if (mm == 0) sgn = (n % 2 == 0) ? 1.0 : -1.0;
        else { int s0 = (n % 2 == 0) ? 1 : -1; sgn = ((mm - 1) % 2 == 0) ? s0 : -s0; }
        Mout[i] = sgn * v;
      } else Mout[i] = v;
    }
    return;
  }
  const int cnt = p2 * (p2 + 1) / 2;
  for (int idx = tm.rank; idx < cnt; idx += tm.size) {
    int n = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
    while (n * (n + 1) / 2 > idx) n--;
    while ((n + 1) * (n + 2) / 2 <= idx) n++;
    const int k = idx - n * (n + 1) / 2;       // m (forward) or s (transposed)
    const double *Mi = Min + IDX(n);
    double2 out;
    if (bFor) {
      const int m = k;
      out = cmul(rs.R[rot_at(n, 0, m)], make_double2(Mi[0], 0.0));
      for (int s = 1; s <= n; s++) {
        double2 inc = make_double2(Mi[2 * s - 1], Mi[2 * s]);
        out = cadd(out, cadd(cmul(rs.R[rot_at(n, s, m)], inc), cmul(rs.R[rot_at(n, -s, m)], cconj(inc))));
      }
    } else {
      const int s = k;
      out = cmul(rs.R[rot_at(n, -s, 0)], make_double2(Mi[0], 0.0));
      for (int m = 1; m <= n; m++) {
        double2 inc = make_double2(Mi[2 * m - 1], Mi[2 * m]);
        out = cadd(out, cadd(cmul(cconj(rs.R[rot_at(n, s, m)]), inc), cmul(rs.R[rot_at(n, -s, m)], cconj(inc))));
      }
    }
    if (k == 0) Mout[IDX(n)] = out.x;
    else { Mout[IDX(n) + 2 * k - 1] = out.x; Mout[IDX(n) + 2 * k] = out.y; }
  }
}

// molecule-frame rotation with the xi angle (src/rotcoeff.cpp:249-350)
__device__ void rot_apply_xi(const Team &tm, const RotState &rs, const double *Min, double *Mout, int p2, bool bFor,
                             int zero_to)
{
  if (!rs.sing) { rot_apply(tm, rs, Min, Mout, p2, bFor, zero_to); return; }
  for (int i = tm.rank + p2 * p2; i < zero_to * zero_to; i += tm.size) Mout[i] = 0.0;
  const double x = bFor ? rs.xi : -rs.xi;
  const int cnt = p2 * (p2 + 1) / 2;
  for (int idx = tm.rank; idx < cnt; idx += tm.size) {
    int n = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
    while (n * (n + 1) / 2 > idx) n--;
    while ((n + 1) * (n + 2) / 2 <= idx) n++;
    const int m = idx - n * (n + 1) / 2;
    const double *Mi = Min + IDX(n);
    if (m == 0) {
      Mout[IDX(n)] = (rs.cost == -1.0 && (n % 2 != 0)) ? -Mi[0] : Mi[0];
      continue;
    }
    double2 inc = make_double2(Mi[2 * m - 1], Mi[2 * m]);
    double se, ce; sincos(m * x, &se, &ce);
    double2 o = cmul(make_double2(ce, se), inc);
    if (rs.cost == -1.0) {
      const double s = (n % 2 == 0) ? 1.0 : -1.0;
      Mout[IDX(n) + 2 * m - 1] = s * o.x;
      Mout[IDX(n) + 2 * m] = -s * o.y;
    } else {
      Mout[IDX(n) + 2 * m - 1] = o.x;
      Mout[IDX(n) + 2 * m] = o.y;
    }
  }
}

__device__ __forceinline__ double2 derv(double2 c, int s) { return make_double2(-s * c.y, s * c.x); }

// singular-case derivative helpers (src/rotcoeff.cpp:616-771), evaluated per (n, m)
__device__ __forceinline__ double2 sing_in0(const double *Mi, int m)
{ return (m == 1) ? make_double2(Mi[0], 0.0) : make_double2(Mi[2 * (m - 1) - 1], Mi[2 * (m - 1)]); }

// team: dR/dtheta (kind 0) or dR/dphi (kind 1) applied to Min (src/rotcoeff.cpp:449-606)
template <class TM>
__device__ void drot_apply(const TM &tm, const Tab &T, const RotState &rs, const double *Min, double *Mout, int p2,
                           bool bFor, int kind, int zero_to)
{
  for (int i = tm.rank + p2 * p2; i < zero_to * zero_to; i += tm.size) Mout[i] = 0.0;
  const int cnt = p2 * (p2 + 1) / 2;
  for (int idx = tm.rank; idx < cnt; idx += tm.size) {
    int n = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
    while (n * (n + 1) / 2 > idx) n--;
    while ((n + 1) * (n + 2) / 2 <= idx) n++;
    const int k = idx - n * (n + 1) / 2;
    const double *Mi = Min + IDX(n);
    double2 out = make_double2(0.0, 0.0);
    if (rs.sing) {
      if (n == 0) { Mout[0] = 0.0; continue; }
      double flip = 1.0;
      if (kind == 0) { if (!bFor) flip = -1.0; }
      else { if (!bFor && rs.cost == 1.0) flip = -1.0; }
      const bool up = (rs.cost == 1.0);
      const double s = (kind == 0) ? ((n % 2 == 1) ? -1.0 : 1.0) : ((n % 2 == 1) ? 1.0 : -1.0);
      if (k == 0) {
        double v;
        if (kind == 0) v = up ? 2.0 * T.MQ(n, 0, 1) * Mi[1] : 2.0 * s * T.MQ(n, 0, 1) * Mi[1];
        else v = up ? 2.0 * T.MQ(n, 0, 1) * Mi[2] : s * 2 * T.MQ(n, 0, 1) * Mi[2];
        Mout[IDX(n)] = flip * v;
        continue;
      }
      const int m = k;
      double2 i0 = sing_in0(Mi, m);
      double2 o;
      if (m < n) {
        double2 i1 = make_double2(Mi[2 * (m + 1) - 1], Mi[2 * (m + 1)]);
        if (kind == 0) {
          if (up) o = cadd(cscale(T.MQ(n, m, 0), i0), cscale(T.MQ(n, m, 1), i1));
          else o = cscale(s, cadd(cscale(T.MQ(n, m, 0), cconj(i0)), cscale(T.MQ(n, m, 1), cconj(i1))));
        } else {
          if (up) o = csub(cmul(make_double2(0.0, T.MQ(n, m, 0)), i0), cmul(make_double2(0.0, T.MQ(n, m, 1)), i1));
          else o = cscale(s, csub(cmul(make_double2(0.0, T.MQ(n, m, 1)), cconj(i1)), cmul(make_double2(0.0, T.MQ(n, m, 0)), cconj(i0))));
        }
      } else {
        if (kind == 0) {
          if (up) o = cscale(T.MQ(n, n, 0), i0);
          else o = cscale(s * T.MQ(n, n, 0), cconj(i0));
        } else {
          if (up) o = cmul(make_double2(0.0, T.MQ(n, n, 0)), i0);
          else o = cmul(make_double2(0.0, -s * T.MQ(n, n, 0)), cconj(i0));
        }
      }
      Mout[IDX(n) + 2 * m - 1] = flip * o.x;
      Mout[IDX(n) + 2 * m] = flip * o.y;
      continue;
    }
    if (kind == 0) {
      if (bFor) {
        const int m = k;
        out = cmul(rs.dR[rot_at(n, 0, m)], make_double2(Mi[0], 0.0));
        for (int s = 1; s <= n; s++) {
          double2 inc = make_double2(Mi[2 * s - 1], Mi[2 * s]);
          out = cadd(out, cadd(cmul(rs.dR[rot_at(n, s, m)], inc), cmul(rs.dR[rot_at(n, -s, m)], cconj(inc))));
        }
      } else {
        const int s = k;
        out = cmul(rs.dR[rot_at(n, -s, 0)], make_double2(Mi[0], 0.0));
        for (int m = 1; m <= n; m++) {
          double2 inc = make_double2(Mi[2 * m - 1], Mi[2 * m]);
          out = cadd(out, cadd(cmul(cconj(rs.dR[rot_at(n, s, m)]), inc), cmul(rs.dR[rot_at(n, -s, m)], cconj(inc))));
        }
      }
    } else {
      if (bFor) {
        const int m = k;
        for (int s = 1; s <= n; s++) {
          double2 inc = make_double2(Mi[2 * s - 1], Mi[2 * s]);
          out = csub(out, cadd(cmul(rs.R[rot_at(n, s, m)], derv(inc, s)), cmul(rs.R[rot_at(n, -s, m)], derv(cconj(inc), -s))));
        }
      } else {
        const int s = k;
        out = cmul(rs.R[rot_at(n, -s, 0)], derv(make_double2(Mi[0], 0.0), s));
        for (int m = 1; m <= n; m++) {
          double2 inc = make_double2(Mi[2 * m - 1], Mi[2 * m]);
          out = cadd(out, cadd(cmul(cconj(rs.R[rot_at(n, s, m)]), derv(inc, s)), cmul(rs.R[rot_at(n, -s, m)], derv(cconj(inc), s))));
        }
      }
    }
    if (k == 0) Mout[IDX(n)] = out.x;
    else { Mout[IDX(n) + 2 * k - 1] = out.x; Mout[IDX(n) + 2 * k] = out.y; }
  }
}

// ---------------------------------------------------------------- translation coefficients
// T(l,n,m): l < 2p-1, n <= l, m <= l, stored [l][n][m] (src/transcoeff.h:166-167)
__host__ __device__ __forceinline__ int tr_off(int l) { return (l * (l + 1) * (2 * l + 1)) / 6; }
__device__ __forceinline__ int tr_at(int l, int n, int m) { return tr_off(l) + n * (l + 1) + m; }

struct TransState {
  int p;
  double scalei, scaleo;
  const double *T, *dT;
};

// CTransCoeff::reset + computeCoeff + computeCoeff_ (src/transcoeff.cpp:150-449).
// kap is this transform's screening (0 for the F re-expansion); the recursion
// itself always uses the context's kappa, as the reference does.
template <class TM>
__device__ void trans_compute(const TM &tm, const Tab &T, double d, double kap, int p, double scalei, double scaleo,
                              bool grad, TransState &ts, double *Tc, double *dTc, double *kbuf)
{
  ts.p = p; ts.scalei = scalei; ts.scaleo = scaleo; ts.T = Tc; ts.dT = dTc;
  const int NL = 2 * p - 1;
  if (tm.rank == 0) {
    const double kd = kap * d;
    double ir = 0, exkid = 0;
    if (d > 0.0) { ir = 1.0 / d; exkid = exp(-kd) * ir; }
    bessel_k(T, kbuf, 2 * p, kd);
    Tc[tr_at(0, 0, 0)] = exkid * kbuf[0];
    exkid *= ir;
    if (grad) dTc[tr_at(0, 0, 0)] = -exkid * kbuf[1];
    exkid *= scalei;
    for (int l = 1; l < NL; l++) {
      Tc[tr_at(l, 0, 0)] = exkid * kbuf[l];
      exkid *= ir;
      if (grad) dTc[tr_at(l, 0, 0)] = exkid * (l * kbuf[l] - (2 * l + 1) * kbuf[l + 1]);
      exkid *= scalei;
    }
  }
  tm.sync();
  const double kappasqr = T.kappa * T.kappa;
  const double kpio = kappasqr * scalei * scaleo, kpoo = kappasqr * scaleo * scaleo, o_i = scaleo / scalei;
  const int nu = grad ? 2 : 1;
  // m = 0, n = 0 -> 1
  for (int idx = tm.rank; idx < (2 * p - 3) * nu; idx += tm.size) {
    int l = 1 + idx % (2 * p - 3);
    double *U = (idx / (2 * p - 3)) ? dTc : Tc;
    U[tr_at(l, 1, 0)] = -(kpio * T.BETA(l - 1, 0) * U[tr_at(l - 1, 0, 0)] + o_i * T.ALPHA(l, 0) * U[tr_at(l + 1, 0, 0)]) / T.ALPHA(0, 0);
  }
  tm.sync();
  // m = 0, n -> n+1
  for (int n = 1; n < p - 1; n++) {
    const int l0 = n + 1, l1 = 2 * p - 2 - n, w = l1 - l0;
    for (int idx = tm.rank; idx < w * nu; idx += tm.size) {
      int l = l0 + idx % w;
      double *U = (idx / w) ? dTc : Tc;
      U[tr_at(l, n + 1, 0)] = -(kpio * T.BETA(l - 1, 0) * U[tr_at(l - 1, n, 0)] + kpoo * T.BETA(n - 1, 0) * U[tr_at(l, n - 1, 0)] +
                                o_i * T.ALPHA(l, 0) * U[tr_at(l + 1, n, 0)]) / T.ALPHA(n, 0);
    }
    tm.sync();
  }
  // diagonals (l, m, m) chain in m
  for (int m = 1; m < p; m++) {
    const int l0 = m, l1 = 2 * p - 1 - m, w = l1 - l0;
    for (int idx = tm.rank; idx < w * nu; idx += tm.size) {
      int l = l0 + idx % w;
      double *U = (idx / w) ? dTc : Tc;
      U[tr_at(l, m, m)] = -(kpio * T.DELTA(l, -m) * U[tr_at(l - 1, m - 1, m - 1)] + o_i * T.GAMMA(l + 1, m - 1) * U[tr_at(l + 1, m - 1, m - 1)]) /
                          T.GAMMA(m, -m);
    }
    tm.sync();
  }
  // per-m recursion in n: step t computes n = m + t -> n + 1 for all m >= 1 at once
  for (int t = 0; t < p - 2; t++) {
    // items: m in [1, p-2-t], l in [n+1, 2p-2-n) with n = m + t
    const int W = 2 * p;
    const int cnt = (p - 1) * W * nu;
    for (int idx = tm.rank; idx < cnt; idx += tm.size) {
      int u = idx / ((p - 1) * W);
      int r = idx % ((p - 1) * W);
      int m = 1 + r / W, l = r % W;
      int n = m + t;
      if (n > p - 2) continue;
      if (l < n + 1 || l >= 2 * p - 2 - n) continue;
      double *U = u ? dTc : Tc;
      double v = kpio * T.BETA(l - 1, m) * U[tr_at(l - 1, n, m)];
      if (t > 0) v += kpoo * T.BETA(n - 1, m) * U[tr_at(l, n - 1, m)];
      v += o_i * T.ALPHA(l, m) * U[tr_at(l + 1, n, m)];
      U[tr_at(l, n + 1, m)] = -v / T.ALPHA(n, m);
    }
    tm.sync();
  }
}

// team: forward translate (src/transcoeff.cpp:210-286 and 293-364 with tpose = false);
// fact[k] = (scaleo/scalei)^k.  Out written for p degrees, zeroed up to zero_to.
template <class TM>
__device__ void trans_apply(const TM &tm, const TransState &ts, const double *fact, const double *Min, double *Mout,
                            bool deriv, int zero_to)
{
  const int p = ts.p;
  const double *C = deriv ? ts.dT : ts.T;
  for (int i = tm.rank + p * p; i < zero_to * zero_to; i += tm.size) Mout[i] = 0.0;
  for (int i = tm.rank; i < p * p; i += tm.size) {
    int n = (int)sqrt((double)i);
    while (n * n > i) n--;
    while ((n + 1) * (n + 1) <= i) n++;
    const int mm = i - n * n;
    const int m = (mm + 1) / 2;
    double acc = 0.0;
    int l;
    for (l = m; l <= n; l++) {
      double t = ((n + l) % 2 == 0) ? C[tr_at(n, l, m)] : -C[tr_at(n, l, m)];
      acc += fact[n - l] * t * Min[IDX(l) + mm];
    }
    for (; l < p; l++) acc += C[tr_at(l, n, m)] * Min[IDX(l) + mm];
    Mout[i] = acc;
  }
}

}  // namespace pbsam
