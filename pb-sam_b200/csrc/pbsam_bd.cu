// Brownian-dynamics integrator of the force path: the Ermak-McCammon step of
// the reference's two drivers, for every independent system of a batch.
//
//   NAM   (bdnam, src/BDnam.cpp:166-417): two molecules; molecule 0 stays at its
//         place and only rotates, molecule 1 translates and rotates; forces are
//         evaluated while the centre-to-centre distance is below force_dist;
//         escape beyond escape_dist; rotations are accumulated while the pair is
//         far apart and applied when it comes back inside force_dist.
//   MULTI (bdm, src/BDmulti.cpp:396-566): every molecule translates and rotates
//         in turn; forces while the minimum separation is below the interaction
//         cutoff; the time step follows that minimum separation.
//
// One step is three launches on the system's stream: pbsam_bd_pre_kernel
// (time step, whether forces are needed: the mask the force kernel reads),
// pbsam_forces_kernel (skips masked systems) and pbsam_bd_move_kernel (drift
// from the forces, Gaussian noise, rejection of moves that make spheres of two
// molecules overlap, at most max_tries draws per move as the reference's maxc).
//
// Noise: Philox4x64-10 (Salmon et al., "Parallel random numbers: as easy as
// 1, 2, 3", SC 2011), key (seed, 0), counter (draw, system, 0, 0); one block of
// four 64-bit words gives four uniforms in (0,1) and, by the Box-Muller
// transform, the three normal deviates of one random vector.  Or (noise 1) the
// reference's own stream: drand48 with the polar Box-Muller method
// (src/util.h:489-539), sequential per system, with which a trajectory repeats
// the reference's bdnam run of the same seed.
#pragma once
#include "pbsam_types.cuh"

namespace pbsam {

enum { BD_RUNNING = 0, BD_ESCAPED = 1, BD_STUCK = 2, BD_DOCKED = 3, BD_FAILED = 4 };
enum { BD_NAM = 0, BD_MULTI = 1 };
#define PBSAM_BD_THREADS 128

struct BDParams {
  int mode, max_tries;
  double force_dist, escape_dist;     // NAM: f_DIST, q_DIST (src/BDnam.h:23-24)
  double dt_min, dt_max, dt_ref, dt_div;
  double fact_tr, ikbt, coul_k;       // FACT2, IKbT, COUL_K (src/BDnam.h:10-20)
  double interact_cut;                // MULTI: interaction cutoff (force evaluation)
  unsigned long long seed;
  int noise;                          // 0: Philox4x64-10; 1: the reference's drand48 stream
};

struct BDView {
  int *status, *steps, *fevals;       // [B]
  double *time, *dt;                  // [B]
  unsigned long long *ctr;            // [B] Philox blocks drawn
  double *rot;                        // [B][nmol][4] rotations stored while far apart (NAM)
  int *need;                          // [B] force evaluation this step (read by the force kernel)
  double *cen;                        // [B][S][3] sphere centres rotated by the current orientation
  double *pos, *quat;                 // the system's poses (BatchView::pos/quat), written here
  const double *dtr, *drot;           // [nmol] translational / rotational diffusion coefficients
  unsigned long long *lcg;            // [B] drand48 state (noise 1)
  double *nr_val;                     // [B] the second deviate kept by the polar method (noise 1)
  int *nr_saved;                      // [B]
  // docking definitions of molecule 0 (NAM; CMolContact lists, src/contact.h): n_dock
  // definitions, definition d needing dock_ncon[d] of its sphere pairs dock_off[d] ..
  // dock_off[d+1]-1 (sphere dock_k1 of molecule 0, dock_k2 of molecule 1) within
  // dock_dist of each other, counted only when dock_partner[d] is 1 (the partner species)
  int n_dock;
  const int *dock_partner, *dock_ncon, *dock_off, *dock_k1, *dock_k2;
  const double *dock_dist;
};

// ---------------------------------------------------------------- Philox4x64-10
__host__ __device__ __forceinline__ unsigned long long umulhi64(unsigned long long a, unsigned long long b)
{
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (unsigned long long)(((unsigned __int128)a * b) >> 64);
#endif
}

__host__ __device__ __forceinline__ void philox4x64_10(unsigned long long c[4], unsigned long long k0,
                                                       unsigned long long k1)
{
  const unsigned long long M0 = 0xD2E7470EE14C6C93ULL, M1 = 0xCA5A826395121157ULL;
  const unsigned long long W0 = 0x9E3779B97F4A7C15ULL, W1 = 0xBB67AE8584CAA73BULL;
  for (int r = 0; r < 10; r++) {
    if (r) { k0 += W0; k1 += W1; }
    const unsigned long long hi0 = umulhi64(M0, c[0]), lo0 = M0 * c[0];
    const unsigned long long hi1 = umulhi64(M1, c[2]), lo1 = M1 * c[2];
    const unsigned long long n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
  }
}

// three standard normal deviates from Philox block (draw, sys) of key (seed, 0)
__device__ __forceinline__ void bd_normal3(unsigned long long seed, unsigned long long draw, int sys, double z[3])
{
  unsigned long long c[4] = {draw, (unsigned long long)sys, 0ULL, 0ULL};
  philox4x64_10(c, seed, 0ULL);
  double u[4];
  for (int i = 0; i < 4; i++) u[i] = ((double)(c[i] >> 11) + 0.5) * 0x1p-53;
  const double r0 = sqrt(-2.0 * log(u[0])), r1 = sqrt(-2.0 * log(u[2]));
  z[0] = r0 * cos(2.0 * PB_PI * u[1]);
  z[1] = r0 * sin(2.0 * PB_PI * u[1]);
  z[2] = r1 * cos(2.0 * PB_PI * u[3]);
}

// ---------------------------------------------------------------- quaternions (w, x, y, z)
// a (x) b as CQuat::operator*= computes b *= a (src/util.h:242-263): no normalization
__device__ __forceinline__ void qmul(const double *a, const double *b, double *o)
{
  const double w = a[0] * b[0] - (a[1] * b[1] + a[2] * b[2] + a[3] * b[3]);
  const double x = a[0] * b[1] + b[0] * a[1] + (a[2] * b[3] - a[3] * b[2]);
  const double y = a[0] * b[2] + b[0] * a[2] + (a[3] * b[1] - a[1] * b[3]);
  const double z = a[0] * b[3] + b[0] * a[3] + (a[1] * b[2] - a[2] * b[1]);
  o[0] = w; o[1] = x; o[2] = y; o[3] = z;
}

// CQuat(axis, angle) (src/util.h:220-229)
__device__ __forceinline__ void quat_axis_angle(const double *ax, double angle, double *q)
{
  const double n2 = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
  if (angle != 0.0 && n2 != 0.0) {
    const double in = 1.0 / sqrt(n2);
    const double s = sin(0.5 * angle);
    double w = cos(0.5 * angle), x = s * (ax[0] * in), y = s * (ax[1] * in), z = s * (ax[2] * in);
    const double qn = 1.0 / sqrt((x * x + y * y + z * z) + w * w);
    q[0] = w * qn; q[1] = x * qn; q[2] = y * qn; q[3] = z * qn;
  } else {
    q[0] = 1.0; q[1] = 0.0; q[2] = 0.0; q[3] = 0.0;
  }
}

__device__ __forceinline__ double bd_dt(const BDParams &p, double d)   // compute_dt (src/BDnam.cpp:409-417)
{
  double dt = (d - p.dt_ref > 0) ? p.dt_min + (d - p.dt_ref) / p.dt_div : p.dt_min;
  return dt < p.dt_max ? dt : p.dt_max;
}

__device__ __forceinline__ double c2c_dist(const double *a, const double *b, double box)   // getC2CDist
{
  double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
  min_image(box, d);
  return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

// block-wide test: does molecule i, its centre at P and its sphere centres
// relative to P given by rel (rel == null: the stored rotated centres), overlap
// a sphere of any other molecule?  form 0: isCollided (src/moldynamics.cpp:167-193),
// form 1: willRotCollide (src/moldynamics.cpp:43-85)
__device__ bool bd_collides(const Ctx &c, const BDView &v, int b, int i, const double *P, const double *rel, int form)
{
  const BatchView &bv = c.bv;
  const int nmol = bv.nmol, S = bv.S;
  const double *pos = bv.pos + (size_t)b * nmol * 3;
  const double *cen = v.cen + (size_t)b * S * 3;
  const double maxRi = c.tv.maxR[bv.mol_type[i]];
  int hit = 0;
  for (int j = 0; j < nmol; j++) {
    if (j == i) continue;
    if (c2c_dist(P, pos + 3 * j, c.prm.box) - maxRi - c.tv.maxR[bv.mol_type[j]] > 0) continue;
    const int i0 = bv.mol_off[i], ni = bv.mol_off[i + 1] - i0;
    const int j0 = bv.mol_off[j], nj = bv.mol_off[j + 1] - j0;
    for (int u = threadIdx.x; u < ni * nj && !hit; u += blockDim.x) {
      const int ki = i0 + u / nj, kj = j0 + u % nj;
      const double *ci = rel ? rel + 3 * (ki - i0) : cen + 3 * ki;
      const double *cj = cen + 3 * kj, *pj = pos + 3 * j;
      const double ri = c.tv.rad[bv.sph_ts[ki]], rj = c.tv.rad[bv.sph_ts[kj]];
      double d[3];
      for (int a = 0; a < 3; a++) d[a] = ((P[a] + ci[a]) - pj[a]) - cj[a];
      min_image(c.prm.box, d);
      const double dist = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (form == 0 ? ((dist - ri) - rj < 0.0) : ((ri + rj) - dist > 0.0)) hit = 1;
    }
  }
  return __syncthreads_or(hit) != 0;
}

__device__ void bd_rotate_centres(const Ctx &c, const BDView &v, int b, int i)
{
  const BatchView &bv = c.bv;
  const double *q = bv.quat + ((size_t)b * bv.nmol + i) * 4;
  for (int k = bv.mol_off[i] + threadIdx.x; k < bv.mol_off[i + 1]; k += blockDim.x)
    qrot(q, c.tv.cen + 3 * bv.sph_ts[k], v.cen + ((size_t)b * bv.S + k) * 3);
}

// time step and force mask of every running system
__device__ void bd_pre_body(const Ctx &c, const BDParams &p, const BDView &v, int b)
{
  const BatchView &bv = c.bv;
  const int nmol = bv.nmol;
  if (b >= bv.B) return;
  if (v.status[b] != BD_RUNNING) {
    if (threadIdx.x == 0) v.need[b] = 0;
    return;
  }
  for (int i = 0; i < nmol; i++) bd_rotate_centres(c, v, b, i);
  __syncthreads();
  const double *pos = bv.pos + (size_t)b * nmol * 3;
  if (p.mode == BD_NAM) {
    if (threadIdx.x == 0) {
      const double cc = c2c_dist(pos, pos + 3, c.prm.box);
      const double d = cc - c.tv.maxR[bv.mol_type[0]] - c.tv.maxR[bv.mol_type[1]];
      v.dt[b] = bd_dt(p, d);
      v.need[b] = cc < p.force_dist;
    }
    return;
  }
  // computeMinSepDist (src/BDmulti.cpp:527-566) as bdm runs it: CBDmulti::initConstants
  // (src/BDmulti.cpp:26-38) sets its limits before the molecules exist
  // (src/BDmulti_main.cpp:67-69), while CMolecule::m_interactRcutoff is still DBL_MAX
  // (src/molecule.cpp:26), so every molecule pair is tracked sphere by sphere and the
  // smallest gap is floored at DISTCUTOFF_TIME (dt_ref)
  const double maxd = 1e300;
  const double mind = p.dt_ref;
  const double *cen = v.cen + (size_t)b * bv.S * 3;
  double smin = 1e300, mmin = 1e300;
  int track = 0;
  for (int i = 0; i < nmol; i++)
    for (int j = i + 1; j < nmol; j++) {
      const double dm = c2c_dist(pos + 3 * i, pos + 3 * j, c.prm.box) - c.tv.maxR[bv.mol_type[i]] - c.tv.maxR[bv.mol_type[j]];
      if (dm < maxd) {
        track = 1;
        const int i0 = bv.mol_off[i], ni = bv.mol_off[i + 1] - i0;
        const int j0 = bv.mol_off[j], nj = bv.mol_off[j + 1] - j0;
        for (int u = threadIdx.x; u < ni * nj; u += blockDim.x) {
          const int ki = i0 + u / nj, kj = j0 + u % nj;
          double d[3];
          for (int a = 0; a < 3; a++) d[a] = ((pos[3 * i + a] + cen[3 * ki + a]) - pos[3 * j + a]) - cen[3 * kj + a];
          min_image(c.prm.box, d);
          const double g = (sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) - c.tv.rad[bv.sph_ts[ki]]) -
                           c.tv.rad[bv.sph_ts[kj]];
          smin = g < smin ? g : smin;
        }
      } else if (dm < mmin) {
        mmin = dm;
      }
    }
  __shared__ double red[PBSAM_BD_THREADS];
  red[threadIdx.x] = smin;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h && red[threadIdx.x + h] < red[threadIdx.x]) red[threadIdx.x] = red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double md;
    if (track) md = red[0] < mind ? mind : red[0];
    else md = mmin > 0 ? mmin : 0;
    v.dt[b] = bd_dt(p, md);
    v.need[b] = md < p.interact_cut;
  }
}
__global__ void __launch_bounds__(PBSAM_BD_THREADS) pbsam_bd_pre_kernel(Ctx c, BDParams p, BDView v)
{
  bd_pre_body(c, p, v, blockIdx.x);
}

// The reference's own stream (noise 1), per system: drand48 (POSIX: X <- (0x5DEECE66D X
// + 0xB) mod 2^48, value X / 2^48) seeded as srand48(seed + system), and the polar
// Box-Muller method of normRand (src/util.h:515-539), which keeps its second deviate
// for the next call.  The rejection loop is capped at 4096 draws (it ends after the
// first with probability pi/4 each time).
__device__ __forceinline__ double bd_drand48(unsigned long long &x)
{
  x = (0x5DEECE66DULL * x + 0xBULL) & ((1ULL << 48) - 1);
  return (double)x / 281474976710656.0;
}
__device__ double bd_norm_rand(const BDView &v, int b)
{
  if (v.nr_saved[b]) {
    v.nr_saved[b] = 0;
    return v.nr_val[b];
  }
  unsigned long long x = v.lcg[b];
  double v1 = 0.0, v2 = 0.0, rsq = 0.0;
  for (int k = 0; k < 4096; k++) {
    v1 = 2.0 * bd_drand48(x) - 1.0;
    v2 = 2.0 * bd_drand48(x) - 1.0;
    rsq = v1 * v1 + v2 * v2;
    if (!(rsq >= 1.0 || rsq == 0.0)) break;
  }
  v.lcg[b] = x;
  const double fac = sqrt(-2.0 * log(rsq) / rsq);
  v.nr_val[b] = v1 * fac;
  v.nr_saved[b] = 1;
  return fac * v2;
}

// one random vector of standard deviation sd added to base (thread 0 only); with
// the reference's stream the deviates are drawn z first, as gcc evaluates the
// arguments of CPnt(normRand(), normRand(), normRand()) in CBDnam::getRandVec
__device__ __forceinline__ void bd_kick(const BDParams &p, const BDView &v, int b, const double *base, double sd,
                                        double *o)
{
  double z[3];
  if (p.noise == 1) {
    z[2] = bd_norm_rand(v, b);
    z[1] = bd_norm_rand(v, b);
    z[0] = bd_norm_rand(v, b);
  } else {
    bd_normal3(p.seed, v.ctr[b]++, b, z);
  }
  for (int a = 0; a < 3; a++) o[a] = base[a] + sd * z[a];
}

// translation with rejection (src/BDnam.cpp:263-286, src/BDmulti.cpp:455-479);
// returns the number of draws
__device__ int bd_translate(const Ctx &c, const BDParams &p, const BDView &v, int b, int i, const double *drift,
                            double sd, double *sm)
{
  double *pos = v.pos + ((size_t)b * c.bv.nmol + i) * 3;
  int tries = 0;
  bool done = false;
  while (!done && tries < p.max_tries) {
    tries++;
    if (threadIdx.x == 0) {
      double d[3];
      bd_kick(p, v, b, drift, sd, d);
      for (int a = 0; a < 3; a++) sm[a] = pos[a] + d[a];
      min_image(c.prm.box, sm);   // CMolecule::translate wraps into the box
    }
    __syncthreads();
    done = !bd_collides(c, v, b, i, sm, nullptr, 0);
    if (done && threadIdx.x == 0)
      for (int a = 0; a < 3; a++) pos[a] = sm[a];
    __syncthreads();
  }
  return tries;
}

// rotation with rejection (src/BDnam.cpp:318-361, src/BDmulti.cpp:481-501): the
// last drawn quaternion is left in sm[0..3]; returns the number of draws
__device__ int bd_rotate(const Ctx &c, const BDParams &p, const BDView &v, int b, int i, const double *drift,
                         double sd, double *sm, double *rel)
{
  const BatchView &bv = c.bv;
  double *q = v.quat + ((size_t)b * bv.nmol + i) * 4;
  const double *P = bv.pos + ((size_t)b * bv.nmol + i) * 3;
  const int i0 = bv.mol_off[i], ni = bv.mol_off[i + 1] - i0;
  int tries = 0;
  bool done = false;
  while (!done && tries < p.max_tries) {
    tries++;
    if (threadIdx.x == 0) {
      double dO[3];
      bd_kick(p, v, b, drift, sd, dO);
      quat_axis_angle(dO, sqrt(dO[0] * dO[0] + dO[1] * dO[1] + dO[2] * dO[2]), sm);
      qmul(sm, q, sm + 4);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < ni; k += blockDim.x) qrot(sm + 4, c.tv.cen + 3 * bv.sph_ts[i0 + k], rel + 3 * k);
    __syncthreads();
    done = !bd_collides(c, v, b, i, P, rel, 1);
    if (done && threadIdx.x == 0)
      for (int a = 0; a < 4; a++) q[a] = sm[4 + a];
    __syncthreads();
  }
  if (done) bd_rotate_centres(c, v, b, i);
  __syncthreads();
  return tries;
}

__device__ void bd_move_body(const Ctx &c, const BDParams &p, const BDView &v, int b)
{
  extern __shared__ double bd_rel[];          // [max spheres of a molecule][3]
  __shared__ double sm[8];
  __shared__ int s_status;
  const BatchView &bv = c.bv;
  const int nmol = bv.nmol;
  if (b >= bv.B || v.status[b] != BD_RUNNING) return;
  const double dt = v.dt[b];
  const bool need = v.need[b] != 0;
  if (need && bv.status[b] != PBSAM_STATUS_OK && bv.status[b] != PBSAM_STATUS_NOT_CONVERGED) {   // the reference exits here (src/BDnam.cpp:210-212)
    if (threadIdx.x == 0) { v.status[b] = BD_FAILED; v.fevals[b]++; }
    return;
  }
  const double *F = bv.force + (size_t)b * nmol * 3, *T = bv.torque + (size_t)b * nmol * 3;
  double *pos = v.pos + (size_t)b * nmol * 3;
  if (threadIdx.x == 0) s_status = BD_RUNNING;
  __syncthreads();
  if (p.mode == BD_NAM) {
    // drifts (src/BDnam.cpp:214-218); zero beyond force_dist
    double dR[3] = {0, 0, 0}, dO1[3] = {0, 0, 0}, dO2[3] = {0, 0, 0};
    if (need) {
      const double ft = (v.dtr[1] * dt) * p.fact_tr;
      const double f1 = ((v.drot[0] * dt) * p.ikbt) * p.coul_k, f2 = ((v.drot[1] * dt) * p.ikbt) * p.coul_k;
      for (int a = 0; a < 3; a++) { dR[a] = ft * F[3 + a]; dO1[a] = f1 * T[a]; dO2[a] = f2 * T[3 + a]; }
    }
    const double bdist = c2c_dist(pos, pos + 3, c.prm.box);
    const int ct = bd_translate(c, p, v, b, 1, dR, sqrt(2 * dt * v.dtr[1]), sm);
    if (threadIdx.x == 0) {
      if (ct == p.max_tries) s_status = BD_STUCK;
      else if (c2c_dist(pos, pos + 3, c.prm.box) > p.escape_dist) s_status = BD_ESCAPED;
    }
    __syncthreads();
    if (s_status == BD_RUNNING) {
      double *rot = v.rot + (size_t)b * nmol * 4;
      double *q = v.quat + (size_t)b * nmol * 4;
      const double s1 = sqrt(2 * dt * v.drot[0]), s2 = sqrt(2 * dt * v.drot[1]);
      const double adist = c2c_dist(pos, pos + 3, c.prm.box);
      if (threadIdx.x == 0) {
        double o1[3], o2[3], Q1[4], Q2[4];
        bd_kick(p, v, b, dO1, s1, o1);
        bd_kick(p, v, b, dO2, s2, o2);
        quat_axis_angle(o1, sqrt(o1[0] * o1[0] + o1[1] * o1[1] + o1[2] * o1[2]), Q1);
        quat_axis_angle(o2, sqrt(o2[0] * o2[0] + o2[1] * o2[1] + o2[2] * o2[2]), Q2);
        if (adist > p.force_dist) {            // far: store the rotations
          qmul(Q1, rot, rot);
          qmul(Q2, rot + 4, rot + 4);
        } else if (bdist > p.force_dist) {     // just came inside: apply the stored ones
          qmul(rot, q, q);
          qmul(rot + 4, q + 4, q + 4);
          for (int k = 0; k < 8; k++) rot[k] = (k % 4 == 0) ? 1.0 : 0.0;
        }
      }
      __syncthreads();
      if (!(adist > p.force_dist) && bdist > p.force_dist) {
        bd_rotate_centres(c, v, b, 0);
        bd_rotate_centres(c, v, b, 1);
      } else if (!(adist > p.force_dist)) {
        for (int i = 0; i < 2 && s_status == BD_RUNNING; i++) {
          const int cr = bd_rotate(c, p, v, b, i, i ? dO2 : dO1, i ? s2 : s1, sm, bd_rel);
          if (cr == p.max_tries) {
            if (threadIdx.x == 0) { qmul(sm, rot + 4 * i, rot + 4 * i); s_status = BD_STUCK; }
          }
          __syncthreads();
        }
      }
    }
    // CBDnam::IsDocked (src/BDnam.cpp:379-399) after a move that left the trajectory
    // running: a definition is met when ncontact of its pairs have a surface gap
    // (CMolecule::getSepDist, src/moldynamics.cpp:36-41) of at most their distance;
    // the reference stops counting at ncontact, which decides the same
    if (s_status == BD_RUNNING && v.n_dock > 0) {
      __shared__ int s_hits;
      const int o0 = bv.mol_off[0], o1 = bv.mol_off[1];
      const double *cen = v.cen + (size_t)b * bv.S * 3;
      for (int d = 0; d < v.n_dock && s_status == BD_RUNNING; d++) {
        if (v.dock_partner[d] != 1 || v.dock_ncon[d] < 1) continue;
        if (threadIdx.x == 0) s_hits = 0;
        __syncthreads();
        for (int e = v.dock_off[d] + threadIdx.x; e < v.dock_off[d + 1]; e += blockDim.x) {
          const int s1 = o0 + v.dock_k1[e], s2 = o1 + v.dock_k2[e];
          double dd[3];
          for (int a = 0; a < 3; a++)
            dd[a] = (pos[a] + cen[3 * s1 + a]) - (pos[3 + a] + cen[3 * s2 + a]);
          min_image(c.prm.box, dd);
          const double g = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]) - c.tv.rad[bv.sph_ts[s1]] -
                           c.tv.rad[bv.sph_ts[s2]];
          if (g <= v.dock_dist[e]) atomicAdd(&s_hits, 1);
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_hits >= v.dock_ncon[d]) s_status = BD_DOCKED;
        __syncthreads();
      }
    }
  } else {
    // every molecule in turn (src/BDmulti.cpp:425-503); a move that finds no
    // free place within max_tries draws is given up
    for (int i = 0; i < nmol; i++) {
      const int m = i;
      double dR[3] = {0, 0, 0}, dO[3] = {0, 0, 0};
      if (need) {
        const double ft = (v.dtr[m] * dt) * p.fact_tr, fr = ((v.drot[m] * dt) * p.ikbt) * p.coul_k;
        for (int a = 0; a < 3; a++) { dR[a] = ft * F[3 * i + a]; dO[a] = fr * T[3 * i + a]; }
      }
      bd_translate(c, p, v, b, i, dR, sqrt(2 * dt * v.dtr[m]), sm);
      bd_rotate(c, p, v, b, i, dO, sqrt(2 * dt * v.drot[m]), sm, bd_rel);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v.status[b] = s_status;
    v.steps[b]++;
    v.time[b] += dt;
    if (need) v.fevals[b]++;
  }
}
__global__ void __launch_bounds__(PBSAM_BD_THREADS) pbsam_bd_move_kernel(Ctx c, BDParams p, BDView v)
{
  bd_move_body(c, p, v, blockIdx.x);
}

// Groups of system handles (pbsam_group_*): one launch over every system of every
// handle, CTA k taking work[k] = (handle, system); handles keep their own views.
__global__ void __launch_bounds__(PBSAM_BD_THREADS) pbsam_bd_pre_group_kernel(const Ctx *cs, const BDParams *ps,
                                                                             const BDView *vs, const int2 *work)
{
  const int2 w = work[blockIdx.x];
  bd_pre_body(cs[w.x], ps[w.x], vs[w.x], w.y);
}
__global__ void __launch_bounds__(PBSAM_BD_THREADS) pbsam_bd_move_group_kernel(const Ctx *cs, const BDParams *ps,
                                                                              const BDView *vs, const int2 *work)
{
  const int2 w = work[blockIdx.x];
  bd_move_body(cs[w.x], ps[w.x], vs[w.x], w.y);
}

__global__ void pbsam_bd_init_kernel(Ctx c, BDParams p, BDView v)
{
  const BatchView &bv = c.bv;
  const int b = blockIdx.x;
  if (b >= bv.B) return;
  if (threadIdx.x == 0) {
    v.status[b] = BD_RUNNING; v.steps[b] = 0; v.fevals[b] = 0;
    v.time[b] = 0.0; v.dt[b] = 0.0; v.ctr[b] = 0ULL; v.need[b] = 0;
    // srand48(seed + b): high 32 bits of the state from the seed, low 16 bits 0x330E
    v.lcg[b] = (((p.seed + (unsigned long long)b) & 0xFFFFFFFFULL) << 16) | 0x330EULL;
    v.nr_saved[b] = 0;
    v.nr_val[b] = 0.0;
  }
  for (int k = threadIdx.x; k < bv.nmol * 4; k += blockDim.x) v.rot[(size_t)b * bv.nmol * 4 + k] = (k % 4 == 0) ? 1.0 : 0.0;
}

}  // namespace pbsam
