// CUDA kernels of the PB-SAM mutual-polarization drop-in (sm_100a, FP64).
//
// One team (a CTA of PBSAM_TEAM threads) owns one independent system and runs
// the whole CMolecule::computeForces sequence for it in a single launch:
// pair lists, the first round from self-polarized values, the selective
// Gauss-Seidel sweeps, the per-molecule gradient solves and the force/torque
// reduction, in exactly the order and with the stopping rules of the
// reference (src/moldynamics.cpp:553-587, src/molecule.cpp:1988-2263).  Every
// loop is bounded by the reference's own iteration caps; no thread ever waits
// on another team.
#include <cstdio>
#include <cooperative_groups.h>
#include "pbsam_types.cuh"

namespace pbsam {
namespace cg = cooperative_groups;

#define PBSAM_TEAM 512
#define PBSAM_MAX_CREW 16       // CTAs (one thread-block cluster) per system at most

// ------------------------------------------------------------------ scratch
struct Scr {
  int NP2;
  int ld;                // row stride of the IMat and of the matvec operands (NP2 rounded up to even)
  int tile_pts;          // points per numeric-expansion tile
  double *sh;            // (2NP)^2
  double2 *R, *dR;       // rotation coefficients
  double *TH, *dTH, *TF; // translation coefficients
  double *kbuf, *fact;   // 2NP+2, NP
  double *e;             // 16 * NP2
  double *g;             // 8 * 3 * NP2
  double *sol;           // 6 * 3 * NP2 (solver work)
  double *mv;            // 12 * NP2 (multi-vector pair transform stages)
  double *misc;          // 4096
  double2 *lvA, *lvB;    // shared memory: rotation recursion levels, (2NP-1)^2 each
  double *tile;          // shared memory (aliases the levels): numeric-expansion point tiles
  double *xs;            // shared memory: matvec operands, 3 * ld
  double *ims;           // shared memory after the team region: the IMat of a single-CTA solve (p <= 12)
  __device__ double *E(int i) const { return e + (size_t)i * NP2; }
  __device__ double *G(int i) const { return g + (size_t)i * 3 * NP2; }
};

__host__ __device__ inline long long scr_doubles(int NP, long long S)
{
  const long long NP2 = (long long)NP * NP;
  const int NN = 2 * NP - 1;
  const long long rotE = rot_off(NN), trE = tr_off(NN);
  long long n = 0;
  n += 4LL * NP * NP;           // sh
  n += 2 * 2 * rotE;            // R, dR (double2)
  n += 3 * trE;                 // TH, dTH, TF
  n += 2 * NP + 2 + NP + 8;     // kbuf, fact
  n += 16 * NP2;                // e
  n += 8 * 3 * NP2;             // g
  n += 6 * 3 * NP2;             // sol
  n += 12 * NP2;                // mv
  n += 4096 + S * S;            // misc + list building workspace
  // a multiple of 8 doubles: consecutive blocks stay 64-byte aligned (R and dR are
  // double2, whose accesses need 16-byte alignment)
  return (n + 7) & ~7LL;
}

// IMat rows and matvec operands are stored with an even stride so that every row
// starts on a 16-byte boundary (double2 loads); the pad column is zero.
__host__ __device__ inline int imat_ld(int NP2) { return (NP2 + 1) & ~1; }
// per-sphere stride of the row-major IMat store
__host__ __device__ inline size_t imat_stride(int NP2) { return (size_t)NP2 * imat_ld(NP2); }

// numeric-expansion tile: per point the P^2 harmonics, 2 x P radial factors,
// 5 geometry words and 2 x 3 weights
__host__ __device__ inline size_t tile_point_bytes(int NP) { return ((size_t)NP * NP + 2 * NP + 11) * sizeof(double); }
// F/H solve state kept in shared memory: F, H, new H, F base, H base, new F (3
// operands each), a degree table and the four per-degree coefficients of the operands
__host__ __device__ inline size_t solve_state_bytes(int NP)
{
  return 6 * 3 * (size_t)NP * NP * sizeof(double) + (size_t)NP * NP * sizeof(short) + 16 + 4 * (size_t)NP * sizeof(double);
}
__host__ __device__ inline size_t dyn_region_bytes(int NP)
{
  const size_t NN = 2 * NP - 1;
  size_t lv = 2 * NN * NN * sizeof(double2);
  if (solve_state_bytes(NP) > lv) lv = solve_state_bytes(NP);
  size_t tp = (160 * 1024) / tile_point_bytes(NP);
  if (tp > 32) tp = 32;
  if (tp < 1) tp = 1;
  const size_t tb = tp * tile_point_bytes(NP);
  return ((lv > tb ? lv : tb) + 15) & ~(size_t)15;
}
// dynamic shared memory of every team kernel: [rotation levels | numeric tiles][matvec operands]
__host__ __device__ inline size_t team_smem_bytes(int NP)
{
  return dyn_region_bytes(NP) + 3 * (size_t)imat_ld(NP * NP) * sizeof(double) + 64;
}
// The force kernel also reserves, at pole orders up to PBSAM_SMEM_IMAT_NP, room for one
// IMat after the team region (80 KB at p = 10, 166 KB at p = 12) and its mbarrier: a
// single-CTA solve copies its sphere's IMat there once (a TMA bulk copy) and its inner
// iterations read it from shared memory instead of re-reading it from L2.
#define PBSAM_SMEM_IMAT_NP 12
__host__ __device__ inline size_t imat_smem_bytes(int NP)
{
  return NP <= PBSAM_SMEM_IMAT_NP ? imat_stride(NP * NP) * sizeof(double) + 64 : 0;
}
__host__ __device__ inline size_t forces_smem_bytes(int NP) { return team_smem_bytes(NP) + imat_smem_bytes(NP); }

__device__ Scr make_scr(double *base, int NP, void *smem)
{
  Scr s;
  const int NP2 = NP * NP;
  const int NN = 2 * NP - 1;
  {
    const size_t lv = dyn_region_bytes(NP);
    s.lvA = (double2 *)smem;
    s.lvB = s.lvA + NN * NN;
    s.tile = (double *)smem;
    int tp = (int)(lv / tile_point_bytes(NP));
    s.tile_pts = tp > 64 ? 64 : tp;
    s.xs = (double *)((char *)smem + lv);
    s.ims = (double *)((char *)smem + team_smem_bytes(NP));
  }
  const long long rotE = rot_off(NN), trE = tr_off(NN);
  s.NP2 = NP2;
  s.ld = imat_ld(NP2);
  double *p = base;
  s.sh = p; p += 4 * NP * NP;
  s.R = (double2 *)p; p += 2 * rotE;
  s.dR = (double2 *)p; p += 2 * rotE;
  s.TH = p; p += trE;
  s.dTH = p; p += trE;
  s.TF = p; p += trE;
  s.kbuf = p; p += 2 * NP + 2;
  s.fact = p; p += NP + 8;
  s.e = p; p += 16 * NP2;
  s.g = p; p += 8 * 3 * NP2;
  s.sol = p; p += 6 * 3 * NP2;
  s.mv = p; p += 12 * NP2;
  s.misc = p;
  return s;
}

// Pairs of truncation order <= PBSAM_WARP_P in the gradient re-expansion lists are
// transformed by single warps, each with its own scratch block in global memory:
// spherical harmonics, rotation coefficients (R for n < p, dR for n < 2p-1) and
// their two recursion levels, translation coefficients and their derivative, the
// factor table, three work expansions, the transform's output and the warp's sum.
#define PBSAM_WARP_P 12
#define PBSAM_WARP_MAX_NP 16      // warp transforms only at pole orders up to this (measured: they pay at
                                  // p = 10; at p = 30 the wide CTA path stays)
#define PBSAM_WARPS 16            // warp scratch blocks per CTA (a 512-thread team)
__host__ __device__ inline long long even_up(long long n) { return (n + 1) & ~1LL; }
__host__ __device__ inline long long warp_scr_doubles(int NP)
{
  const int pw = NP < PBSAM_WARP_P ? NP : PBSAM_WARP_P, NN = 2 * pw - 1;
  const long long NP2 = (long long)NP * NP;
  long long n = even_up((long long)NN * NN);
  n += even_up(2LL * rot_off(pw)) + even_up(2LL * rot_off(NN));
  n += 2 * even_up(tr_off(NN));
  n += even_up(2 * NP + 2) + even_up(NP + 8);
  n += 3 * even_up(3 * NP2);
  n += 2 * even_up(2LL * NN * NN);
  return (n + 7) & ~7LL;
}
__device__ Scr warp_scr(double *base, int NP)
{
  const int pw = NP < PBSAM_WARP_P ? NP : PBSAM_WARP_P, NN = 2 * pw - 1;
  Scr s;
  s.NP2 = NP * NP;
  s.ld = imat_ld(s.NP2);
  s.tile_pts = 0;
  double *p = base;
  auto take = [&](long long n) { double *r = p; p += even_up(n); return r; };
  s.sh = take((long long)NN * NN);
  s.R = (double2 *)take(2LL * rot_off(pw));
  s.dR = (double2 *)take(2LL * rot_off(NN));
  s.TH = take(tr_off(NN));
  s.dTH = take(tr_off(NN));
  s.TF = nullptr;
  s.kbuf = take(2 * NP + 2);
  s.fact = take(NP + 8);
  s.e = take(3LL * s.NP2);        // E(0..2)
  s.g = take(3LL * s.NP2);        // G(0): the transform's output
  s.misc = take(3LL * s.NP2);     // the warp's running sum
  s.lvA = (double2 *)take(2LL * NN * NN);
  s.lvB = (double2 *)take(2LL * NN * NN);
  s.sol = nullptr; s.mv = nullptr; s.tile = nullptr; s.xs = nullptr; s.ims = nullptr;
  return s;
}

// scratch block of CTA `rank` of system b's crew
__device__ __forceinline__ double *scr_of(const BatchView &bv, int b, int rank)
{
  return bv.scr + ((size_t)b * bv.crew + rank) * bv.scr_stride;
}
// warp scratch block w of CTA `rank` of system b's crew
__device__ __forceinline__ double *wscr_of(const BatchView &bv, int b, int rank, int w)
{
  return bv.wscr + (((size_t)b * bv.crew + rank) * PBSAM_WARPS + w) * bv.wscr_stride;
}

// ------------------------------------------------------------------ phase timers
enum { PH_SOLVE = 0, PH_SURF, PH_NUMERIC, PH_INTRA, PH_LS, PH_DTA, PH_GRX, PH_TOTAL, PH_GSURF, PH_SETUP, PH_GBOOK,
       PH_FORCE, PH_GX_INTER, PH_GX_ANALYTIC, PH_GX_NUMERIC, PH_MATVEC, PH_N = 16 };
__device__ __forceinline__ unsigned long long gtimer()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
struct PhaseClock {
  double *acc;
  unsigned long long t0;
  __device__ void start(const Team &tm) { if (tm.rank == 0) t0 = gtimer(); }
  __device__ void stop(const Team &tm, int ph) { if (tm.rank == 0 && acc) acc[ph] += (double)(gtimer() - t0); }
};


// ------------------------------------------------------------------ team helpers
template <class TM>
__device__ __forceinline__ void tcopy(const TM &tm, double *dst, const double *src, int n)
{ for (int i = tm.rank; i < n; i += tm.size) dst[i] = src[i]; }
template <class TM>
__device__ __forceinline__ void tzero(const TM &tm, double *dst, int n)
{ for (int i = tm.rank; i < n; i += tm.size) dst[i] = 0.0; }
template <class TM>
__device__ __forceinline__ void tadd(const TM &tm, double *dst, const double *src, int n)
{ for (int i = tm.rank; i < n; i += tm.size) dst[i] += src[i]; }

// deterministic team sum: xor butterfly within each warp, then the warp sums in order
__device__ double team_sum(const Team &tm, double v, double *red)
{
  const int lane = tm.rank & 31, warp = tm.rank >> 5, nw = tm.size >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) red[warp] = v;
  tm.sync();
  double r = 0.0;
  for (int w = 0; w < nw; w++) r += red[w];
  tm.sync();
  return r;
}

// two team sums at once (each the same as team_sum's; red holds 2 x warps doubles)
__device__ void team_sum2(const Team &tm, double a, double b, double *red, double &ra, double &rb)
{
  const int lane = tm.rank & 31, warp = tm.rank >> 5, nw = tm.size >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) { red[warp] = a; red[nw + warp] = b; }
  tm.sync();
  double x = 0.0, z = 0.0;
  for (int w = 0; w < nw; w++) { x += red[w]; z += red[nw + w]; }
  tm.sync();
  ra = x;
  rb = z;
}

// per-pair truncation order (src/xforms.cpp:401-414), MAX_ERROR 1e-6
__device__ __forceinline__ int compute_order(int NP, double rho, double TQ, double scale)
{
  if (TQ < 1e-10) return 1;
  double c = rho / scale - 1;
  if (c <= 1) return NP;
  int p = int(log(TQ / (1e-6 * scale * (c - 1))) / log(c) - 1 + 0.5);
  if (p < 1) p = 1;
  if (p > NP) p = NP;
  return p;
}

// ------------------------------------------------------------------ pair transforms
// Prepared analytic re-expansion between two sphere centres
// (CXFormA / CXFormAIntra, src/xforms.cpp:11-270).
struct PairXf {
  RotState rs;
  TransState th, tf;
  int pH, pF;
  double Rm[9];
};

// Coefficients for re-expanding a source centred at c_src into a target centred
// at c_tgt, P = c_tgt - c_src.  pF > 0 also prepares the unscreened (F) translation.
template <class TM>
__device__ void prep_pair(const TM &tm, const Tab &T, const Scr &sc, const double *P, int pH, int pF,
                          double sS, double sT, bool grad, PairXf &X)
{
  const Sph S = cart2sph(P[0], P[1], P[2]);
  const int prot = pF > pH ? pF : pH;
  X.pH = pH; X.pF = pF;
  rot_compute(tm, T, S.theta, S.phi, PB_PI, prot, grad, X.rs, sc.R, sc.dR, sc.sh, sc.lvA, sc.lvB);
  trans_compute(tm, T, S.rho, T.kappa, pH, sS, sT, grad, X.th, sc.TH, sc.dTH, sc.kbuf);
  if (pF > 0) trans_compute(tm, T, S.rho, 0.0, pF, sS, sT, false, X.tf, sc.TF, nullptr, sc.kbuf);
  if (tm.rank == 0) {
    sc.fact[0] = 1.0;
    for (int n = 1; n < T.NP; n++) sc.fact[n] = sc.fact[n - 1] * (sT / sS);
  }
  // spherical-to-Cartesian gradient matrix (src/xforms.cpp:59-76)
  const double ir = 1.0 / S.rho;
  if (X.rs.sing) {
    const double c = X.rs.cost;
    double m[9] = {0.0, ir * c, 0.0, 0.0, 0.0, ir, c, 0.0, 0.0};
    for (int i = 0; i < 9; i++) X.Rm[i] = m[i];
  } else {
    const double st = X.rs.sint, ct = X.rs.cost, sp = X.rs.exphi.y, cp = X.rs.exphi.x;
    const double irst = ir / st, irct = ir * ct;
    double m[9] = {st * cp, irct * cp, -irst * sp, st * sp, irct * sp, irst * cp, ct, -ir * st, 0.0};
    for (int i = 0; i < 9; i++) X.Rm[i] = m[i];
  }
  tm.sync();
}

// Prepared intra-molecular pair from the molecule-type tables (coefficients of
// intra pair entry e computed once at set-up; the per-pair orders only truncate them).
__device__ void table_pair(const Team &tm, const Tab &T, const TypeView &tv, const Scr &sc, int e, int pH, int pF,
                           double sS, double sT, PairXf &X)
{
  const int NP = T.NP;
  const double *v = tv.pS + 16 * (size_t)e;
  X.pH = pH; X.pF = pF;
  X.rs.p = pH > pF ? pH : pF;
  X.rs.sing = v[0] != 0.0;
  X.rs.cost = v[1]; X.rs.sint = v[2]; X.rs.cott = v[3]; X.rs.xi = v[4];
  X.rs.exphi = make_double2(v[5], v[6]);
  X.rs.exiphi = cconj(X.rs.exphi);
  X.rs.exxi = make_double2(v[7], v[8]);
  X.rs.R = tv.pR + (size_t)e * rot_off(NP);
  X.rs.dR = nullptr;
  X.th.p = pH; X.th.scalei = sS; X.th.scaleo = sT; X.th.T = tv.pTH + (size_t)e * tr_off(NP); X.th.dT = nullptr;
  X.tf.p = pF; X.tf.scalei = sS; X.tf.scaleo = sT; X.tf.T = tv.pTF + (size_t)e * tr_off(NP); X.tf.dT = nullptr;
  if (tm.rank == 0) {
    sc.fact[0] = 1.0;
    for (int n = 1; n < NP; n++) sc.fact[n] = sc.fact[n - 1] * (sT / sS);
  }
  tm.sync();
}

// table entry of the intra pair (ki -> target, kj -> source) of type sphere ts = type_off + ki
__device__ __forceinline__ int intra_pair(const TypeView &tv, int ts, int ki, int kj)
{
  return tv.pair_off[ts] + (kj < ki ? kj : kj - 1);
}

// rotate -> translate -> rotate back (src/xforms.cpp:122-132, 260-270); Mout zero-padded to NP
template <class TM>
__device__ void pair_apply(const TM &tm, const Tab &T, const Scr &sc, const PairXf &X, bool useF, const double *Min,
                           double *Mout)
{
  const int p = useF ? X.pF : X.pH;
  const TransState &ts = useF ? X.tf : X.th;
  double *tM = sc.E(0), *tL = sc.E(1);
  rot_apply(tm, X.rs, Min, tM, p, true, p);
  tm.sync();
  trans_apply(tm, ts, sc.fact, tM, tL, false, p);
  tm.sync();
  rot_apply(tm, X.rs, tL, Mout, p, false, T.NP);
  tm.sync();
}

// ------------------------------------------------------------------ multi-vector pair transform
// Several expansions through the same pair transform at once (the x, y, z
// components of a gradient, and the F and H expansions of one source): the
// rotation coefficients are read once per entry for all vectors and each stage
// is one pass of the team.  Vector v uses the unscreened translation at order pF
// (useF) or the screened one at order pH; per vector the arithmetic is that of
// pair_apply.  ACC: out[v] += result, else out[v] = result zero-padded to NP.
#define PBSAM_MV 6
struct MultiVec {
  int n;
  const double *in[PBSAM_MV];
  double *out[PBSAM_MV];
  bool useF[PBSAM_MV];
};

// rotation of vector v (degrees < p[v]) for every v at once (rot_apply per vector)
template <bool ACC>
__device__ void rot_apply_multi(const Team &tm, const RotState &rs, int nv, const double *const *in, double *const *out,
                                const int *pv, int pmax, bool bFor, int zero_to)
{
  if (!ACC)
    for (int v = 0; v < nv; v++)
      for (int i = tm.rank + pv[v] * pv[v]; i < zero_to * zero_to; i += tm.size) out[v][i] = 0.0;
  if (rs.sing) {
    for (int i = tm.rank; i < pmax * pmax; i += tm.size) {
      int n = (int)sqrt((double)i);
      while (n * n > i) n--;
      while ((n + 1) * (n + 1) <= i) n++;
      const int mm = i - n * n;
      double sgn = 1.0;
      if (rs.cost == -1.0) {
        if (mm == 0) sgn = (n % 2 == 0) ? 1.0 : -1.0;
        else { int s0 = (n % 2 == 0) ? 1 : -1; sgn = ((mm - 1) % 2 == 0) ? s0 : -s0; }
      }
      for (int v = 0; v < nv; v++) {
        if (n >= pv[v]) continue;
        const double r = (rs.cost == -1.0) ? sgn * in[v][i] : in[v][i];
        if (ACC) out[v][i] += r;
        else out[v][i] = r;
      }
    }
    return;
  }
  const int cnt = pmax * (pmax + 1) / 2;
  for (int idx = tm.rank; idx < cnt; idx += tm.size) {
    int n = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
    while (n * (n + 1) / 2 > idx) n--;
    while ((n + 1) * (n + 2) / 2 <= idx) n++;
    const int k = idx - n * (n + 1) / 2;
    double2 o[PBSAM_MV];
    bool act[PBSAM_MV];
#pragma unroll
    for (int v = 0; v < PBSAM_MV; v++) act[v] = v < nv && n < pv[v];
    if (bFor) {
      const int m = k;
      const double2 r0 = rs.R[rot_at(n, 0, m)];
#pragma unroll
      for (int v = 0; v < PBSAM_MV; v++)
        if (act[v]) o[v] = cmul(r0, make_double2(in[v][IDX(n)], 0.0));
      for (int s = 1; s <= n; s++) {
        const double2 rp = rs.R[rot_at(n, s, m)], rn = rs.R[rot_at(n, -s, m)];
#pragma unroll
        for (int v = 0; v < PBSAM_MV; v++)
          if (act[v]) {
            const double2 inc = make_double2(in[v][IDX(n) + 2 * s - 1], in[v][IDX(n) + 2 * s]);
            o[v] = cadd(o[v], cadd(cmul(rp, inc), cmul(rn, cconj(inc))));
          }
      }
    } else {
      const int s = k;
      const double2 r0 = rs.R[rot_at(n, -s, 0)];
#pragma unroll
      for (int v = 0; v < PBSAM_MV; v++)
        if (act[v]) o[v] = cmul(r0, make_double2(in[v][IDX(n)], 0.0));
      for (int m = 1; m <= n; m++) {
        const double2 rp = cconj(rs.R[rot_at(n, s, m)]), rn = rs.R[rot_at(n, -s, m)];
#pragma unroll
        for (int v = 0; v < PBSAM_MV; v++)
          if (act[v]) {
            const double2 inc = make_double2(in[v][IDX(n) + 2 * m - 1], in[v][IDX(n) + 2 * m]);
            o[v] = cadd(o[v], cadd(cmul(rp, inc), cmul(rn, cconj(inc))));
          }
      }
    }
#pragma unroll
    for (int v = 0; v < PBSAM_MV; v++) {
      if (!act[v]) continue;
      if (k == 0) {
        if (ACC) out[v][IDX(n)] += o[v].x;
        else out[v][IDX(n)] = o[v].x;
      } else {
        if (ACC) { out[v][IDX(n) + 2 * k - 1] += o[v].x; out[v][IDX(n) + 2 * k] += o[v].y; }
        else { out[v][IDX(n) + 2 * k - 1] = o[v].x; out[v][IDX(n) + 2 * k] = o[v].y; }
      }
    }
  }
}

// forward translation of every vector (trans_apply per vector, deriv = false)
__device__ void trans_apply_multi(const Team &tm, const PairXf &X, const double *fact, int nv, const double *const *in,
                                  double *const *out, const bool *useF, int pmax)
{
  bool has[2] = {false, false};   // [0] some vector uses F, [1] some uses H
  for (int v = 0; v < nv; v++) has[useF[v] ? 0 : 1] = true;
  for (int i = tm.rank; i < pmax * pmax; i += tm.size) {
    int n = (int)sqrt((double)i);
    while (n * n > i) n--;
    while ((n + 1) * (n + 1) <= i) n++;
    const int mm = i - n * n;
    const int m = (mm + 1) / 2;
    for (int g = 0; g < 2; g++) {
      if (!has[g]) continue;     // (the F transform is not prepared when no vector uses it)
      const bool gF = (g == 0);
      const TransState &ts = gF ? X.tf : X.th;
      const int p = ts.p;
      if (n >= p) continue;
      double acc[PBSAM_MV];
      bool act[PBSAM_MV];
#pragma unroll
      for (int v = 0; v < PBSAM_MV; v++) { act[v] = v < nv && useF[v] == gF; acc[v] = 0.0; }
      const double *C = ts.T;
      int l;
      for (l = m; l <= n; l++) {
        const double t = ((n + l) % 2 == 0) ? C[tr_at(n, l, m)] : -C[tr_at(n, l, m)];
        const double f = fact[n - l];
#pragma unroll
        for (int v = 0; v < PBSAM_MV; v++)
          if (act[v]) acc[v] += f * t * in[v][IDX(l) + mm];
      }
      for (; l < p; l++) {
        const double c = C[tr_at(l, n, m)];
#pragma unroll
        for (int v = 0; v < PBSAM_MV; v++)
          if (act[v]) acc[v] += c * in[v][IDX(l) + mm];
      }
#pragma unroll
      for (int v = 0; v < PBSAM_MV; v++)
        if (act[v]) out[v][i] = acc[v];
    }
  }
}

__device__ __noinline__ void pair_apply_multi(const Team &tm, const Tab &T, const Scr &sc, const PairXf &X, const MultiVec &V,
                                 bool accumulate)
{
  int pv[PBSAM_MV];
  const double *tMc[PBSAM_MV];
  double *tM[PBSAM_MV], *tL[PBSAM_MV];
  int pmax = 0;
  for (int v = 0; v < PBSAM_MV; v++) {
    pv[v] = (v < V.n) ? (V.useF[v] ? X.pF : X.pH) : 0;
    if (pv[v] > pmax) pmax = pv[v];
    tM[v] = sc.mv + (size_t)v * sc.NP2;
    tMc[v] = tM[v];
    tL[v] = sc.mv + (size_t)(PBSAM_MV + v) * sc.NP2;
  }
  rot_apply_multi<false>(tm, X.rs, V.n, V.in, tM, pv, pmax, true, 0);
  tm.sync();
  trans_apply_multi(tm, X, sc.fact, V.n, tMc, tL, V.useF, pmax);
  tm.sync();
  const double *tLc[PBSAM_MV];
  for (int v = 0; v < PBSAM_MV; v++) tLc[v] = tL[v];
  if (accumulate) rot_apply_multi<true>(tm, X.rs, V.n, tLc, V.out, pv, pmax, false, T.NP);
  else rot_apply_multi<false>(tm, X.rs, V.n, tLc, V.out, pv, pmax, false, T.NP);
  tm.sync();
}

// gradient of the re-expansion w.r.t. the target position (src/xforms.cpp:85-115, 164-192);
// G holds 3 expansions (x, y, z), each zero-padded to NP.
template <class TM>
__device__ void pair_apply_grad(const TM &tm, const Tab &T, const Scr &sc, const PairXf &X, const double *Min,
                                double *G)
{
  const int p = X.pH, NP2 = T.NP * T.NP;
  double *tM = sc.E(0), *tL = sc.E(1), *tmp = sc.E(2);
  double *G0 = G, *G1 = G + NP2, *G2 = G + 2 * NP2;
  rot_apply(tm, X.rs, Min, tM, p, true, p);
  tm.sync();
  trans_apply(tm, X.th, sc.fact, tM, tL, true, p);
  tm.sync();
  rot_apply(tm, X.rs, tL, G0, p, false, T.NP);
  tm.sync();
  trans_apply(tm, X.th, sc.fact, tM, tL, false, p);
  tm.sync();
  drot_apply(tm, T, X.rs, tL, G1, p, false, 0, T.NP);
  drot_apply(tm, T, X.rs, tL, G2, p, false, 1, T.NP);
  tm.sync();
  drot_apply(tm, T, X.rs, Min, tM, p, true, 0, p);
  tm.sync();
  trans_apply(tm, X.th, sc.fact, tM, tL, false, p);
  tm.sync();
  rot_apply(tm, X.rs, tL, tmp, p, false, p);
  tm.sync();
  tadd(tm, G1, tmp, p * p);
  tm.sync();
  drot_apply(tm, T, X.rs, Min, tM, p, true, 1, p);
  tm.sync();
  trans_apply(tm, X.th, sc.fact, tM, tL, false, p);
  tm.sync();
  rot_apply(tm, X.rs, tL, tmp, p, false, p);
  tm.sync();
  tadd(tm, G2, tmp, p * p);
  tm.sync();
  for (int i = tm.rank; i < p * p; i += tm.size) {
    const double a0 = G0[i], a1 = G1[i], a2 = G2[i];
    G0[i] = X.Rm[0] * a0 + X.Rm[1] * a1 + X.Rm[2] * a2;
    G1[i] = X.Rm[3] * a0 + X.Rm[4] * a1 + X.Rm[5] * a2;
    G2[i] = X.Rm[6] * a0 + X.Rm[7] * a1 + X.Rm[8] * a2;
  }
  tm.sync();
}

// ------------------------------------------------------------------ numeric expansions
// Expansion about the target centre of point charges located at pts[h] - shift
// (CLocalExpan / CMulExpan / CGradExpan over charge sets, src/expansion.cpp:203-264,
// src/triexpan.cpp:127-153).  NC = 1: weights w[h] (points with w == 0 skipped),
// NC = 3: weights w[3h..3h+2] (points with |w|^2 < 1e-15 skipped, unit charge).
// local: true = local expansion (k-hat radial part, e^{-kappa rho}/rho (a/rho)^n),
// false = multipole ((rho/a)^n, unscreened).  out: NC expansions of NP2, P degrees
// written, zero-padded to NP.
//
// Two weight sets over the same points (the F and H charges of one sphere) are
// expanded together so the spherical harmonics are evaluated once per point.
// The points stream through shared memory in tiles: one thread per (point, set)
// builds the radial factors, one thread per (point, column pair) writes the point's
// harmonics, then every thread adds the tile's points, in point order, into the
// coefficients it owns (registers; coefficient c = rank + j * size).
struct NumSet {
  const double *w;    // weights (nullptr: set unused)
  bool local, kappa;
  int P;              // degrees
  double *out;
};
#define PBSAM_NUM_CPT 2   // coefficients per thread: NP2 <= PBSAM_NUM_CPT * team size

__device__ __forceinline__ void radial_factors(const Tab &T, double rho, double ch, bool local, bool kappa, int P,
                                               double scale, double *rad)
{
  if (local) {
    const double val = kappa ? rho * T.kappa : 0.0;
    // k-hat_n (src/expansion.cpp:421-436) times e^{-val}/rho (scale/rho)^n
    double km2 = 1.0, km1 = 1.0 + val;
    const double vs = val * val;
    double r = 1.0 / rho;
    double k = ch * (r * (kappa ? exp(-val) : 1.0));
    r *= scale;
    for (int n = 0; n < P; n++) {
      double kn;
      if (n == 0) kn = 1.0;
      else if (n == 1) kn = (val != 0.0) ? km1 : 1.0;
      else {
        kn = (val != 0.0) ? km1 + vs * km2 * T.C4[n] : 1.0;
        km2 = km1; km1 = kn;
      }
      rad[n] = kn * k;
      k *= r;
    }
  } else {
    double k = ch;
    const double r = rho * (1.0 / scale);
    for (int n = 0; n < P; n++) { rad[n] = 1.0 * k; k *= r; }
  }
}

template <int NC>
__device__ __noinline__ void numeric_expand2(const Team &tm, const Tab &T, const Scr &sc, const double *pts, int N,
                                const double *shift, double scale, NumSet A, NumSet B, int part_rank = 0,
                                int part_size = 1, double *part = nullptr)
{
  // part != nullptr: this CTA takes tiles part_rank, part_rank + part_size, ... and
  // writes its partial sums to part[(set * NC + k) * NP2 + c] instead of the outputs
  const int NP = T.NP, NP2 = NP * NP;
  const bool useB = B.w != nullptr;
  const int P = (useB && B.P > A.P) ? B.P : A.P, P2 = P * P;
  const int PA2 = A.P * A.P, PB2 = useB ? B.P * B.P : 0;
  const int TP = sc.tile_pts;
  double *Yt = sc.tile;                        // [TP][P2] harmonics
  double *ra = Yt + (size_t)TP * P2;           // [TP][P]  radial factors, set A
  double *rb = ra + (size_t)TP * P;            // [TP][P]  radial factors, set B
  double *pg = rb + (size_t)TP * P;            // [TP][5]  cos t, sin t, phi, set A valid, set B valid
  double *pw = pg + 5 * TP;                    // [TP][6]  weights A, B
  // With few harmonics (at least two team-sized copies of them fit the team) the
  // team splits into G groups, group g adding the tile points g, g + G, ... into its
  // own partial sums, which are added in group order at the end; otherwise every
  // thread owns coefficients rank + j * size over all points.
  const int nsets = useB ? 2 : 1;
  int G = 1;
  if (2 * P2 <= tm.size) {
    G = tm.size / P2;
    while (G > 1 && (size_t)(G + 1) * 2 * NC * NP2 * sizeof(double) > dyn_region_bytes(NP)) G--;
  }
  const int grp = (G > 1) ? tm.rank / P2 : 0;
  double accA[PBSAM_NUM_CPT][NC], accB[PBSAM_NUM_CPT][NC];
  int deg[PBSAM_NUM_CPT];
#pragma unroll
  for (int j = 0; j < PBSAM_NUM_CPT; j++) {
    const int c = (G > 1) ? ((j == 0 && grp < G) ? tm.rank % P2 : P2) : tm.rank + j * tm.size;
    int n = (int)sqrt((double)c);
    while (n * n > c) n--;
    while ((n + 1) * (n + 1) <= c) n++;
    deg[j] = n;
#pragma unroll
    for (int k = 0; k < NC; k++) { accA[j][k] = 0.0; accB[j][k] = 0.0; }
  }
  const int npair = (P + 1) / 2;
  for (int h0 = part_rank * TP; h0 < N; h0 += part_size * TP) {
    const int nt = (N - h0 < TP) ? N - h0 : TP;
    // per (point, set): weights, validity, radial factors; set A also the angles
    for (int u = tm.rank; u < 2 * nt; u += tm.size) {
      const int t = u >> 1, set = u & 1;
      const NumSet &S = set ? B : A;
      const int h = h0 + t;
      bool ok = false;
      double wv[NC];
      if (!set || useB) {
        if (NC == 1) {
          wv[0] = S.w[h];
          ok = wv[0] != 0.0;
        } else {
          wv[0] = S.w[3 * h]; wv[1] = S.w[3 * h + 1]; wv[2] = S.w[3 * h + 2];
          ok = !(wv[0] * wv[0] + wv[1] * wv[1] + wv[2] * wv[2] < 1e-15);
        }
        for (int k = 0; k < NC; k++) pw[6 * t + 3 * set + k] = wv[k];
      }
      pg[5 * t + 3 + set] = ok ? 1.0 : 0.0;
      const double dx = pts[3 * h] - shift[0], dy = pts[3 * h + 1] - shift[1], dz = pts[3 * h + 2] - shift[2];
      const Sph s = cart2sph(dx, dy, dz);
      if (set == 0) {
        double st, ct;
        sincos(s.theta, &st, &ct);
        pg[5 * t] = ct; pg[5 * t + 1] = st; pg[5 * t + 2] = s.phi;
      }
      if (ok) radial_factors(T, s.rho, (NC == 1) ? wv[0] : 1.0, S.local, S.kappa, S.P, scale,
                             (set ? rb : ra) + (size_t)t * P);
    }
    tm.sync();
    for (int u = tm.rank; u < nt * npair; u += tm.size) {
      const int t = u / npair, cp = u % npair;
      if (pg[5 * t + 3] == 0.0 && pg[5 * t + 4] == 0.0) continue;
      double *yt = Yt + (size_t)t * P2;
      const double ct = pg[5 * t], st = pg[5 * t + 1], ph = pg[5 * t + 2];
      const int m1 = cp, m2 = P - 1 - cp;
      auto put = [&](int m) {
        return [&, m](int n, double re, double im) {
          if (m == 0) yt[IDX(n)] = re;
          else { yt[IDX(n) + 2 * m - 1] = re; yt[IDX(n) + 2 * m] = im; }
        };
      };
      sh_column(T, ct, st, ph, m1, P, put(m1));
      if (m2 != m1) sh_column(T, ct, st, ph, m2, P, put(m2));
    }
    tm.sync();
    for (int t = grp; t < nt; t += G) {
      const bool okA = pg[5 * t + 3] != 0.0, okB = pg[5 * t + 4] != 0.0;
      if (!okA && !okB) continue;
      const double *yt = Yt + (size_t)t * P2;
#pragma unroll
      for (int j = 0; j < PBSAM_NUM_CPT; j++) {
        const int c = (G > 1) ? ((j == 0 && grp < G) ? tm.rank % P2 : P2) : tm.rank + j * tm.size;
        if (c < P2) {
          const double yv = yt[c];
          if (okA && c < PA2) {
            const double v = yv * ra[(size_t)t * P + deg[j]];
            if (NC == 1) accA[j][0] += v;
            else {
#pragma unroll
              for (int k = 0; k < NC; k++) accA[j][k] += pw[6 * t + k] * v;
            }
          }
          if (okB && c < PB2) {
            const double v = yv * rb[(size_t)t * P + deg[j]];
            if (NC == 1) accB[j][0] += v;
            else {
#pragma unroll
              for (int k = 0; k < NC; k++) accB[j][k] += pw[6 * t + 3 + k] * v;
            }
          }
        }
      }
    }
    tm.sync();
  }
  if (G > 1) {
    // group partial sums staged after the first 2 * NC * NP2 doubles of the tile
    // region (part may be the tile region itself), then added in group order
    double *gp = sc.tile + (size_t)2 * NC * NP2;
    if (grp < G) {
      const int c = tm.rank % P2;
#pragma unroll
      for (int k = 0; k < NC; k++) {
        gp[((size_t)(grp * 2) * NC + k) * P2 + c] = accA[0][k];
        gp[((size_t)(grp * 2 + 1) * NC + k) * P2 + c] = accB[0][k];
      }
    }
    tm.sync();
    for (int u = tm.rank; u < nsets * NC * NP2; u += tm.size) {
      const int set = u / (NC * NP2), k = (u / NP2) % NC, c = u % NP2;
      double v = 0.0;
      if (c < (set ? PB2 : PA2))
        for (int g = 0; g < G; g++) v += gp[((size_t)(g * 2 + set) * NC + k) * P2 + c];
      double *o = part ? part + (size_t)(set * NC + k) * NP2 : (set ? B.out : A.out) + (size_t)k * NP2;
      o[c] = v;
    }
    tm.sync();
    return;
  }
#pragma unroll
  for (int j = 0; j < PBSAM_NUM_CPT; j++) {
    const int c = tm.rank + j * tm.size;
    if (c < NP2)
#pragma unroll
      for (int k = 0; k < NC; k++) {
        double *oa = part ? part + (size_t)k * NP2 : A.out + (size_t)k * NP2;
        double *ob = part ? part + (size_t)(NC + k) * NP2 : (useB ? B.out + (size_t)k * NP2 : nullptr);
        oa[c] = (c < PA2) ? accA[j][k] : 0.0;
        if (useB) ob[c] = (c < PB2) ? accB[j][k] : 0.0;
      }
  }
  tm.sync();
}

template <int NC>
__device__ void numeric_expand(const Team &tm, const Tab &T, const Scr &sc, const double *pts, int N,
                               const double *shift, const double *w, bool local, bool kappa, int P, double scale,
                               double *out)
{
  numeric_expand2<NC>(tm, T, sc, pts, N, shift, scale, NumSet{w, local, kappa, P, out},
                      NumSet{nullptr, false, false, 0, nullptr});
}

// ------------------------------------------------------------------ surface charges
// q[h] = dA * sum_n (2 sum_{m>0} E(n,m) Y(n,m) c_n + E(n,0) Y(n,0) c_n) at each
// exposed point (computeExposedSurfaceChargesFH, src/expcenter.cpp:1419-1440),
// with sum |q| over the points.  Two sets share the points (the F and H expansions
// of a sphere, or their gradients): set 1 from E1 with per-degree factors c1 into
// q1, set 2 (optional, E2 != nullptr) from E2/c2 into q2; NC expansions per set
// (stride NP2), q written as q[NC*h + k].  The weights (m > 0 ? 2 : 1) * c_n * E
// are staged in shared memory; this CTA takes points rank*team + t, strided by
// size*team, and its |q| sums are reduced over the team into tot1 / tot2.
template <int NC>
__device__ __noinline__ void surface_q2(const Team &tm, const Tab &T, const Scr &sc, const double *pts, int N, double dA,
                           const double *E1, const double *c1, double *q1, const double *E2, const double *c2,
                           double *q2, int rank, int size, double *tot1, double *tot2, double *red)
{
  const int NP = T.NP, NP2 = NP * NP;
  const bool two = E2 != nullptr;
  double *W = sc.tile;
  for (int u = tm.rank; u < (two ? 2 : 1) * NC * NP2; u += tm.size) {
    const int set = u / (NC * NP2), r = u - set * NC * NP2, c = r % NP2;
    int n = (int)sqrt((double)c);
    while (n * n > c) n--;
    while ((n + 1) * (n + 1) <= c) n++;
    const double *E = set ? E2 : E1;
    const double *cd = set ? c2 : c1;
    W[u] = ((c - n * n > 0) ? 2.0 : 1.0) * (cd[n] * E[r]);
  }
  tm.sync();
  double ta1[NC], ta2[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) { ta1[k] = 0.0; ta2[k] = 0.0; }
  for (int h = rank * tm.size + tm.rank; h < N; h += size * tm.size) {
    const Sph s = cart2sph(pts[3 * h], pts[3 * h + 1], pts[3 * h + 2]);
    double st, ct;
    sincos(s.theta, &st, &ct);
    double a1[NC], a2[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) { a1[k] = 0.0; a2[k] = 0.0; }
    for (int m = 0; m < NP; m++) {
      sh_column(T, ct, st, s.phi, m, NP, [&](int n, double re, double im) {
        const int i0 = IDX(n) + (m ? 2 * m - 1 : 0);
#pragma unroll
        for (int k = 0; k < NC; k++) {
          const double *w = W + (size_t)k * NP2 + i0;
          a1[k] += (m ? w[0] * re + w[1] * im : w[0] * re);
          if (two) {
            const double *w2 = W + (size_t)(NC + k) * NP2 + i0;
            a2[k] += (m ? w2[0] * re + w2[1] * im : w2[0] * re);
          }
        }
      });
    }
#pragma unroll
    for (int k = 0; k < NC; k++) {
      const double v1 = a1[k] * dA;
      q1[NC * h + k] = v1;
      ta1[k] += fabs(v1);
      if (two) {
        const double v2 = a2[k] * dA;
        q2[NC * h + k] = v2;
        ta2[k] += fabs(v2);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NC; k++) {
    tot1[k] = team_sum(tm, ta1[k], red);
    const double t2 = two ? team_sum(tm, ta2[k], red) : 0.0;
    if (tot2) tot2[k] = t2;
  }
}

// surface_q2 with one expansion per set and both sets, for the exact form: each point's
// (cos t, sin t, cos phi, sin phi) is read from the type's table (ang, four per point)
// instead of computed from its coordinates, each column's (cos m phi, sin m phi) comes
// from the previous column's by angle addition instead of a sincos per column, and
// sin^m t by one product per column.  The same harmonics to rounding (the exact form's
// results are set by its fixed point, not by the reference's order of operations).
__device__ __noinline__ void surface_q2_ang(const Team &tm, const Tab &T, const Scr &sc, const double *ang, int N,
                                            double dA, const double *E1, const double *c1, double *q1,
                                            const double *E2, const double *c2, double *q2, double *tot1,
                                            double *tot2, double *red)
{
  const int NP = T.NP, NP2 = NP * NP;
  double *W = sc.tile;
  for (int u = tm.rank; u < 2 * NP2; u += tm.size) {
    const int set = u / NP2, c = u - set * NP2;
    int n = (int)sqrt((double)c);
    while (n * n > c) n--;
    while ((n + 1) * (n + 1) <= c) n++;
    const double *E = set ? E2 : E1;
    const double *cd = set ? c2 : c1;
    W[u] = ((c - n * n > 0) ? 2.0 : 1.0) * (cd[n] * E[c]);
  }
  tm.sync();
  double ta1 = 0.0, ta2 = 0.0;
  for (int h = tm.rank; h < N; h += tm.size) {
    const double4 a = ((const double4 *)ang)[h];
    const double ct = a.x, st = a.y, cf = a.z, sf = a.w;
    double a1 = 0.0, a2 = 0.0, cp = 1.0, sp = 0.0, sq = 1.0;
    for (int m = 0; m < NP; m++) {
      if (m > 0) {
        const double c0 = cp;
        cp = c0 * cf - sp * sf;
        sp = sp * cf + c0 * sf;
        sq *= st;
      }
      sh_column_cs(T, ct, cp, sp, sq, m, NP, [&](int n, double re, double im) {
        const int i0 = IDX(n) + (m ? 2 * m - 1 : 0);
        const double *w = W + i0, *w2 = W + NP2 + i0;
        a1 += (m ? w[0] * re + w[1] * im : w[0] * re);
        a2 += (m ? w2[0] * re + w2[1] * im : w2[0] * re);
      });
    }
    const double v1 = a1 * dA, v2 = a2 * dA;
    q1[h] = v1;
    q2[h] = v2;
    ta1 += fabs(v1);
    ta2 += fabs(v2);
  }
  team_sum2(tm, ta1, ta2, red, *tot1, *tot2);
}

// ------------------------------------------------------------------ IMat product
// Y[d*NP2 + i] = scale[n(i)] * sum_k IMT[i][k] x[d*ld + k] for d < D (applyMMat,
// src/lautil.cpp:57-72, followed by revertF / revertH).  IMT is the IMat stored
// row-major with an even row stride ld (zero pad column), x holds the D operands
// in shared memory with the same stride (zero pad).  Each warp owns four rows at a
// time and its lanes stride the rows with 16-byte read-only loads, two column
// blocks per step, so 128 bytes per lane are in flight; the D operands share every
// loaded IMat element.  The row sums are reduced across the warp in a fixed order.
// push > 0: Y is in shared memory and each row result is stored into Y of every CTA
// of the cluster (ranks 0 .. push-1, distributed shared memory), lane 4 g + j storing
// row j to ranks g, g + 8, ...; the cluster barrier that follows publishes them.
// S: IMT is in shared memory (plain loads instead of read-only global loads; the same
// sums in the same order).
template <int D, int U, bool S>
__device__ __noinline__ void imat_apply_t(const Team &tm, const double *IMT, int ld, const double *x, int NP2,
                                          int r_begin, int r_end, double *Y, const double *scale, int push)
{
  const int lane = tm.rank & 31, warp = tm.rank >> 5, nw = tm.size >> 5;
  const int NV = ld >> 1;
  const double2 *x2 = (const double2 *)x;
  for (int r0 = r_begin + warp * 4; r0 < r_end; r0 += nw * 4) {
    const double2 *rp[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int r = (r0 + j < NP2) ? r0 + j : NP2 - 1;
      rp[j] = (const double2 *)(IMT + (size_t)r * ld);
    }
    double acc[4][D];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int d = 0; d < D; d++) acc[j][d] = 0.0;
    // U column blocks of 32 double2 per step: 4 * U 16-byte loads per lane in flight
    for (int k0 = lane; k0 < NV; k0 += 32 * U) {
      double2 a[U][4];
#pragma unroll
      for (int b = 0; b < U; b++)
#pragma unroll
        for (int j = 0; j < 4; j++)
          a[b][j] = (k0 + 32 * b < NV) ? (S ? rp[j][k0 + 32 * b] : __ldg(rp[j] + k0 + 32 * b)) : make_double2(0.0, 0.0);
#pragma unroll
      for (int b = 0; b < U; b++) {
        if (k0 + 32 * b >= NV) break;
#pragma unroll
        for (int d = 0; d < D; d++) {
          const double2 u = x2[d * NV + k0 + 32 * b];
#pragma unroll
          for (int j = 0; j < 4; j++) acc[j][d] += a[b][j].x * u.x + a[b][j].y * u.y;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int d = 0; d < D; d++) {
        double v = acc[j][d];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        acc[j][d] = v;
      }
    if (push > 0) {
      const int jj = lane & 3, g = lane >> 2;
      const int i = r0 + jj;
      if (i < r_end && g < push) {
        int n = (int)sqrt((double)i);
        while (n * n > i) n--;
        while ((n + 1) * (n + 1) <= i) n++;
        double v[D];
#pragma unroll
        for (int d = 0; d < D; d++) v[d] = 0.0;
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (j == jj)
#pragma unroll
            for (int d = 0; d < D; d++) v[d] = acc[j][d] * scale[n];
        cg::cluster_group cl = cg::this_cluster();
        for (int q = g; q < push; q += 8) {
          double *dst = cl.map_shared_rank(Y, q);
#pragma unroll
          for (int d = 0; d < D; d++) dst[d * NP2 + i] = v[d];
        }
      }
    } else if (lane < 4) {
      const int i = r0 + lane;
      if (i < r_end) {
        int n = (int)sqrt((double)i);
        while (n * n > i) n--;
        while ((n + 1) * (n + 1) <= i) n++;
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (j == lane)
#pragma unroll
            for (int d = 0; d < D; d++) Y[d * NP2 + i] = acc[j][d] * scale[n];
      }
    }
  }
}

__device__ __forceinline__ void imat_apply(const Team &tm, const double *IMT, int ld, const double *x, int NP2, int D,
                                           int r_begin, int r_end, double *Y, const double *scale, int push = 0,
                                           bool smem = false)
{
  if (smem) {
    if (D == 1) imat_apply_t<1, 4, true>(tm, IMT, ld, x, NP2, r_begin, r_end, Y, scale, push);
    else imat_apply_t<3, 4, true>(tm, IMT, ld, x, NP2, r_begin, r_end, Y, scale, push);
  } else {
    if (D == 1) imat_apply_t<1, 4, false>(tm, IMT, ld, x, NP2, r_begin, r_end, Y, scale, push);
    else imat_apply_t<3, 4, false>(tm, IMT, ld, x, NP2, r_begin, r_end, Y, scale, push);
  }
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// Copy one IMat (bytes, a multiple of 16, both addresses 16-byte aligned) into shared
// memory with a TMA bulk copy completed on an mbarrier that sits after it.  The wait is
// bounded: if the copy has not landed after 2^22 polls the staging is switched off for
// the rest of the launch (the flag after the mbarrier) and the caller reads the IMat
// from global memory; the copy, should it land later, writes only into this region.
__device__ bool stage_imat(const Team &tm, double *dst, const double *src, unsigned bytes)
{
  unsigned long long *bar = (unsigned long long *)((char *)dst + bytes);
  volatile int *off = (volatile int *)(bar + 1);
  if (*off) return false;
  const unsigned b = smem_u32(bar), d = smem_u32(dst);
  if (tm.rank == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(d), "l"(src), "r"(bytes), "r"(b) : "memory");
  }
  __syncthreads();
  int ok = 0;
  for (int it = 0; it < (1 << 22) && !ok; it++) {
    unsigned done;
    asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(done) : "r"(b) : "memory");
    ok = done != 0;
  }
  ok = __syncthreads_and(ok);
  if (tm.rank == 0) {
    if (ok) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(b) : "memory");
    else *off = 1;
  }
  __syncthreads();
  return ok != 0;
}

// ------------------------------------------------------------------ crews (thread-block clusters)
// A system may own a cluster of CTAs (a crew).  CTA 0 (the leader) runs the whole
// evaluation; the others (helpers) take a share of the IMat rows of every matvec.
// Protocol, all on cluster barriers (no flags, no spinning): the leader publishes
// a command in its shared memory next to the operands and arrives; every CTA
// applies its rows, writing them to the global output; a second barrier makes the
// rows visible to the leader.  The exit command is followed by one last barrier so
// no helper reads the leader's shared memory after it has gone.
struct CrewCmd {
  int op;                 // 0: exit, 1: matvec, 2: numeric expansion, 3: DTA list, 4: gradient pairs, 5: surface charges
  int D, ts;              // F/H solve of type sphere ts with D operands
  double *F, *H;
  const double *LF, *LH;
  double *xg;             // the leader's exchange buffers (new F rows, new H rows)
  int NC, N;              // numeric expansion
  const double *pts;
  double shift[3], nscale;
  NumSet A, B;
  int s, self, filter_mol, use_ipol, use_iact;   // gradient re-expansion list (DTA)
  double *acc;
  const double *E1, *c1, *E2, *c2;               // surface charges
  double *q1, *q2, dA;
  double ptot[6];         // a helper's |q| sums (read by the leader)
};
struct Crew {
  int rank, size;         // CTA rank in the cluster, CTAs per system
  CrewCmd *cmd;           // this CTA's command block (the leader writes every CTA's copy)
};

// leader: write the command into every CTA's command block, one 8-byte word per
// thread (every thread holds the same command; the cluster barrier that follows
// publishes it)
__device__ __forceinline__ void crew_post(const Team &tm, const Crew &cw, const CrewCmd &c)
{
  constexpr int NW = sizeof(CrewCmd) / sizeof(unsigned long long);
  static_assert(sizeof(CrewCmd) % sizeof(unsigned long long) == 0, "command block size");
  cg::cluster_group cl = cg::this_cluster();
  for (int t = tm.rank; t < NW * cw.size; t += tm.size) {
    const int q = t / NW, w = t % NW;
    unsigned long long *dst = (unsigned long long *)cl.map_shared_rank(cw.cmd, q);
    dst[w] = ((const unsigned long long *)&c)[w];
  }
}

__device__ __forceinline__ void crew_rows(int NP2, int rank, int size, int &r0, int &r1)
{
  const int per = ((NP2 + size - 1) / size + 3) & ~3;
  r0 = rank * per;
  r1 = r0 + per;
  if (r0 > NP2) r0 = NP2;
  if (r1 > NP2) r1 = NP2;
}

// Numeric expansion (numeric_expand2) shared by the crew: each CTA sums a share of
// the point tiles into its shared memory, the leader adds the partials in rank order.
template <int NC>
__device__ void crew_numeric_expand2(const Team &tm, const Crew &cw, const Tab &T, const Scr &sc, const double *pts,
                                     int N, const double *shift, double scale, NumSet A, NumSet B)
{
  if (cw.size == 1) { numeric_expand2<NC>(tm, T, sc, pts, N, shift, scale, A, B); return; }
  cg::cluster_group cl = cg::this_cluster();
  {
    CrewCmd c;
    c.op = 2; c.NC = NC; c.N = N; c.pts = pts; c.nscale = scale; c.A = A; c.B = B;
    c.shift[0] = shift[0]; c.shift[1] = shift[1]; c.shift[2] = shift[2];
    crew_post(tm, cw, c);
  }
  cl.sync();
  numeric_expand2<NC>(tm, T, sc, pts, N, shift, scale, A, B, 0, cw.size, sc.tile);
  cl.sync();                    // every CTA's partial sums are in its shared memory
  const double *parts[PBSAM_MAX_CREW];
  for (int q = 0; q < cw.size; q++) parts[q] = cl.map_shared_rank(sc.tile, q);
  const int NP2 = T.NP * T.NP, nsets = B.w ? 2 : 1;
  for (int u = tm.rank; u < nsets * NC * NP2; u += tm.size) {
    double v = 0.0;
    for (int q = 0; q < cw.size; q++) v += parts[q][u];
    const int set = u / (NC * NP2);
    (set ? B.out : A.out)[u - set * NC * NP2] = v;
  }
  tm.sync();
}

// Surface charges (surface_q2) shared by the crew: points split over the CTAs,
// |q| sums added in rank order.
template <int NC>
__device__ void crew_surface_q2(const Team &tm, const Crew &cw, const Tab &T, const Scr &sc, double *red,
                                const double *pts, int N, double dA, const double *E1, const double *c1, double *q1,
                                double *tot1, const double *E2, const double *c2, double *q2, double *tot2)
{
  if (cw.size == 1) {
    surface_q2<NC>(tm, T, sc, pts, N, dA, E1, c1, q1, E2, c2, q2, 0, 1, tot1, tot2, red);
    return;
  }
  cg::cluster_group cl = cg::this_cluster();
  {
    CrewCmd c;
    c.op = 5; c.NC = NC; c.pts = pts; c.N = N; c.dA = dA;
    c.E1 = E1; c.c1 = c1; c.q1 = q1; c.E2 = E2; c.c2 = c2; c.q2 = q2;
    crew_post(tm, cw, c);
  }
  cl.sync();
  double t1[NC], t2[NC];
  surface_q2<NC>(tm, T, sc, pts, N, dA, E1, c1, q1, E2, c2, q2, 0, cw.size, t1, t2, red);
  cl.sync();                    // helpers' charges written, their sums in their command blocks
#pragma unroll
  for (int k = 0; k < NC; k++) {
    double a = t1[k], b = t2[k];
    for (int q = 1; q < cw.size; q++) {
      const CrewCmd *r = cl.map_shared_rank(cw.cmd, q);
      a += r->ptot[k];
      b += r->ptot[3 + k];
    }
    tot1[k] = a;
    if (tot2) tot2[k] = b;
  }
  tm.sync();
}

// leader: release the helpers at the end of the evaluation
__device__ void crew_finish(const Team &tm, const Crew &cw)
{
  if (cw.size == 1) return;
  cg::cluster_group cl = cg::this_cluster();
  CrewCmd c;
  c.op = 0;
  crew_post(tm, cw, c);
  cl.sync();
  cl.sync();
}

// ------------------------------------------------------------------ F/H inner solve
// Fixed-point solve of one sphere's surface-charge expansions
// (CSolExpCenter::solveFH, src/expcenter.cpp:1079-1370) for D = 1 (F, H) or
// D = 3 (x, y, z gradients).  F and H (D*NP2) are updated in place; returns the
// deviation of H from its value on entry (computeDev2).
// The F/H inner solve, run by every CTA of the crew on a full copy of the state in
// its shared memory: each CTA forms the operands itself and applies its share of
// the IMat rows, writing them to the exchange buffer xg in global memory (L2); after
// one cluster barrier per matvec every CTA reads the whole new F (H) back.  The new
// F and the new H have separate exchange buffers, and every CTA takes the same
// stopping decision from identical data.  Returns computeDev2 on the leader (rank
// 0), which writes F and H back to the system state.
__device__ __noinline__ double solve_core(const Team &tm, const Crew &cw, double *tph, const Tab &T,
                                          const TypeView &tv, const SolveParams &prm, const Scr &sc, double *xg,
                                          int ts, int D, double *F, double *H, const double *LF, const double *LH,
                                          double *red, int *stats)
{
  const int NP = T.NP, NP2 = NP * NP, len = D * NP2;
  const double *cst = tv.cst + (size_t)ts * CST_N * NP;
  const double *Dfix = tv.Dfix + (size_t)ts * NP2, *Vfix = tv.Vfix + (size_t)ts * NP2;
  const double *IMT = tv.imat + (size_t)ts * imat_stride(NP2);
  const int ld = sc.ld;
  double *sF = sc.tile, *sH = sF + len, *sHn = sH + len, *sFb = sHn + len, *sHb = sFb + len, *sFn = sHb + len;
  short *deg = (short *)(sFn + len);
  // the operands' per-degree coefficients, copied once per solve
  double *cH1 = (double *)(((size_t)(deg + NP2) + 15) & ~(size_t)15), *cF1 = cH1 + NP, *cH2 = cF1 + NP, *cF2 = cH2 + NP;
  double *sOut = xg + 6 * NP2;               // H at entry (leader only; the leader's scratch)
  const bool lead = cw.rank == 0, crew = cw.size > 1;
  cg::cluster_group cl = cg::this_cluster();
  for (int k = tm.rank; k < NP2; k += tm.size) {
    int n = (int)sqrt((double)k);
    while (n * n > k) n--;
    while ((n + 1) * (n + 1) <= k) n++;
    deg[k] = (short)n;
  }
  for (int d = tm.rank; d < D; d += tm.size)
    for (int k = NP2; k < ld; k++) sc.xs[d * ld + k] = 0.0;   // pad columns (the IMat's are zero too)
  for (int n = tm.rank; n < NP; n += tm.size) {
    cH1[n] = cst[CST_H1 * NP + n];
    cF1[n] = cst[CST_F1 * NP + n];
    cH2[n] = cst[CST_H2 * NP + n];
    cF2[n] = cst[CST_F2 * NP + n];
  }
  tm.sync();
  for (int k = tm.rank; k < len; k += tm.size) {
    const int kk = k % NP2, n = deg[kk];
    if (D == 1) {
      sFb[k] = Vfix[kk] + cst[CST_LH1 * NP + n] * LH[k] + cst[CST_LF1 * NP + n] * LF[k];
      sHb[k] = Dfix[kk] + cst[CST_LH2 * NP + n] * LH[k] + cst[CST_LF2 * NP + n] * LF[k];
    } else {
      sFb[k] = cst[CST_LH1 * NP + n] * LH[k] + cst[CST_LF1 * NP + n] * LF[k];
      sHb[k] = cst[CST_LH2 * NP + n] * LH[k] + cst[CST_LF2 * NP + n] * LF[k];
    }
    const double h = H[k];
    sF[k] = F[k];
    sH[k] = h;
    if (lead) sOut[k] = h;
  }
  tm.sync();
  int r0, r1;
  crew_rows(NP2, cw.rank, cw.size, r0, r1);
  // a single-CTA solve at p <= 12 reads its IMat from shared memory when the launch
  // reserved the room (the force kernel does, forces_smem_bytes)
  bool sim = false;
  if (!crew && NP <= PBSAM_SMEM_IMAT_NP) {
    unsigned dsz;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dsz));
    if (dsz >= forces_smem_bytes(NP)) sim = stage_imat(tm, sc.ims, IMT, (unsigned)(imat_stride(NP2) * sizeof(double)));
  }
  const double *IMA = sim ? sc.ims : IMT;
  int ct = 0;
  double dev = 0.0;
  PhaseClock mv{tph, 0};
  const int lane = tm.rank & 31, warp = tm.rank >> 5, nwarp = tm.size >> 5;
  const int ncx = D * NP * (NP + 1) / 2;
  for (;;) {
    mv.start(tm);
    // the F operands of this iteration and, from the second iteration on, the last
    // iteration's computeDev over complex entries (d, n, m) of its old (sHn) and new
    // (sH) H: the per-thread sums and their reduction are those of team_sum, taken at
    // the operands' barrier; the stop test then comes before this iteration's products
    double part = 0.0;
    for (int k = tm.rank; k < len; k += tm.size) {
      const int kk = k % NP2, n = deg[kk];
      sc.xs[(k / NP2) * ld + kk] = sFb[k] + cH1[n] * sH[k] + cF1[n] * sF[k];
    }
    if (ct > 0) {
      for (int u = tm.rank; u < ncx; u += tm.size) {
        const int d = u / (NP * (NP + 1) / 2), r = u % (NP * (NP + 1) / 2);
        int n = (int)((sqrt(8.0 * r + 1.0) - 1.0) * 0.5);
        while (n * (n + 1) / 2 > r) n--;
        while ((n + 1) * (n + 2) / 2 <= r) n++;
        const int m = r - n * (n + 1) / 2;
        const int base = d * NP2 + IDX(n);
        double ar, ai = 0.0, br, bi = 0.0;
        if (m == 0) { ar = sHn[base]; br = sH[base]; }
        else { ar = sHn[base + 2 * m - 1]; ai = sHn[base + 2 * m]; br = sH[base + 2 * m - 1]; bi = sH[base + 2 * m]; }
        const double PL = 1e-30;
        double sv;
        if (fabs(ar) < PL && fabs(ai) < PL) {
          if (fabs(br) < PL && fabs(bi) < PL) continue;
          sv = 1.0;
        } else if (fabs(br) < PL && fabs(bi) < PL) sv = 1.0;
        else {
          const double dr = ar - br, di = ai - bi;
          const double top = dr * dr + di * di;
          const double bot = ar * ar + ai * ai + br * br + bi * bi;
          sv = (m != 0) ? 2 * top / bot : top / bot;
        }
        part += sv;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if (lane == 0) red[warp] = part;
    }
    tm.sync();
    if (ct > 0) {
      double r = 0.0;
      for (int w = 0; w < nwarp; w++) r += red[w];
      dev = r / (4 * NP * NP);
      // red is written again only at the next iteration's operands, two barriers on
      if (!(dev > prm.solve_tol && ct < prm.solve_max_ct)) {
        mv.stop(tm, PH_MATVEC);
        break;
      }
    }
    if (crew) {
      // every CTA pushes its rows of the new F into every CTA's sFn (distributed
      // shared memory); after the cluster barrier each holds the whole vector.  F is
      // double-buffered: a CTA still forming its operands from sF is never written to
      imat_apply(tm, IMT, ld, sc.xs, NP2, D, r0, r1, sFn, T.CONST3, cw.size);
      cl.sync();
      { double *t = sF; sF = sFn; sFn = t; }
    } else {
      imat_apply(tm, IMA, ld, sc.xs, NP2, D, 0, NP2, sF, T.CONST3, 0, sim);
      tm.sync();
    }
    for (int k = tm.rank; k < len; k += tm.size) {
      const int kk = k % NP2, n = deg[kk];
      sc.xs[(k / NP2) * ld + kk] = sHb[k] + cH2[n] * sH[k] + cF2[n] * sF[k];
    }
    tm.sync();
    if (crew) {
      // the same for the new H, into sHn (read only by computeDev below, after this
      // barrier, and written again only after the next F barrier)
      imat_apply(tm, IMT, ld, sc.xs, NP2, D, r0, r1, sHn, cst + CST_INVH * NP, cw.size);
      cl.sync();
    } else {
      imat_apply(tm, IMA, ld, sc.xs, NP2, D, 0, NP2, sHn, cst + CST_INVH * NP, 0, sim);
      tm.sync();
    }
    mv.stop(tm, PH_MATVEC);
    { double *t = sH; sH = sHn; sHn = t; }
    ct++;
  }
  if (!lead) return 0.0;
  if (tm.rank == 0 && stats) { stats[1] += ct; stats[2] += 1; }
  // results back to the system state; computeDev2 (outer deviation)
  double pd = 0.0, ps = 0.0;
  for (int u = tm.rank; u < len; u += tm.size) {
    F[u] = sF[u];
    H[u] = sH[u];
    const int i = u % NP2, n = deg[i];
    const int mm = i - n * n;
    const double a = sOut[u], b = sH[u], df = a - b;
    const double w = (mm == 0) ? 1.0 : 2.0;
    pd += w * (df * df);
    ps += w * (a * a + b * b);
  }
  const double td = team_sum(tm, pd, red), tsm = team_sum(tm, ps, red);
  return td / (4 * tsm) / double(D);
}

// Fixed-point solve of one sphere's surface-charge expansions
// (CSolExpCenter::solveFH, src/expcenter.cpp:1079-1370) for D = 1 (F, H) or
// D = 3 (x, y, z gradients), called by the leader: F and H (D*NP2) are updated in
// place; returns the deviation of H from its value on entry (computeDev2).
__device__ double solve_fh(const Team &tm, const Crew &cw, double *tph, const Tab &T, const TypeView &tv,
                           const SolveParams &prm, const Scr &sc, int ts, int D, double *F, double *H,
                           const double *LF, const double *LH, double *red, int *stats)
{
  if (cw.size == 1) return solve_core(tm, cw, tph, T, tv, prm, sc, sc.sol, ts, D, F, H, LF, LH, red, stats);
  cg::cluster_group cl = cg::this_cluster();
  {
    CrewCmd c;
    c.op = 1; c.D = D; c.ts = ts; c.F = F; c.H = H; c.LF = LF; c.LH = LH; c.xg = sc.sol;
    crew_post(tm, cw, c);
  }
  cl.sync();
  const double dv = solve_core(tm, cw, tph, T, tv, prm, sc, sc.sol, ts, D, F, H, LF, LH, red, stats);
  cl.sync();                    // the crew has left the solve
  return dv;
}

// ------------------------------------------------------------------ system state access
struct Sys {
  const Ctx *c;
  int b, NP, NP2, S;
  Crew cw;
  Scr sc;
  double *red;
  double *tph;
  __device__ int ts(int s) const { return c->bv.sph_ts[s]; }
  __device__ int mol(int s) const { return c->bv.sph_mol[s]; }
  __device__ double rad(int s) const { return c->tv.rad[ts(s)]; }
  __device__ size_t vs(int s) const { return ((size_t)b * S + s) * NP2; }
  __device__ size_t gs(int s) const { return ((size_t)b * S + s) * 3 * NP2; }
  __device__ size_t sc1(int s) const { return (size_t)b * S + s; }
  __device__ double *F(int s) const { return c->bv.F + vs(s); }
  __device__ double *H(int s) const { return c->bv.H + vs(s); }
  __device__ double *Hrot(int s) const { return c->bv.Hrot + vs(s); }
  __device__ double *HselfRot(int s) const { return c->bv.HselfRot + vs(s); }
  __device__ double *LS(int s) const { return c->bv.LS + vs(s); }
  __device__ double *LFS(int s) const { return c->bv.LFS + vs(s); }
  __device__ double *LHS(int s) const { return c->bv.LHS + vs(s); }
  __device__ double *gLHN(int s) const { return c->bv.gLHN + gs(s); }
  __device__ double *gH(int s) const { return c->bv.gH + gs(s); }
  __device__ int npts(int s) const { return c->bv.pt_off[s + 1] - c->bv.pt_off[s]; }
  __device__ double *qF(int s) const { return c->bv.qF + (size_t)b * c->bv.SP + c->bv.pt_off[s]; }
  __device__ double *qH(int s) const { return c->bv.qH + (size_t)b * c->bv.SP + c->bv.pt_off[s]; }
  __device__ double *gFp(int s) const { return c->bv.gFp + ((size_t)b * c->bv.SP + c->bv.pt_off[s]) * 3; }
  __device__ double *gHp(int s) const { return c->bv.gHp + ((size_t)b * c->bv.SP + c->bv.pt_off[s]) * 3; }
  __device__ const double *spx(int s) const { return c->tv.spx + 3 * (size_t)c->tv.spx_off[ts(s)]; }
  __device__ const double *cen(int s) const { return c->tv.cen + 3 * ts(s); }
  __device__ double *cenRot(int s) const { return c->bv.cenRot + 3 * sc1(s); }
  __device__ void cen_lab(int s, double *o) const
  {
    const int i = mol(s);
    const double *p = c->bv.pos + 3 * ((size_t)b * c->bv.nmol + i);
    const double *r = cenRot(s);
    o[0] = p[0] + r[0]; o[1] = p[1] + r[1]; o[2] = p[2] + r[2];
  }
  __device__ int *ipol(int s) const { return c->bv.ipol + ((size_t)b * S + s) * S; }
  __device__ int nipol(int s) const { return c->bv.ipol_n[sc1(s)]; }
  __device__ int *iact(int s) const { return c->bv.iact + ((size_t)b * S + s) * S; }
  __device__ int niact(int s) const { return c->bv.iact_n[sc1(s)]; }
  __device__ double *gw(double *base, int k) const { return base + ((size_t)b * S + k) * 3 * NP2; }
  __device__ int *stats() const { return c->bv.stats + (size_t)b * 8; }
  // molecule rotation state (coefficients computed once per call)
  __device__ RotState molrot(int i) const
  {
    RotState rs;
    const double *v = c->bv.molRS + ((size_t)b * c->bv.nmol + i) * 16;
    rs.p = NP;
    rs.sing = v[0] != 0.0;
    rs.cost = v[1]; rs.sint = v[2]; rs.cott = v[3]; rs.xi = v[4];
    rs.exphi = make_double2(v[5], v[6]);
    rs.exiphi = cconj(rs.exphi);
    rs.exxi = make_double2(v[7], v[8]);
    rs.R = c->bv.molR + ((size_t)b * c->bv.nmol + i) * rot_off(2 * NP - 1);
    rs.dR = nullptr;
    return rs;
  }
};

template <class TM>
__device__ void add_vec_into(const TM &tm, double *dst, const double *src, int n)
{
  for (int i = tm.rank; i < n; i += tm.size) dst[i] += src[i];
  tm.sync();
}

// LS from the inter-molecular polarization neighbours (src/molecule.cpp:1265-1358)
__device__ void reexpand_LS(const Team &tm, const Sys &y, int s, bool fromSelf)
{
  const Tab &T = y.c->T;
  PhaseClock pc{y.tph, 0};
  pc.start(tm);
  double *LSrot = y.sc.E(6), *tL = y.sc.E(7);
  tzero(tm, LSrot, y.NP2);
  tm.sync();
  const int *lst = y.ipol(s);
  const int nl = y.nipol(s);
  double ci[3];
  y.cen_lab(s, ci);
  for (int e = 0; e < nl; e++) {
    const int s2 = lst[e];
    double cj[3];
    y.cen_lab(s2, cj);
    double P[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
    min_image(y.c->prm.box, P);
    const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
    const double TQ = fromSelf ? y.c->tv.tHself[y.ts(s2)] : y.c->bv.tH[y.sc1(s2)];
    const int p = compute_order(y.NP, rho, TQ, y.rad(s2));
    PairXf X;
    prep_pair(tm, T, y.sc, P, p, 0, y.rad(s2), y.rad(s), false, X);
    pair_apply(tm, T, y.sc, X, false, fromSelf ? y.HselfRot(s2) : y.Hrot(s2), tL);
    add_vec_into(tm, LSrot, tL, y.NP2);
  }
  const RotState mr = y.molrot(y.mol(s));
  rot_apply_xi(tm, mr, LSrot, y.LS(s), y.NP, false, y.NP);
  tm.sync();
  pc.stop(tm, PH_LS);
}

// ------------------------------------------------------------------ small operator products
// Row products of NM (1 or 2) small row-major operators of the exact form (the direct
// inner solve, the near-field operators), row stride ld: for operator m the rows
// r < rows[m] give sum_{j < cols[m]} M[m][r][j] x[m][j], the rows rows[m] <= r < nout
// give 0, and emit(m, r, v) receives each result on one lane.  A warp takes R rows of
// every operator at a time and issues all their loads of a 128-column block together
// (4 R NM per lane).  Per row, a lane's sums are those of a warp per row (four
// accumulators over the full 128-column blocks, the ragged block added to the first in
// column order) and the warp adds them in a fixed butterfly, so a result does not
// depend on how the rows are dealt to the warps.
template <int NM, int R, class Emit>
__device__ __forceinline__ void rows_apply(const Team &tm, const double *const *M, const int *rows, const int *cols,
                                           int ld, const double *const *x, int nout, Emit emit)
{
  const int lane = tm.rank & 31, w = tm.rank >> 5, nw = tm.size >> 5;
  int cmax = 0;
#pragma unroll
  for (int m = 0; m < NM; m++) cmax = cols[m] > cmax ? cols[m] : cmax;
  for (int r0 = R * w; r0 < nout; r0 += R * nw) {
    double a[NM][R][4];
#pragma unroll
    for (int m = 0; m < NM; m++)
#pragma unroll
      for (int q = 0; q < R; q++)
#pragma unroll
        for (int b = 0; b < 4; b++) a[m][q][b] = 0.0;
    for (int j = lane; j < cmax; j += 128) {
      double v[NM][R][4], u[NM][4];
#pragma unroll
      for (int m = 0; m < NM; m++) {
#pragma unroll
        for (int b = 0; b < 4; b++) u[m][b] = (j + 32 * b < cols[m]) ? x[m][j + 32 * b] : 0.0;
#pragma unroll
        for (int q = 0; q < R; q++) {
          const double *row = M[m] + (size_t)(r0 + q) * ld;
          const bool ok = r0 + q < rows[m];
#pragma unroll
          for (int b = 0; b < 4; b++) v[m][q][b] = (ok && j + 32 * b < cols[m]) ? row[j + 32 * b] : 0.0;
        }
      }
#pragma unroll
      for (int m = 0; m < NM; m++) {
        if (j + 96 < cols[m]) {
#pragma unroll
          for (int q = 0; q < R; q++)
#pragma unroll
            for (int b = 0; b < 4; b++) a[m][q][b] += v[m][q][b] * u[m][b];
        } else if (j < cols[m]) {
#pragma unroll
          for (int q = 0; q < R; q++)
#pragma unroll
            for (int b = 0; b < 3; b++)
              if (j + 32 * b < cols[m]) a[m][q][0] += v[m][q][b] * u[m][b];
        }
      }
    }
#pragma unroll
    for (int m = 0; m < NM; m++)
#pragma unroll
      for (int q = 0; q < R; q++) {
        double acc = (a[m][q][0] + a[m][q][1]) + (a[m][q][2] + a[m][q][3]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        const int r = r0 + q;
        if (lane == R * m + q && r < nout) emit(m, r, r < rows[m] ? acc : 0.0);
      }
  }
}

// Column products (the transposes) of NM (1 or 2) small row-major operators: for
// operator m the columns j < cols[m] give sum_{k < rows[m]} M[m][k][j] y[m][k], passed
// to emit(m, j, v).  A column's sum has eight accumulators (row k to accumulator k mod 8
// over the full blocks of eight rows, the ragged end to the first, in row order),
// combined as ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7)).  With G = 2, 4 or 8
// groups of threads per column (as many as the columns of both operators leave room
// for), group g holds accumulators [g 8/G, (g + 1) 8/G) and adds them as its subtree of
// that sum; the subtree sums meet in shared memory (part, G x columns doubles) and are
// combined in the same tree, so the result does not depend on G.  Every lane keeps up
// to sixteen loads in flight.
template <int NM, int G, class Emit>
__device__ __forceinline__ void cols_apply_g(const Team &tm, const double *const *M, const int *rows, const int *cols,
                                             int ld, const double *const *y, double *part, Emit emit)
{
  constexpr int A = 8 / G, UB = 16 / A;
  const int C = cols[0] + (NM > 1 ? cols[NM - 1] : 0);
  if (tm.rank < G * C) {
    const int g = tm.rank / C, c = tm.rank - g * C;
    const int m = (NM > 1 && c >= cols[0]) ? 1 : 0, j = m ? c - cols[0] : c;
    const double *Mm = M[m], *ym = y[m];
    const int nb = rows[m] >> 3;
    double a[A];
#pragma unroll
    for (int u = 0; u < A; u++) a[u] = 0.0;
    for (int i = 0; i < nb; i += UB) {
      double v[UB][A], w[UB][A];
#pragma unroll
      for (int t = 0; t < UB; t++)
#pragma unroll
        for (int u = 0; u < A; u++) {
          const int k = 8 * (i + t) + g * A + u;
          const bool ok = i + t < nb;
          v[t][u] = ok ? Mm[(size_t)k * ld + j] : 0.0;
          w[t][u] = ok ? ym[k] : 0.0;
        }
#pragma unroll
      for (int t = 0; t < UB; t++)
        if (i + t < nb)
#pragma unroll
          for (int u = 0; u < A; u++) a[u] += v[t][u] * w[t][u];
    }
    if (g == 0)
      for (int k = 8 * nb; k < rows[m]; k++) a[0] += Mm[(size_t)k * ld + j] * ym[k];
    double s;
    if constexpr (A == 8) s = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    else if constexpr (A == 4) s = (a[0] + a[1]) + (a[2] + a[3]);
    else if constexpr (A == 2) s = a[0] + a[1];
    else s = a[0];
    if (G == 1) emit(m, j, s);
    else part[g * C + c] = s;
  }
  if (G > 1) {
    tm.sync();
    for (int c = tm.rank; c < C; c += tm.size) {
      const int m = (NM > 1 && c >= cols[0]) ? 1 : 0, j = m ? c - cols[0] : c;
      const double *p = part + c;
      double s;
      if constexpr (G == 2) s = p[0] + p[C];
      else if constexpr (G == 4) s = (p[0] + p[C]) + (p[2 * C] + p[3 * C]);
      else s = ((p[0] + p[C]) + (p[2 * C] + p[3 * C])) + ((p[4 * C] + p[5 * C]) + (p[6 * C] + p[7 * C]));
      emit(m, j, s);
    }
  }
  tm.sync();
}

// cols_apply_g with the largest group count that the team and the shared-memory region
// part (cap doubles) allow
template <int NM, class Emit>
__device__ __forceinline__ void cols_apply(const Team &tm, const double *const *M, const int *rows, const int *cols,
                                           int ld, const double *const *y, double *part, int cap, Emit emit)
{
  const int C = cols[0] + (NM > 1 ? cols[NM - 1] : 0);
  const int lim = tm.size < cap ? tm.size : cap;
  if (C > 0 && 8 * C <= lim) cols_apply_g<NM, 8>(tm, M, rows, cols, ld, y, part, emit);
  else if (C > 0 && 4 * C <= lim) cols_apply_g<NM, 4>(tm, M, rows, cols, ld, y, part, emit);
  else if (C > 0 && 2 * C <= lim) cols_apply_g<NM, 2>(tm, M, rows, cols, ld, y, part, emit);
  else {
    // one thread per column (more columns than threads: stride over them)
    for (int c0 = 0; c0 < C; c0 += tm.size) {
      const int c = c0 + tm.rank;
      if (c < C) {
        const int m = (NM > 1 && c >= cols[0]) ? 1 : 0, j = m ? c - cols[0] : c;
        const double *Mm = M[m], *ym = y[m];
        double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int k = 0;
        for (; k + 7 < rows[m]; k += 8) {
#pragma unroll
          for (int u = 0; u < 8; u++) a[u] += Mm[(size_t)(k + u) * ld + j] * ym[k + u];
        }
        for (; k < rows[m]; k++) a[0] += Mm[(size_t)k * ld + j] * ym[k];
        emit(m, j, ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7])));
      }
    }
    tm.sync();
  }
}

// The inner F/H fixed point of one sphere solved directly (the exact form): with
// fb = Vfix + cLH1 LH + cLF1 LF and hb = Dfix + cLH2 LH + cLF2 LF, (F, H) = G (fb, hb),
// G (2 NP2 x 2 NP2, row-major, one warp per row) the solution operator of the fixed
// point of CSolExpCenter::solveFH (src/expcenter.cpp:1079-1135) prepared per sphere
// type by pbsam_direct_kernel.  Returns computeDev2 (src/expcenter.cpp:1336-1370) of H.
__device__ __noinline__ double solve_direct(const Team &tm, const Tab &T, const TypeView &tv, const Scr &sc, int ts,
                                            double *F, double *H, const double *LF, const double *LH, double *red,
                                            int *stats, double omega)
{
  const int NP = T.NP, NP2 = NP * NP, n2 = 2 * NP2;
  const double *cst = tv.cst + (size_t)ts * CST_N * NP;
  const double *Dfix = tv.Dfix + (size_t)ts * NP2, *Vfix = tv.Vfix + (size_t)ts * NP2;
  const double *G = tv.Gdir + (size_t)ts * n2 * n2;
  double *x = sc.xs, *Hold = sc.sol, *Fold = sc.sol + NP2;
  for (int k = tm.rank; k < NP2; k += tm.size) {
    int n = (int)sqrt((double)k);
    while (n * n > k) n--;
    while ((n + 1) * (n + 1) <= k) n++;
    x[k] = Vfix[k] + cst[CST_LH1 * NP + n] * LH[k] + cst[CST_LF1 * NP + n] * LF[k];
    x[NP2 + k] = Dfix[k] + cst[CST_LH2 * NP + n] * LH[k] + cst[CST_LF2 * NP + n] * LF[k];
    Hold[k] = H[k];
    Fold[k] = F[k];
  }
  tm.sync();
  {
    const double *Ms[1] = {G}, *xs[1] = {x};
    const int nr[1] = {n2};
    rows_apply<1, 4>(tm, Ms, nr, nr, n2, xs, n2, [&](int, int r, double acc) {
      // omega != 1: the sweep's update over-relaxed (the fixed point is the same)
      if (r < NP2) F[r] = omega == 1.0 ? acc : Fold[r] + omega * (acc - Fold[r]);
      else H[r - NP2] = omega == 1.0 ? acc : Hold[r - NP2] + omega * (acc - Hold[r - NP2]);
    });
  }
  tm.sync();
  double pd = 0.0, ps = 0.0;
  for (int u = tm.rank; u < NP2; u += tm.size) {
    int n = (int)sqrt((double)u);
    while (n * n > u) n--;
    while ((n + 1) * (n + 1) <= u) n++;
    const double a = Hold[u], b = H[u], df = a - b;
    const double wt = (u == n * n) ? 1.0 : 2.0;
    pd += wt * (df * df);
    ps += wt * (a * a + b * b);
  }
  double td, tsm;
  team_sum2(tm, pd, ps, red, td, tsm);
  if (tm.rank == 0 && stats) { stats[1] += 1; stats[2] += 1; }
  return tsm > 0.0 ? td / (4 * tsm) : 0.0;
}

// F/H solve + surface charges of one sphere (src/expcenter.cpp:594-629)
__device__ double solve_surface(const Team &tm, const Sys &y, int s, bool rotH)
{
  const Tab &T = y.c->T;
  const int ts = y.ts(s);
  PhaseClock pc{y.tph, 0};
  pc.start(tm);
  double dv = y.c->prm.exact
                  ? solve_direct(tm, T, y.c->tv, y.sc, ts, y.F(s), y.H(s), y.LFS(s), y.LHS(s), y.red, y.stats(),
                                 rotH ? 1.0 : y.c->prm.exact_relax)
                  : solve_fh(tm, y.cw, y.tph, T, y.c->tv, y.c->prm, y.sc, ts, 1, y.F(s), y.H(s), y.LFS(s), y.LHS(s),
                             y.red, y.stats());
  pc.stop(tm, PH_SOLVE);
  pc.start(tm);
  if (rotH) {
    const RotState mr = y.molrot(y.mol(s));
    rot_apply_xi(tm, mr, y.H(s), y.Hrot(s), y.NP, true, y.NP);
  }
  const double *cst = y.c->tv.cst + (size_t)ts * CST_N * y.NP;
  const double dA = 4 * PB_PI / double(y.c->tv.nspx[ts]);
  double totF[1], tot[1];
  if (y.c->prm.exact && y.c->tv.spang && y.cw.size == 1)
    surface_q2_ang(tm, T, y.sc, y.c->tv.spang + 4 * (size_t)y.c->tv.spx_off[ts], y.npts(s), dA, y.F(s), T.CONST2,
                   y.qF(s), y.H(s), cst + CST_CHGH * y.NP, y.qH(s), totF, tot, y.red);
  else
    crew_surface_q2<1>(tm, y.cw, T, y.sc, y.red, y.spx(s), y.npts(s), dA, y.F(s), T.CONST2, y.qF(s), totF, y.H(s),
                       cst + CST_CHGH * y.NP, y.qH(s), tot);
  double tF = totF[0];
  pc.stop(tm, PH_SURF);
  if (tm.rank == 0) {
    y.c->bv.tF[y.sc1(s)] = tF;
    y.c->bv.tH[y.sc1(s)] = tot[0];
    y.c->bv.hscale[y.sc1(s)] = 1.0 / y.rad(s);
    y.c->bv.dev[y.sc1(s)] = dv;
  }
  tm.sync();
  return dv;
}

__device__ double recompute_from_self(const Team &tm, const Sys &y, int s)   // src/molecule.cpp:1136-1160
{
  const int ts = y.ts(s);
  reexpand_LS(tm, y, s, true);
  const double *LHi = y.c->tv.LHintra + (size_t)ts * y.NP2, *LFi = y.c->tv.LFintra + (size_t)ts * y.NP2;
  const double *Fs = y.c->tv.Fself + (size_t)ts * y.NP2, *Hs = y.c->tv.Hself + (size_t)ts * y.NP2;
  for (int i = tm.rank; i < y.NP2; i += tm.size) {
    y.LHS(s)[i] = y.LS(s)[i] + LHi[i];
    y.LFS(s)[i] = LFi[i];
    y.F(s)[i] = Fs[i];
    y.H(s)[i] = Hs[i];
  }
  tm.sync();
  return solve_surface(tm, y, s, true);
}

// (a, b) += (rows of degree < pF of NF) xF, (rows of degree < pH of NH) xH, nothing
// beyond (NF, NH: NP2 x NP2 row-major), reading the columns of degree < pinF (pinH)
__device__ __noinline__ void num_apply2(const Team &tm, const double *NF, const double *NH, int pF, int pH, int pinF,
                                        int pinH, const double *xF, const double *xH, double *a, double *b, int NP2)
{
  const double *Ms[2] = {NF, NH}, *xs[2] = {xF, xH};
  const int rows[2] = {pF * pF, pH * pH}, cols[2] = {pinF * pinF, pinH * pinH};
  rows_apply<2, 2>(tm, Ms, rows, cols, NP2, xs, NP2, [&](int m, int r, double v) { (m ? b : a)[r] += v; });
  tm.sync();
}

// outF[j] += sum over rows k of degree < pF of NF[k][j] yF[k] for the columns j of
// degree < pinF, and the same for H (the transpose of num_apply2); part: shared memory
// of cap doubles for the column groups' partial sums
__device__ __noinline__ void num_apply2_T(const Team &tm, const double *NF, const double *NH, int pF, int pH, int pinF,
                                          int pinH, const double *yF, const double *yH, double *outF, double *outH,
                                          int NP2, double *part, int cap)
{
  const double *Ms[2] = {NF, NH}, *ys[2] = {yF, yH};
  const int rows[2] = {pF * pF, pH * pH}, cols[2] = {pinF * pinF, pinH * pinH};
  cols_apply<2>(tm, Ms, rows, cols, NP2, ys, part, cap, [&](int m, int j, double v) { (m ? outH : outF)[j] += v; });
}

// intra near re-expansion with the latest values (src/molecule.cpp:1413-1473).
// part 0: every near neighbour, LFS = sum, LHS = LS + sum.  The exact form splits the
// sum: its sweeps update only the polarized spheres, so the terms of the other
// neighbours (F, H and surface charges fixed for the whole solve) are summed once per
// evaluation (part 1, into slots 0 and 1 of the sphere's gradient work set gLHN,
// which the exact form does not use otherwise) and every sweep adds the polarized
// neighbours' terms to them (part 2).
__device__ void reexpand_intra_near(const Team &tm, const Sys &y, int s, int part = 0)
{
  const Tab &T = y.c->T;
  const int ts = y.ts(s), i = y.mol(s);
  const int mo = y.c->bv.mol_off[i];
  const int to = y.c->tv.type_off[y.c->bv.mol_type[i]];
  double *a = y.sc.E(7), *bq = y.sc.E(8);
  double *LF = part == 1 ? y.gLHN(s) : y.LFS(s), *LH = part == 1 ? y.gLHN(s) + y.NP2 : y.LHS(s);
  if (part == 1) {
    tzero(tm, LF, y.NP2);
    tzero(tm, LH, y.NP2);
  } else if (part == 2) {
    const double *cF = y.gLHN(s), *cH = y.gLHN(s) + y.NP2, *ls = y.LS(s);
    for (int t = tm.rank; t < y.NP2; t += tm.size) { LF[t] = cF[t]; LH[t] = ls[t] + cH[t]; }
  } else {
    tzero(tm, LF, y.NP2);
    tcopy(tm, LH, y.LS(s), y.NP2);
  }
  tm.sync();
  const double *ci = y.cen(s);
  for (int e = y.c->tv.near_off[ts]; e < y.c->tv.near_off[ts + 1]; e++) {
    const int kj = y.c->tv.near[e];
    const int s2 = mo + kj;
    if (part != 0 && (y.nipol(s2) > 0) != (part == 2)) continue;
    const double *cj = y.c->tv.cen + 3 * (to + kj);
    const double P[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
    const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
    const double rj = y.rad(s2);
    const double sep = rho - y.rad(s) - rj;
    const int pF = compute_order(y.NP, rho, y.c->bv.tF[y.sc1(s2)], rj);
    const int pH = compute_order(y.NP, rho, y.c->bv.tH[y.sc1(s2)], rj);
    PhaseClock pc{y.tph, 0};
    pc.start(tm);
    const bool analytic = sep > 0 && !(sep < y.c->prm.min_sep_numeric);
    const int slot = (part != 0 && y.c->tv.nslot) ? y.c->tv.nslot[e] : -1;
    if (slot >= 0 && y.c->tv.nkind[slot] == (analytic ? 0 : 1)) {
      // the exact form's precomputed operators of the pair, the same maps of F and H of
      // s2: an analytic transform at order p is the block of degrees < p of its
      // full-order operator, a numeric one the rows of degree < p.  The pair's terms
      // are added into LF and LH as they are formed (each entry by the one lane that
      // sums it: the same additions as through a and bq below)
      const double *NF = y.c->tv.Nmat + (size_t)slot * 2 * y.NP2 * y.NP2;
      num_apply2(tm, NF, NF + (size_t)y.NP2 * y.NP2, pF, pH, analytic ? pF : y.NP, analytic ? pH : y.NP, y.F(s2),
                 y.H(s2), LF, LH, y.NP2);
      pc.stop(tm, analytic ? PH_INTRA : PH_NUMERIC);
      continue;
    } else if (analytic) {
      PairXf X;
      table_pair(tm, T, y.c->tv, y.sc, intra_pair(y.c->tv, ts, s - mo, kj), pH, pF, rj, y.rad(s), X);
      MultiVec V;
      V.n = 2;
      V.in[0] = y.F(s2); V.out[0] = a; V.useF[0] = true;
      V.in[1] = y.H(s2); V.out[1] = bq; V.useF[1] = false;
      pair_apply_multi(tm, T, y.sc, X, V, false);
      pc.stop(tm, PH_INTRA);
    } else {
      crew_numeric_expand2<1>(tm, y.cw, T, y.sc, y.spx(s2), y.npts(s2), P, y.rad(s),
                              NumSet{y.qF(s2), true, false, pF, a}, NumSet{y.qH(s2), true, true, pH, bq});
      pc.stop(tm, PH_NUMERIC);
    }
    for (int t = tm.rank; t < y.NP2; t += tm.size) { LF[t] += a[t]; LH[t] += bq[t]; }
    tm.sync();
  }
}

__device__ double recompute(const Team &tm, const Sys &y, int s)             // src/molecule.cpp:1168-1229
{
  const int ts = y.ts(s);
  // the exact form computes LS once before its sweeps (its sources, the Hrot of the
  // first round, stay fixed)
  if (!y.c->prm.exact) reexpand_LS(tm, y, s, false);
  reexpand_intra_near(tm, y, s, y.c->prm.exact ? 2 : 0);
  const double *LHf = y.c->tv.LHfar + (size_t)ts * y.NP2, *LFf = y.c->tv.LFfar + (size_t)ts * y.NP2;
  for (int i = tm.rank; i < y.NP2; i += tm.size) { y.LHS(s)[i] += LHf[i]; y.LFS(s)[i] += LFf[i]; }
  tm.sync();
  return solve_surface(tm, y, s, false);
}

// gradient re-expansion of neighbour m's rotated H into sphere s, accumulated in acc (3*NP2)
__device__ __noinline__ void grad_xform_from(const Team &tm, const Sys &y, int s, int sm, bool self, double *acc)
{
  const Tab &T = y.c->T;
  double ci[3], cm[3];
  y.cen_lab(s, ci);
  y.cen_lab(sm, cm);
  // prepareDTA takes the plain difference of the (wrapped) centres, no minimum image
  // (src/molecule.cpp:1515, 1546, 1562, 1602, 1619)
  double P[3] = {ci[0] - cm[0], ci[1] - cm[1], ci[2] - cm[2]};
  const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
  const double TQ = self ? y.c->tv.tHself[y.ts(sm)] : y.c->bv.tH[y.sc1(sm)];
  const int p = compute_order(y.NP, rho, TQ, y.rad(sm));
  PairXf X;
  prep_pair(tm, T, y.sc, P, p, 0, y.rad(sm), y.rad(s), true, X);
  double *G = y.sc.G(0);
  pair_apply_grad(tm, T, y.sc, X, self ? y.HselfRot(sm) : y.Hrot(sm), G);
  add_vec_into(tm, acc, G, 3 * y.NP2);
}

// truncation order of the re-expansion of sphere sm into sphere s (src/molecule.cpp:1516)
__device__ __forceinline__ int pair_order(const Sys &y, int s, int sm, bool self)
{
  double ci[3], cm[3];
  y.cen_lab(s, ci);
  y.cen_lab(sm, cm);
  double P[3] = {ci[0] - cm[0], ci[1] - cm[1], ci[2] - cm[2]};   // as grad_xform_from
  const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
  const double TQ = self ? y.c->tv.tHself[y.ts(sm)] : y.c->bv.tH[y.sc1(sm)];
  return compute_order(y.NP, rho, TQ, y.rad(sm));
}

// grad_xform_from run by one warp (tw) with its own scratch ws, added into acc
__device__ __noinline__ void grad_xform_warp(const WarpTeam &tw, const Sys &y, const Scr &ws, int s, int sm, bool self,
                                             double *acc)
{
  const Tab &T = y.c->T;
  double ci[3], cm[3];
  y.cen_lab(s, ci);
  y.cen_lab(sm, cm);
  const double P[3] = {ci[0] - cm[0], ci[1] - cm[1], ci[2] - cm[2]};   // as grad_xform_from
  const int p = pair_order(y, s, sm, self);
  PairXf X;
  prep_pair(tw, T, ws, P, p, 0, y.rad(sm), y.rad(s), true, X);
  double *G = ws.G(0);
  pair_apply_grad(tw, T, ws, X, self ? y.HselfRot(sm) : y.Hrot(sm), G);
  add_vec_into(tw, acc, G, 3 * y.NP2);
}

// This CTA's share of a list of gradient re-expansions into sphere s: the
// neighbours of s's polarization list (use_ipol) then of its interaction list
// (use_iact), optionally only those of molecule filter_mol; entries rank,
// rank + size, ... are summed into part (3 * NP2, written here).  The pair orders
// are computed first, one entry per thread.  When the pole order is at most
// PBSAM_WARP_MAX_NP and the share holds at least two pairs of order <=
// PBSAM_WARP_P per warp (most pairs of these lists are far apart
// and of low order, too narrow to keep a whole CTA busy), those pairs are dealt
// round-robin to the CTA's warps, each transforming its pairs alone, and the
// warps' sums are added in warp order; the other pairs are added one by one, each
// transformed by the whole CTA.
__device__ __noinline__ void dta_share(const Team &tm, const Sys &y, int s, bool self, int filter_mol, bool use_ipol, bool use_iact,
                          int rank, int size, double *part)
{
  const int NP2 = y.NP2, nw = tm.size >> 5, w = tm.rank >> 5;
  const int pw = y.NP < PBSAM_WARP_P ? y.NP : PBSAM_WARP_P;
  const int n1 = use_ipol ? y.nipol(s) : 0, n2 = use_iact ? y.niact(s) : 0;
  const int cnt = (n1 + n2 > rank) ? (n1 + n2 - rank + size - 1) / size : 0;
  const BatchView &bv = y.c->bv;
  int *ord = bv.dorder + ((size_t)y.b * bv.crew + rank) * bv.S;     // order of local entry u, -1 if filtered out
  int n_low = 0;
  for (int u0 = 0; u0 < cnt; u0 += tm.size) {
    const int u = u0 + tm.rank;
    int low = 0;
    if (u < cnt) {
      const int e = rank + u * size;
      const int sm = e < n1 ? y.ipol(s)[e] : y.iact(s)[e - n1];
      int o = -1;
      if (filter_mol < 0 || y.mol(sm) == filter_mol) o = pair_order(y, s, sm, self);
      ord[u] = o;
      low = (o >= 0 && o <= pw);
    }
    n_low += __syncthreads_count(low);
  }
  const bool warps = y.NP <= PBSAM_WARP_MAX_NP && n_low >= 2 * nw;
  if (warps) {
    const WarpTeam tw{tm.rank & 31, 32};
    const Scr ws = warp_scr(wscr_of(bv, y.b, rank, w), y.NP);
    double *wacc = ws.misc;
    tzero(tw, wacc, 3 * NP2);
    tw.sync();
    int j = 0;
    for (int u = 0; u < cnt; u++) {
      const int o = ord[u];
      if (o < 0 || o > pw) continue;
      if ((j++ % nw) != w) continue;
      const int e = rank + u * size;
      grad_xform_warp(tw, y, ws, s, e < n1 ? y.ipol(s)[e] : y.iact(s)[e - n1], self, wacc);
    }
    tm.sync();
    const size_t moff = (size_t)(warp_scr(wscr_of(bv, y.b, rank, 0), y.NP).misc - wscr_of(bv, y.b, rank, 0));
    for (int i = tm.rank; i < 3 * NP2; i += tm.size) {
      double v = 0.0;
      for (int q = 0; q < nw; q++) v += wscr_of(bv, y.b, rank, q)[moff + i];
      part[i] = v;
    }
  } else {
    tzero(tm, part, 3 * NP2);
  }
  tm.sync();
  for (int u = 0; u < cnt; u++) {
    const int o = ord[u];
    if (o < 0 || (warps && o <= pw)) continue;
    const int e = rank + u * size;
    grad_xform_from(tm, y, s, e < n1 ? y.ipol(s)[e] : y.iact(s)[e - n1], self, part);
  }
}

// acc (3 * NP2) += the gradient re-expansions of that list (prepareDTA /
// prepareDTA_iself, src/molecule.cpp:1483-1628), shared by the crew: each CTA sums
// its share in its own scratch, the leader adds the shares in rank order.
__device__ void crew_dta(const Team &tm, const Sys &y, int s, bool self, int filter_mol, bool use_ipol, bool use_iact,
                         double *acc)
{
  PhaseClock pc{y.tph, 0};
  pc.start(tm);
  const Crew &cw = y.cw;
  if (cw.size == 1) {
    double *part = y.sc.G(7);
    dta_share(tm, y, s, self, filter_mol, use_ipol, use_iact, 0, 1, part);
    add_vec_into(tm, acc, part, 3 * y.NP2);
    pc.stop(tm, PH_DTA);
    return;
  }
  cg::cluster_group cl = cg::this_cluster();
  {
    CrewCmd c;
    c.op = 3; c.s = s; c.self = self ? 1 : 0; c.filter_mol = filter_mol;
    c.use_ipol = use_ipol ? 1 : 0; c.use_iact = use_iact ? 1 : 0; c.acc = acc;
    crew_post(tm, cw, c);
  }
  cl.sync();
  dta_share(tm, y, s, self, filter_mol, use_ipol, use_iact, 0, cw.size, y.sc.G(7));
  cl.sync();                    // every CTA's share is in its scratch
  const BatchView &bv = y.c->bv;
  const int n = 3 * y.NP2;
  const size_t off = (size_t)(y.sc.G(7) - scr_of(bv, y.b, 0));
  for (int i = tm.rank; i < n; i += tm.size) {
    double v = acc[i];
    for (int q = 0; q < cw.size; q++) v += scr_of(bv, y.b, q)[off + i];
    acc[i] = v;
  }
  tm.sync();
  pc.stop(tm, PH_DTA);
}

__device__ void prepare_dta_iself(const Team &tm, const Sys &y, int s)     // src/molecule.cpp:1584-1628
{
  double *acc = y.gLHN(s);
  tzero(tm, acc, 3 * y.NP2);
  tm.sync();
  crew_dta(tm, y, s, true, -1, true, true, acc);
}

// This CTA's share of the analytic re-expansions that feed one gradient solve of
// sphere s w.r.t. molecule j (reexpandGrad / reexpandIntraGrad, src/molecule.cpp:
// 1681-1802).  kind 0: the rotated gradient H of the inter-molecular neighbours
// into out0 (tGrot); kind 1: the gradient F and H of the intra list's analytic
// pairs into out0 (LGF) and out1 (LGH2).  Entries counted in list order, this CTA
// taking every size-th from rank; contributions are added to the outputs.
__device__ __noinline__ void grad_share(const Team &tm, const Sys &y, int s, int j, int kind, int rank, int size, double *out0,
                           double *out1)
{
  const Tab &T = y.c->T;
  const BatchView &bv = y.c->bv;
  const int NP2 = y.NP2, i = y.mol(s), ts = y.ts(s);
  int cnt = 0;
  if (kind == 0) {
    double ci[3];
    y.cen_lab(s, ci);
    for (int e = 0; e < y.nipol(s); e++) {
      const int sm = y.ipol(s)[e];
      if (i != j && y.mol(sm) != j) continue;
      if ((cnt++ % size) != rank) continue;
      double cm[3];
      y.cen_lab(sm, cm);
      double P[3] = {ci[0] - cm[0], ci[1] - cm[1], ci[2] - cm[2]};
      min_image(y.c->prm.box, P);
      const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
      const int p = compute_order(y.NP, rho, bv.maxgH[y.sc1(sm)], y.rad(sm));
      PairXf X;
      prep_pair(tm, T, y.sc, P, p, 0, y.rad(sm), y.rad(s), false, X);
      const double *src = y.gw(bv.gHrotw, bv.gkey[y.sc1(sm)]);
      MultiVec V;
      V.n = 3;
      for (int cc = 0; cc < 3; cc++) { V.in[cc] = src + cc * NP2; V.out[cc] = out0 + cc * NP2; V.useF[cc] = false; }
      pair_apply_multi(tm, T, y.sc, X, V, true);
    }
    return;
  }
  const int nlist = (i == j) ? bv.intraPol_n[(size_t)y.b * bv.nmol + j] : bv.interMol_n[(size_t)y.b * bv.nmol + j];
  const int *lst = (i == j) ? bv.intraPol + ((size_t)y.b * bv.nmol + j) * y.S : bv.interMol + ((size_t)y.b * bv.nmol + j) * y.S;
  const double *cis = y.cen(s);
  for (int e = 0; e < nlist; e++) {
    const int sm = lst[e];
    if (i != j && y.mol(sm) != i) continue;
    if (sm == s) continue;
    const double *cms = y.cen(sm);
    const double P[3] = {cis[0] - cms[0], cis[1] - cms[1], cis[2] - cms[2]};
    const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
    const double rm = y.rad(sm);
    const double sep = rho - y.rad(s) - rm;
    if (!(sep > 0 && !(sep < y.c->prm.min_sep_numeric))) continue;
    if ((cnt++ % size) != rank) continue;
    const int pF = compute_order(y.NP, rho, bv.maxgF[y.sc1(sm)], rm);
    const int pH = compute_order(y.NP, rho, bv.maxgH[y.sc1(sm)], rm);
    PairXf X;
    table_pair(tm, T, y.c->tv, y.sc, intra_pair(y.c->tv, ts, s - bv.mol_off[i], sm - bv.mol_off[i]), pH, pF, rm,
               y.rad(s), X);
    const int km = bv.gkey[y.sc1(sm)];
    MultiVec V;
    V.n = 6;
    for (int cc = 0; cc < 3; cc++) {
      V.in[cc] = y.gw(bv.gFw, km) + cc * NP2; V.out[cc] = out0 + cc * NP2; V.useF[cc] = true;
      V.in[3 + cc] = y.gw(bv.gHw, km) + cc * NP2; V.out[3 + cc] = out1 + cc * NP2; V.useF[3 + cc] = false;
    }
    pair_apply_multi(tm, T, y.sc, X, V, true);
  }
}

// grad_share over the whole crew: the leader adds its share straight into the
// outputs, each helper into zeroed buffers of its own scratch, which the leader
// then adds in rank order.
__device__ void crew_grad(const Team &tm, const Sys &y, int s, int j, int kind, double *out0, double *out1)
{
  const Crew &cw = y.cw;
  if (cw.size == 1) { grad_share(tm, y, s, j, kind, 0, 1, out0, out1); return; }
  cg::cluster_group cl = cg::this_cluster();
  {
    CrewCmd c;
    c.op = 4; c.s = s; c.filter_mol = j; c.self = kind;
    crew_post(tm, cw, c);
  }
  cl.sync();
  grad_share(tm, y, s, j, kind, 0, cw.size, out0, out1);
  cl.sync();                    // helpers' shares are in their scratch
  const BatchView &bv = y.c->bv;
  const int n = 3 * y.NP2;
  const size_t o5 = (size_t)(y.sc.G(5) - scr_of(bv, y.b, 0)), o6 = (size_t)(y.sc.G(6) - scr_of(bv, y.b, 0));
  for (int i = tm.rank; i < n; i += tm.size) {
    double v = out0[i];
    for (int q = 1; q < cw.size; q++) v += scr_of(bv, y.b, q)[o5 + i];
    out0[i] = v;
    if (kind == 1) {
      double w = out1[i];
      for (int q = 1; q < cw.size; q++) w += scr_of(bv, y.b, q)[o6 + i];
      out1[i] = w;
    }
  }
  tm.sync();
}

// one gradient recompute of sphere s w.r.t. molecule j (src/molecule.cpp:1680-1843)
__device__ double recompute_grad(const Team &tm, const Sys &y, int s, int j, int key)
{
  const Tab &T = y.c->T;
  const BatchView &bv = y.c->bv;
  const int NP2 = y.NP2, i = y.mol(s), ts = y.ts(s);
  double *tGrot = y.sc.G(1), *LGH = y.sc.G(2), *LGF = y.sc.G(3), *LGH2 = y.sc.G(4), *tmpG = y.sc.G(5);
  PhaseClock gx{y.tph, 0};
  gx.start(tm);
  tcopy(tm, tGrot, y.gw(bv.tGw, key), 3 * NP2);
  tm.sync();
  PhaseClock sub{y.tph, 0};
  sub.start(tm);
  crew_grad(tm, y, s, j, 0, tGrot, nullptr);
  sub.stop(tm, PH_GX_INTER);
  const RotState mr = y.molrot(i);
  for (int cc = 0; cc < 3; cc++) rot_apply_xi(tm, mr, tGrot + cc * NP2, LGH + cc * NP2, y.NP, false, y.NP);
  tm.sync();
  if (j == i) { tcopy(tm, y.gLHN(s), LGH, 3 * NP2); tm.sync(); }
  tzero(tm, LGF, 3 * NP2);
  tzero(tm, LGH2, 3 * NP2);
  tm.sync();
  // analytic pairs of the intra list shared by the crew, then the numeric ones
  sub.start(tm);
  crew_grad(tm, y, s, j, 1, LGF, LGH2);
  sub.stop(tm, PH_GX_ANALYTIC);
  sub.start(tm);
  const int nlist = (i == j) ? bv.intraPol_n[(size_t)y.b * bv.nmol + j] : bv.interMol_n[(size_t)y.b * bv.nmol + j];
  const int *lst = (i == j) ? bv.intraPol + ((size_t)y.b * bv.nmol + j) * y.S : bv.interMol + ((size_t)y.b * bv.nmol + j) * y.S;
  const double *cis = y.cen(s);
  for (int e = 0; e < nlist; e++) {
    const int sm = lst[e];
    if (i != j && y.mol(sm) != i) continue;
    if (sm == s) continue;
    const double *cms = y.cen(sm);
    const double P[3] = {cis[0] - cms[0], cis[1] - cms[1], cis[2] - cms[2]};
    const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
    const double rm = y.rad(sm);
    const double sep = rho - y.rad(s) - rm;
    if (sep > 0 && !(sep < y.c->prm.min_sep_numeric)) continue;
    const int pF = compute_order(y.NP, rho, bv.maxgF[y.sc1(sm)], rm);
    const int pH = compute_order(y.NP, rho, bv.maxgH[y.sc1(sm)], rm);
    double *tmpH = y.sc.G(6);
    crew_numeric_expand2<3>(tm, y.cw, T, y.sc, y.spx(sm), y.npts(sm), P, y.rad(s),
                            NumSet{y.gFp(sm), true, false, pF, tmpG}, NumSet{y.gHp(sm), true, true, pH, tmpH});
    add_vec_into(tm, LGF, tmpG, 3 * NP2);
    add_vec_into(tm, LGH2, tmpH, 3 * NP2);
  }
  sub.stop(tm, PH_GX_NUMERIC);
  add_vec_into(tm, LGH, LGH2, 3 * NP2);
  gx.stop(tm, PH_GRX);
  double *gF = y.gw(bv.gFw, key), *gHk = y.gw(bv.gHw, key);
  PhaseClock pc{y.tph, 0};
  pc.start(tm);
  const double dv = solve_fh(tm, y.cw, y.tph, T, y.c->tv, y.c->prm, y.sc, ts, 3, gF, gHk, LGF, LGH, y.red, y.stats());
  pc.stop(tm, PH_SOLVE);
  pc.start(tm);
  for (int cc = 0; cc < 3; cc++) rot_apply_xi(tm, mr, gHk + cc * NP2, y.gw(bv.gHrotw, key) + cc * NP2, y.NP, true, y.NP);
  tm.sync();
  // exposed gradient charges (src/expcenter.cpp:1377-1412)
  const double *cst = y.c->tv.cst + (size_t)ts * CST_N * y.NP;
  const double dA = 4 * PB_PI / double(y.c->tv.nspx[ts]);
  double totF[3], totH[3];
  crew_surface_q2<3>(tm, y.cw, T, y.sc, y.red, y.spx(s), y.npts(s), dA, gF, T.CONST2, y.gFp(s), totF, gHk,
                     cst + CST_CHGH * y.NP, y.gHp(s), totH);
  if (tm.rank == 0) {
    double mf = totF[0] > totF[1] ? totF[0] : totF[1];
    if (totF[2] > mf) mf = totF[2];
    double mh = totH[0] > totH[1] ? totH[0] : totH[1];
    if (totH[2] > mh) mh = totH[2];
    bv.maxgF[y.sc1(s)] = mf;
    bv.maxgH[y.sc1(s)] = mh;
    bv.dev[y.sc1(s)] = dv;
    y.stats()[3] += 1;
  }
  tm.sync();
  pc.stop(tm, PH_GSURF);
  return dv;
}

// multipole-local inner product with scale bookkeeping (src/expansion.h:705-741)
__device__ double inprod_ml(const double *M, double mscale, const double *L, double lscale, int NP)
{
  double sum = 0.0, fact = 1 / (mscale * lscale), scale = 1.0;
  for (int n = 0; n < NP; n++) {
    double s = 0.0;
    for (int mm = 1; mm < 2 * n + 1; mm++) s += M[IDX(n) + mm] * L[IDX(n) + mm];
    s *= 2.0;
    s += M[IDX(n)] * L[IDX(n)];
    sum += scale * s;
    scale *= fact;
  }
  return sum;
}

// ------------------------------------------------------------------ the force kernel
// helper CTAs: serve the leader's commands until it sends the exit command.  y is
// the helper's view of the system (its own scratch, no phase clocks).
__device__ void crew_serve(const Team &tm, const Sys &y)
{
  const Crew &cw = y.cw;
  const Tab &T = y.c->T;
  const Scr &sc = y.sc;
  cg::cluster_group cl = cg::this_cluster();
  for (;;) {
    cl.sync();
    const CrewCmd c = *cw.cmd;    // posted by the leader before the barrier
    if (c.op == 1) {
      solve_core(tm, cw, nullptr, T, y.c->tv, y.c->prm, sc, c.xg, c.ts, c.D, c.F, c.H, c.LF, c.LH, y.red, nullptr);
    } else if (c.op == 2) {
      if (c.NC == 1)
        numeric_expand2<1>(tm, T, sc, c.pts, c.N, c.shift, c.nscale, c.A, c.B, cw.rank, cw.size, sc.tile);
      else
        numeric_expand2<3>(tm, T, sc, c.pts, c.N, c.shift, c.nscale, c.A, c.B, cw.rank, cw.size, sc.tile);
    } else if (c.op == 3) {
      dta_share(tm, y, c.s, c.self != 0, c.filter_mol, c.use_ipol != 0, c.use_iact != 0, cw.rank, cw.size, sc.G(7));
    } else if (c.op == 4) {
      tzero(tm, sc.G(5), 3 * y.NP2);
      if (c.self == 1) tzero(tm, sc.G(6), 3 * y.NP2);
      tm.sync();
      grad_share(tm, y, c.s, c.filter_mol, c.self, cw.rank, cw.size, sc.G(5), sc.G(6));
    } else if (c.op == 5) {
      double t1[3], t2[3];
      if (c.NC == 1) surface_q2<1>(tm, T, sc, c.pts, c.N, c.dA, c.E1, c.c1, c.q1, c.E2, c.c2, c.q2, cw.rank, cw.size, t1, t2, y.red);
      else surface_q2<3>(tm, T, sc, c.pts, c.N, c.dA, c.E1, c.c1, c.q1, c.E2, c.c2, c.q2, cw.rank, cw.size, t1, t2, y.red);
      if (tm.rank == 0)
        for (int k = 0; k < c.NC; k++) { cw.cmd->ptot[k] = t1[k]; cw.cmd->ptot[3 + k] = t2[k]; }
    } else break;
    cl.sync();
  }
  cl.sync();                    // the leader may leave once every helper has read the exit
}

// a helper CTA's view of system b: its own scratch block, no phase clocks
__device__ Sys helper_sys(const Ctx &c, const Crew &cw, int b, void *dsm, double *red)
{
  Sys y;
  y.c = &c; y.b = b; y.NP = c.T.NP; y.NP2 = y.NP * y.NP; y.S = c.bv.S;
  y.cw = cw;
  y.sc = make_scr(scr_of(c.bv, b, cw.rank), y.NP, dsm);
  y.red = red;
  y.tph = nullptr;
  return y;
}

__device__ __noinline__ bool backward_body(const Team &tm, const Sys &y);   // pbsam_adjoint.cu

// One system (the crew leader's part): CMolecule::computeForces.
__device__ void forces_body(const Team &tm, const Ctx &c, const Crew &cw, int b, void *dsm, double *red)
{
  const BatchView &bv = c.bv;
  Sys y;
  y.c = &c; y.b = b; y.NP = c.T.NP; y.NP2 = y.NP * y.NP; y.S = bv.S;
  y.cw = cw;
  y.sc = make_scr(scr_of(bv, b, 0), y.NP, dsm);
  y.red = red;
  y.tph = bv.tphase + (size_t)b * PH_N;
  const int S = bv.S, nmol = bv.nmol, NP2 = y.NP2;
  int *st = y.stats();
  PhaseClock total{y.tph, 0};
  if (tm.rank == 0) {
    for (int k = 0; k < 8; k++) st[k] = 0;
    for (int k = 0; k < PH_N; k++) y.tph[k] = 0.0;
    st[5] = cw.size;
    bv.status[b] = PBSAM_STATUS_OK;
  }
  total.start(tm);
  PhaseClock setup{y.tph, 0};
  setup.start(tm);
  for (int t = tm.rank; t < nmol * 3; t += tm.size) {
    bv.force[(size_t)b * nmol * 3 + t] = 0.0;
    bv.torque[(size_t)b * nmol * 3 + t] = 0.0;
  }
  // a pose with a non-finite coordinate or a zero quaternion is refused before any
  // pair test (NaN distances would silently drop every pair)
  {
    int bad = 0;
    for (int t = tm.rank; t < nmol * 7; t += tm.size) {
      const double v = t < nmol * 3 ? bv.pos[(size_t)b * nmol * 3 + t] : bv.quat[(size_t)b * nmol * 4 + (t - nmol * 3)];
      if (!isfinite(v)) bad = 1;
    }
    for (int i = tm.rank; i < nmol; i += tm.size) {
      const double *q = bv.quat + 4 * ((size_t)b * nmol + i);
      if (!(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3] > 0.0)) bad = 1;
    }
    if (__syncthreads_or(bad)) {
      if (tm.rank == 0) bv.status[b] = PBSAM_STATUS_NAN;
      return;
    }
  }
  // with a periodic box the molecule centres are wrapped into it as CMolecule::setPos
  // does (src/molecule.h:325): pair distances take the minimum image, but the
  // reference's energy and prepareDTA use the plain difference of the wrapped centres
  if (c.prm.box > 0.0) {
    for (int t = tm.rank; t < nmol * 3; t += tm.size) {
      double *v = const_cast<double *>(bv.pos) + (size_t)b * nmol * 3 + t;   // the system's own pose buffer
      *v = *v - c.prm.box * round(*v / c.prm.box);
    }
    tm.sync();
  }
  // sphere centres for this pose (CMolecule::rotate / rotateCenters)
  for (int s = tm.rank; s < S; s += tm.size) {
    const double *q = bv.quat + 4 * ((size_t)b * nmol + y.mol(s));
    double qn[4];
    const double in = 1.0 / sqrt((q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + q[0] * q[0]);
    qn[0] = q[0] * in; qn[1] = q[1] * in; qn[2] = q[2] * in; qn[3] = q[3] * in;
    qrot(qn, y.cen(s), y.cenRot(s));
  }
  tm.sync();
  if (nmol == 1) return;
  // ---- pair lists (src/molecule.cpp:1035-1126, 122-166)
  double *sep = bv.sep + (size_t)b * S * S;
  for (int u = tm.rank; u < S * S; u += tm.size) {
    const int s1 = u / S, s2 = u % S;
    double a[3], d[3];
    y.cen_lab(s1, a);
    y.cen_lab(s2, d);
    double dd[3] = {a[0] - d[0], a[1] - d[1], a[2] - d[2]};
    min_image(c.prm.box, dd);
    sep[u] = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]) - y.rad(s1) - y.rad(s2);
  }
  tm.sync();
  if (tm.rank == 0) {
    int ok = 1;
    for (int s = 0; s < S; s++) { bv.ipol_n[y.sc1(s)] = 0; bv.iact_n[y.sc1(s)] = 0; }
    for (int i = 0; i < nmol; i++) bv.interX[(size_t)b * nmol + i] = 0;
    for (int j = 1; j < nmol && ok; j++) {
      int neigh[64];
      int nn = 0;
      for (int i = 0; i < j; i++) {
        const double *pi = bv.pos + 3 * ((size_t)b * nmol + i), *pj = bv.pos + 3 * ((size_t)b * nmol + j);
        double dd[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
        min_image(c.prm.box, dd);
        const double c2c = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
        const double ms = c2c - c.tv.maxR[bv.mol_type[i]] - c.tv.maxR[bv.mol_type[j]];
        if (ms < c.prm.interact_cut && nn < 64) neigh[nn++] = i;
      }
      for (int kj = bv.mol_off[j]; kj < bv.mol_off[j + 1] && ok; kj++)
        for (int ii = 0; ii < nn && ok; ii++) {
          const int i = neigh[ii];
          for (int ki = bv.mol_off[i]; ki < bv.mol_off[i + 1]; ki++) {
            const double g = sep[(size_t)ki * S + kj];
            if (g <= 0) { ok = 0; break; }
            if (g < c.prm.interact_cut) {
              if (g > c.prm.inter_cut) {
                y.iact(ki)[bv.iact_n[y.sc1(ki)]++] = kj;
                y.iact(kj)[bv.iact_n[y.sc1(kj)]++] = ki;
              } else {
                y.ipol(ki)[bv.ipol_n[y.sc1(ki)]++] = kj;
                y.ipol(kj)[bv.ipol_n[y.sc1(kj)]++] = ki;
              }
              bv.interX[(size_t)b * nmol + i] = 1;
              bv.interX[(size_t)b * nmol + j] = 1;
            }
          }
        }
    }
    if (!ok) bv.status[b] = PBSAM_STATUS_OVERLAP;
    else {
      for (int i = 0; i < nmol; i++) bv.interMol_n[(size_t)b * nmol + i] = 0;
      for (int s = 0; s < S; s++) {
        unsigned long long added = 0;   // molecules already credited (bit mask; nmol <= 64)
        for (int e = 0; e < y.nipol(s); e++) {
          const int j = y.mol(y.ipol(s)[e]);
          if (added & (1ULL << j)) continue;
          int &n = bv.interMol_n[(size_t)b * nmol + j];
          bv.interMol[((size_t)b * nmol + j) * S + n++] = s;
          added |= (1ULL << j);
        }
      }
      for (int j = 0; j < nmol; j++) {
        int &np = bv.intraPol_n[(size_t)b * nmol + j], &na = bv.intraAct_n[(size_t)b * nmol + j];
        np = 0; na = 0;
        for (int s = bv.mol_off[j]; s < bv.mol_off[j + 1]; s++) {
          if (y.nipol(s) > 0) bv.intraPol[((size_t)b * nmol + j) * S + np++] = s;
          else if (y.niact(s) > 0) bv.intraAct[((size_t)b * nmol + j) * S + na++] = s;
        }
      }
    }
  }
  tm.sync();
  if (bv.status[b] != PBSAM_STATUS_OK) return;
  const Tab &T = c.T;
  // ---- polarize_mutual: molecule rotations, rotated self H (src/molecule.cpp:2002-2015)
  for (int i = 0; i < nmol; i++) {
    if (!bv.interX[(size_t)b * nmol + i]) continue;
    const double *q = bv.quat + 4 * ((size_t)b * nmol + i);
    double qn[4];
    const double in = 1.0 / sqrt((q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + q[0] * q[0]);
    qn[0] = q[0] * in; qn[1] = q[1] * in; qn[2] = q[2] * in; qn[3] = q[3] * in;
    double th, ph, xi;
    quat_angles(qn, th, ph, xi);
    RotState rs;
    double2 *Rm = bv.molR + ((size_t)b * nmol + i) * rot_off(2 * y.NP - 1);
    rot_compute(tm, T, th, ph, xi, y.NP, false, rs, Rm, nullptr, y.sc.sh, y.sc.lvA, y.sc.lvB);
    if (tm.rank == 0) {
      double *v = bv.molRS + ((size_t)b * nmol + i) * 16;
      v[0] = rs.sing ? 1.0 : 0.0; v[1] = rs.cost; v[2] = rs.sint; v[3] = rs.cott; v[4] = rs.xi;
      v[5] = rs.exphi.x; v[6] = rs.exphi.y; v[7] = rs.exxi.x; v[8] = rs.exxi.y;
    }
    tm.sync();
    const RotState mr = y.molrot(i);
    for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
      if (y.nipol(s) == 0 && y.niact(s) == 0) continue;
      rot_apply_xi(tm, mr, c.tv.Hself + (size_t)y.ts(s) * NP2, y.HselfRot(s), y.NP, true, y.NP);
      tm.sync();
      tcopy(tm, y.Hrot(s), y.HselfRot(s), NP2);
      tm.sync();
    }
  }
  setup.stop(tm, PH_SETUP);
  // ---- first round from self values
  double dev = 0.0, MAXDEV = 0.0;
  int mtotal = 0;
  {
    // MAXDEV: the largest change of any sphere (the reference takes the largest of the
    // molecules' largest, the same number)
    for (int i = 0; i < nmol; i++) {
      double dmol = 0.0;
      if (bv.interX[(size_t)b * nmol + i])
        for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
          if (y.nipol(s) == 0) continue;
          const double d = recompute_from_self(tm, y, s);
          dmol += d;
          if (MAXDEV < d) MAXDEV = d;
          mtotal++;
        }
      dev += dmol;
    }
  }
  // the exact form, once before its sweeps: the inter-molecular LS (its sources, the
  // rotated H of the first round, are not updated by the sweeps) and the near terms of
  // the neighbours the sweeps leave fixed
  if (c.prm.exact)
    for (int i = 0; i < nmol; i++)
      if (bv.interX[(size_t)b * nmol + i])
        for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++)
          if (y.nipol(s) > 0) {
            reexpand_LS(tm, y, s, false);
            reexpand_intra_near(tm, y, s, 1);
          }
  int ct = 1;
  const double itot = (mtotal > 0 ? 1.0 / mtotal : 0);
  // the exact form sweeps to the fixed point (exact_tol) whatever max_polar_dev says
  const double tol2 = c.prm.exact ? c.prm.exact_tol * c.prm.exact_tol : c.prm.max_polar_dev * c.prm.max_polar_dev;
  while (dev * itot > tol2 && ct < c.prm.max_pol_rounds) {
    dev = 0.0;
    double next_max = 0.0;
    for (int i = 0; i < nmol; i++) {
      double dmol = 0.0;
      if (bv.interX[(size_t)b * nmol + i])
        for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
          if (y.nipol(s) == 0) continue;
          double d = bv.dev[y.sc1(s)];
          // the exact form recomputes every sphere (the selective update can leave a
          // sphere whose last change was small out of date)
          if (c.prm.exact || d > 0.1 * MAXDEV) d = recompute(tm, y, s);
          if (next_max < d) next_max = d;
          dmol += d;
        }
      dev += dmol;
    }
    MAXDEV = next_max;
    ct++;
  }
  if (tm.rank == 0) {
    st[0] = ct;
    if (dev * itot > tol2) st[4] |= 1;   // polarization hit the sweep cap
  }
  if (c.prm.exact) {
    // forces and torques: the adjoint of the converged state (lab frame)
    tm.sync();
    PhaseClock bk{y.tph, 0};
    bk.start(tm);
    const bool ok = backward_body(tm, y);
    bk.stop(tm, PH_GRX);
    for (int t = tm.rank; t < nmol * 3; t += tm.size) {
      bv.force[(size_t)b * nmol * 3 + t] = -bv.dpos[(size_t)b * nmol * 3 + t];
      bv.torque[(size_t)b * nmol * 3 + t] = -bv.drot[(size_t)b * nmol * 3 + t];
    }
    int bad = 0;
    for (int t = tm.rank; t < nmol * 3; t += tm.size)
      if (!isfinite(bv.force[(size_t)b * nmol * 3 + t]) || !isfinite(bv.torque[(size_t)b * nmol * 3 + t])) bad = 1;
    bad = __syncthreads_or(bad);
    if (tm.rank == 0) {
      if (!ok) st[4] |= 2;
      if (bad) bv.status[b] = PBSAM_STATUS_NAN;
      else if (st[4]) bv.status[b] = PBSAM_STATUS_NOT_CONVERGED;
    }
    tm.sync();
    total.stop(tm, PH_TOTAL);
    return;
  }
  // ---- gradient phase (src/molecule.cpp:2081-2228)
  for (int j = 0; j < nmol; j++) {
    const int ni = bv.interMol_n[(size_t)b * nmol + j];
    if (ni == 0) {
      if (bv.interX[(size_t)b * nmol + j])
        for (int s = bv.mol_off[j]; s < bv.mol_off[j + 1]; s++)
          if (y.nipol(s) > 0 || y.niact(s) > 0) prepare_dta_iself(tm, y, s);
      continue;
    }
    const int na = bv.intraPol_n[(size_t)b * nmol + j];
    const int jsize = ni + na;
    const double itj = 1.0 / double(jsize);
    const int *inter = bv.interMol + ((size_t)b * nmol + j) * S;
    const int *intra = bv.intraPol + ((size_t)b * nmol + j) * S;
    PhaseClock book{y.tph, 0};
    book.start(tm);
    for (int s = tm.rank; s < S; s += tm.size) bv.gkey[y.sc1(s)] = -1;
    tm.sync();
    for (int k = tm.rank; k < jsize; k += tm.size) bv.gkey[y.sc1(k < ni ? inter[k] : intra[k - ni])] = k;
    for (int k = 0; k < jsize; k++) {
      tzero(tm, y.gw(bv.gFw, k), 3 * NP2);
      tzero(tm, y.gw(bv.gHw, k), 3 * NP2);
      tzero(tm, y.gw(bv.gHrotw, k), 3 * NP2);
      tzero(tm, y.gw(bv.tGw, k), 3 * NP2);
    }
    tm.sync();
    book.stop(tm, PH_GBOOK);
    // prepareDTA (src/molecule.cpp:1483-1571)
    for (int k = 0; k < jsize; k++) {
      const int s = k < ni ? inter[k] : intra[k - ni];
      double *acc = y.gw(bv.tGw, k);
      if (k < ni) crew_dta(tm, y, s, false, j, true, false, acc);
      else crew_dta(tm, y, s, false, -1, true, true, acc);
    }
    double *dg = bv.dgrad + (size_t)b * S;
    double dv = 0.0;
    for (int k = 0; k < jsize; k++) {
      const int s = k < ni ? inter[k] : intra[k - ni];
      const double d = recompute_grad(tm, y, s, j, k);
      if (tm.rank == 0) dg[k] = d;
      dv += d;
    }
    tm.sync();
    int gct = 1, k = 0;
    while (dv * itj > tol2 && gct < c.prm.max_pol_rounds) {
      dv -= dg[k];
      const int s = k < ni ? inter[k] : intra[k - ni];
      const double d = recompute_grad(tm, y, s, j, k);
      tm.sync();
      if (tm.rank == 0) dg[k] = d;
      tm.sync();
      dv += d;
      k++;
      if (k == jsize) { k = 0; gct++; }
    }
    if (tm.rank == 0 && dv * itj > tol2) st[4] |= 2;   // a gradient phase hit the sweep cap
    for (int h = 0; h < na; h++) {
      const int s = intra[h];
      tcopy(tm, y.gH(s), y.gw(bv.gHw, bv.gkey[y.sc1(s)]), 3 * NP2);
    }
    tm.sync();
    const int nact = bv.intraAct_n[(size_t)b * nmol + j];
    for (int h = 0; h < nact; h++) prepare_dta_iself(tm, y, bv.intraAct[((size_t)b * nmol + j) * S + h]);
  }
  tm.sync();
  PhaseClock fclk{y.tph, 0};
  fclk.start(tm);
  // ---- forces and torques (src/moldynamics.cpp:524-550, src/expcenter.cpp:123-149)
  double *fk = y.sc.misc;   // [S][3]
  for (int s = tm.rank; s < S; s += tm.size) {
    double f[3] = {0.0, 0.0, 0.0};
    const int i = y.mol(s);
    if (bv.interX[(size_t)b * nmol + i] && (y.nipol(s) > 0 || y.niact(s) > 0)) {
      const double r = y.rad(s);
      for (int cc = 0; cc < 3; cc++) {
        if (y.nipol(s) > 0) {
          f[cc] -= inprod_ml(y.H(s), 1.0 / r, y.gLHN(s) + cc * NP2, r, y.NP);
          f[cc] -= inprod_ml(y.gH(s) + cc * NP2, 1.0 / r, y.LS(s), r, y.NP);
        } else {
          f[cc] -= inprod_ml(c.tv.Hself + (size_t)y.ts(s) * NP2, c.tv.hself_scale[y.ts(s)], y.gLHN(s) + cc * NP2, r, y.NP);
        }
      }
    }
    fk[3 * s] = f[0]; fk[3 * s + 1] = f[1]; fk[3 * s + 2] = f[2];
  }
  tm.sync();
  if (tm.rank < nmol) {
    const int i = tm.rank;
    double F[3] = {0, 0, 0}, Tq[3] = {0, 0, 0};
    if (bv.interX[(size_t)b * nmol + i])
      for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
        if (y.nipol(s) == 0 && y.niact(s) == 0) continue;
        const double *f = fk + 3 * s, *cn = y.cen(s);
        F[0] += f[0]; F[1] += f[1]; F[2] += f[2];
        Tq[0] += cn[1] * f[2] - cn[2] * f[1];
        Tq[1] += cn[2] * f[0] - cn[0] * f[2];
        Tq[2] += cn[0] * f[1] - cn[1] * f[0];
      }
    const double *q = bv.quat + 4 * ((size_t)b * nmol + i);
    double qn[4];
    double in = 1.0 / sqrt((q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + q[0] * q[0]);
    qn[0] = q[0] * in; qn[1] = -(q[1] * in); qn[2] = -(q[2] * in); qn[3] = -(q[3] * in);
    in = 1.0 / sqrt((qn[1] * qn[1] + qn[2] * qn[2] + qn[3] * qn[3]) + qn[0] * qn[0]);
    qn[0] *= in; qn[1] *= in; qn[2] *= in; qn[3] *= in;
    qrot(qn, F, bv.force + ((size_t)b * nmol + i) * 3);
    qrot(qn, Tq, bv.torque + ((size_t)b * nmol + i) * 3);
  }
  tm.sync();
  // per-system outcome: a non-finite force or torque (a blown-up expansion,
  // CExpan::isBlownup, src/expansion.h:216-221) or a sweep cap that was hit ("Polarization
  // does not converge", src/molecule.cpp:1963-1967; the forces are still returned)
  {
    int bad = 0;
    for (int t = tm.rank; t < nmol * 3; t += tm.size)
      if (!isfinite(bv.force[(size_t)b * nmol * 3 + t]) || !isfinite(bv.torque[(size_t)b * nmol * 3 + t])) bad = 1;
    bad = __syncthreads_or(bad);
    if (tm.rank == 0) {
      if (bad) bv.status[b] = PBSAM_STATUS_NAN;
      else if (st[4]) bv.status[b] = PBSAM_STATUS_NOT_CONVERGED;
    }
  }
  fclk.stop(tm, PH_FORCE);
  total.stop(tm, PH_TOTAL);
}

// Grid: crews of cluster-size CTAs (a plain launch is a crew of one), one per
// system; crew k works on system list[k] (list == nullptr: system k).
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_forces_kernel(Ctx c, const int *list)
{
  extern __shared__ double2 dsm[];
  if (threadIdx.x == 0 && c.T.NP <= PBSAM_SMEM_IMAT_NP) {
    // the IMat staging region's flag (stage_imat): staging on
    unsigned dsz;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dsz));
    if (dsz >= forces_smem_bytes(c.T.NP))
      *(int *)((char *)dsm + team_smem_bytes(c.T.NP) + imat_stride(c.T.NP * c.T.NP) * sizeof(double) + 8) = 0;
  }
  __syncthreads();
  __shared__ double red[PBSAM_TEAM];
  __shared__ CrewCmd cmd;
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  cg::cluster_group cl = cg::this_cluster();
  const Crew cw{(int)cl.block_rank(), (int)cl.num_blocks(), &cmd};
  const int k = blockIdx.x / cw.size;
  const int b = list ? list[k] : k;
  if (b >= c.bv.B) return;                 // whole crews only: the grid is (systems in the list) * size
  if (c.bv.fmask && c.bv.fmask[b] == 0) return;   // the whole crew skips a masked system
  if (cw.rank != 0) {
    crew_serve(tm, helper_sys(c, cw, b, dsm, red));
    return;
  }
  forces_body(tm, c, cw, b, dsm, red);
  crew_finish(tm, cw);
}

// One launch over the systems of several handles (pbsam_group_*), possibly of
// different molecule lists, sphere counts and pole orders: CTA k evaluates system
// work[k].y of handle work[k].x with that handle's context view (one CTA per system;
// the dynamic shared memory is that of the largest pole order in the group).
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_forces_group_kernel(const Ctx *cs, const int2 *work)
{
  extern __shared__ double2 dsm[];
  const int2 w = work[blockIdx.x];
  const Ctx &c = cs[w.x];
  if (threadIdx.x == 0 && c.T.NP <= PBSAM_SMEM_IMAT_NP) {
    unsigned dsz;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dsz));
    if (dsz >= forces_smem_bytes(c.T.NP))
      *(int *)((char *)dsm + team_smem_bytes(c.T.NP) + imat_stride(c.T.NP * c.T.NP) * sizeof(double) + 8) = 0;
  }
  __syncthreads();
  __shared__ double red[PBSAM_TEAM];
  __shared__ CrewCmd cmd;
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const Crew cw{0, 1, &cmd};
  const int b = w.y;
  if (b >= c.bv.B) return;
  if (c.bv.fmask && c.bv.fmask[b] == 0) return;
  forces_body(tm, c, cw, b, dsm, red);
}

// interaction energy on the state left by the last force evaluation.
// lab == 0: the reference's convention (src/moldynamics.cpp:358-386,
//   src/molecule.cpp:1850-1890): unrotated sphere centres and molecule-frame H, so
//   the value ignores the molecules' orientations.
// lab == 1: the same sum in the lab frame: sphere centres at pos + q*cen and every
//   H rotated to the lab frame by its molecule's orientation (the rotation the
//   solve applies to H before re-expanding it to other molecules); invariant under
//   a rigid rotation or translation of the whole system.
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_energy_kernel(Ctx c, int lab)
{
  extern __shared__ double2 dsm[];
  __shared__ double red[PBSAM_TEAM];
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const BatchView &bv = c.bv;
  const int b = blockIdx.x;
  if (b >= bv.B) return;
  Sys y;
  y.c = &c; y.b = b; y.NP = c.T.NP; y.NP2 = y.NP * y.NP; y.S = bv.S;
  y.cw = Crew{0, 1, nullptr};
  y.sc = make_scr(scr_of(bv, b, 0), y.NP, dsm);
  y.red = red;
  y.tph = nullptr;
  const Tab &T = c.T;
  const int NP2 = y.NP2;
  double pot = 0.0;
  if (bv.status[b] == PBSAM_STATUS_OK || bv.status[b] == PBSAM_STATUS_NOT_CONVERGED) {
    if (lab) {
      // lab-frame centres and H of every sphere
      for (int i = 0; i < bv.nmol; i++) {
        const double *q = bv.quat + 4 * ((size_t)b * bv.nmol + i);
        double qn[4];
        const double in = 1.0 / sqrt((q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + q[0] * q[0]);
        qn[0] = q[0] * in; qn[1] = q[1] * in; qn[2] = q[2] * in; qn[3] = q[3] * in;
        for (int s = bv.mol_off[i] + tm.rank; s < bv.mol_off[i + 1]; s += tm.size) qrot(qn, y.cen(s), y.cenRot(s));
        double th, ph, xi;
        quat_angles(qn, th, ph, xi);
        RotState rs;
        double2 *Rm = bv.molR + ((size_t)b * bv.nmol + i) * rot_off(2 * y.NP - 1);
        rot_compute(tm, T, th, ph, xi, y.NP, false, rs, Rm, nullptr, y.sc.sh, y.sc.lvA, y.sc.lvB);
        tm.sync();
        for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
          rot_apply_xi(tm, rs, y.H(s), bv.Hlab + ((size_t)b * bv.S + s) * NP2, y.NP, true, y.NP);
          tm.sync();
        }
      }
      tm.sync();
    }
    for (int i = 0; i < bv.nmol; i++)
      for (int j = i + 1; j < bv.nmol; j++) {
        double e = 0.0;
        const double *pi = bv.pos + 3 * ((size_t)b * bv.nmol + i), *pj = bv.pos + 3 * ((size_t)b * bv.nmol + j);
        for (int si = bv.mol_off[i]; si < bv.mol_off[i + 1]; si++) {
          double *Lki = y.sc.E(9), *tL = y.sc.E(10);
          tzero(tm, Lki, y.NP2);
          tm.sync();
          const double *ci = lab ? y.cenRot(si) : y.cen(si);
          for (int sj = bv.mol_off[j]; sj < bv.mol_off[j + 1]; sj++) {
            const double *cj = lab ? y.cenRot(sj) : y.cen(sj);
            double P[3] = {(pi[0] + ci[0]) - (pj[0] + cj[0]), (pi[1] + ci[1]) - (pj[1] + cj[1]),
                           (pi[2] + ci[2]) - (pj[2] + cj[2])};
            // the reference's energy takes the plain difference of the wrapped centres
            // (src/molecule.cpp:1873); the lab-frame form the minimum image
            if (lab) min_image(c.prm.box, P);
            const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
            const int pi2j = compute_order(y.NP, rho, bv.tH[y.sc1(si)], y.rad(si));
            const int pj2i = compute_order(y.NP, rho, bv.tH[y.sc1(sj)], y.rad(sj));
            const int minp = pi2j < pj2i ? pi2j : pj2i;
            PairXf X;
            prep_pair(tm, T, y.sc, P, minp, 0, y.rad(sj), y.rad(si), false, X);
            pair_apply(tm, T, y.sc, X, false, lab ? bv.Hlab + ((size_t)b * bv.S + sj) * NP2 : y.H(sj), tL);
            add_vec_into(tm, Lki, tL, y.NP2);
          }
          e += inprod_ml(lab ? bv.Hlab + ((size_t)b * bv.S + si) * NP2 : y.H(si), bv.hscale[y.sc1(si)], Lki,
                         y.rad(si), y.NP);
          tm.sync();
        }
        pot += e;
      }
  }
  if (tm.rank == 0) bv.energy[b] = pot;
}

// lab-frame sphere centres and H of every sphere of every system (one team per
// system), for the lab-frame potential
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_hlab_kernel(Ctx c)
{
  extern __shared__ double2 dsm[];
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const BatchView &bv = c.bv;
  const int b = blockIdx.x;
  if (b >= bv.B) return;
  const int NP = c.T.NP, NP2 = NP * NP;
  const Scr sc = make_scr(scr_of(bv, b, 0), NP, dsm);
  for (int i = 0; i < bv.nmol; i++) {
    const double *q = bv.quat + 4 * ((size_t)b * bv.nmol + i);
    double qn[4];
    const double in = 1.0 / sqrt((q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + q[0] * q[0]);
    qn[0] = q[0] * in; qn[1] = q[1] * in; qn[2] = q[2] * in; qn[3] = q[3] * in;
    for (int s = bv.mol_off[i] + tm.rank; s < bv.mol_off[i + 1]; s += tm.size)
      qrot(qn, c.tv.cen + 3 * bv.sph_ts[s], bv.cenRot + 3 * ((size_t)b * bv.S + s));
    double th, ph, xi;
    quat_angles(qn, th, ph, xi);
    RotState rs;
    double2 *Rm = bv.molR + ((size_t)b * bv.nmol + i) * rot_off(2 * NP - 1);
    rot_compute(tm, c.T, th, ph, xi, NP, false, rs, Rm, nullptr, sc.sh, sc.lvA, sc.lvB);
    tm.sync();
    for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
      rot_apply_xi(tm, rs, bv.H + ((size_t)b * bv.S + s) * NP2, bv.Hlab + ((size_t)b * bv.S + s) * NP2, NP, true, NP);
      tm.sync();
    }
  }
}

// Electrostatic potential at points from every sphere's H (CMolecule::computePotInSpace,
// src/moldynamics.cpp:470-506, for molecules that are not aggregated, as in the BD
// drivers): at each sphere the local expansion of a unit charge at the point
// (CLExpan, screened, truncated at computeOrder of the sphere's total charge) against
// H.  One thread per (system, point).  lab = 0: the reference's convention, the
// unrotated sphere centres and molecule-frame H (as its energy); lab = 1: the rotated
// centres and lab-frame H of pbsam_hlab_kernel.  pts: [npts][3], or per system
// [B][npts][3] when per_system; pot: [B][npts].
__global__ void pbsam_potential_kernel(Ctx c, int npts, const double *pts, int per_system, int lab, double *pot)
{
  const BatchView &bv = c.bv;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)bv.B * npts) return;
  const int b = (int)(t / npts), k = (int)(t % npts);
  const double *P = pts + 3 * ((per_system ? (size_t)b * npts : 0) + k);
  const Tab &T = c.T;
  const int NP = T.NP, NP2 = NP * NP;
  double rad[64];
  double acc = 0.0;
  for (int i = 0; i < bv.nmol; i++) {
    const double *pi = bv.pos + 3 * ((size_t)b * bv.nmol + i);
    for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
      const int ts = bv.sph_ts[s];
      const double *cs = lab ? bv.cenRot + 3 * ((size_t)b * bv.S + s) : c.tv.cen + 3 * ts;
      double dq[3] = {P[0] - pi[0] - cs[0], P[1] - pi[1] - cs[1], P[2] - pi[2] - cs[2]};
      min_image(c.prm.box, dq);
      const Sph sp = cart2sph(dq[0], dq[1], dq[2]);
      const double r = c.tv.rad[ts];
      const int p = compute_order(NP, sp.rho, bv.tH[(size_t)b * bv.S + s], r);
      radial_factors(T, sp.rho, 1.0, true, true, p, r, rad);
      const double *H = (lab ? bv.Hlab : bv.H) + ((size_t)b * bv.S + s) * NP2;
      const double fact = 1.0 / (bv.hscale[(size_t)b * bv.S + s] * r);
      double scale = 1.0;
      double fn[64];
      for (int n = 0; n < p; n++) { fn[n] = scale * rad[n]; scale *= fact; }
      double st, ct;
      sincos(sp.theta, &st, &ct);
      for (int m = 0; m < p; m++)
        sh_column(T, ct, st, sp.phi, m, p, [&](int n, double re, double im) {
          if (m == 0) acc += fn[n] * H[IDX(n)] * re;
          else acc += 2.0 * fn[n] * (H[IDX(n) + 2 * m - 1] * re + H[IDX(n) + 2 * m] * im);
        });
    }
  }
  pot[t] = acc;
}

// state of every system reset to the self-polarized values (CSolExpCenter BD constructor,
// src/expcenter.cpp:398-425, and initGradient, src/expcenter.cpp:559-569)
__global__ void pbsam_init_kernel(Ctx c)
{
  const BatchView &bv = c.bv;
  const int b = blockIdx.x;
  const int NP2 = c.T.NP * c.T.NP;
  for (int s = 0; s < bv.S; s++) {
    const int ts = bv.sph_ts[s];
    const size_t o = ((size_t)b * bv.S + s) * NP2;
    for (int i = threadIdx.x; i < NP2; i += blockDim.x) {
      bv.F[o + i] = c.tv.Fself[(size_t)ts * NP2 + i];
      bv.H[o + i] = c.tv.Hself[(size_t)ts * NP2 + i];
      bv.Hrot[o + i] = c.tv.Hself[(size_t)ts * NP2 + i];
      bv.HselfRot[o + i] = 0.0;
      bv.LS[o + i] = 0.0; bv.LFS[o + i] = 0.0; bv.LHS[o + i] = 0.0;
    }
    for (int i = threadIdx.x; i < 3 * NP2; i += blockDim.x) {
      bv.gLHN[((size_t)b * bv.S + s) * 3 * NP2 + i] = 0.0;
      bv.gH[((size_t)b * bv.S + s) * 3 * NP2 + i] = 0.0;
    }
    const int p0 = bv.pt_off[s], np = bv.pt_off[s + 1] - p0, tp0 = c.tv.spx_off[ts];
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
      bv.qF[(size_t)b * bv.SP + p0 + i] = c.tv.qFself[tp0 + i];
      bv.qH[(size_t)b * bv.SP + p0 + i] = c.tv.qHself[tp0 + i];
    }
    for (int i = threadIdx.x; i < 3 * np; i += blockDim.x) {
      bv.gFp[((size_t)b * bv.SP + p0) * 3 + i] = 0.0;
      bv.gHp[((size_t)b * bv.SP + p0) * 3 + i] = 0.0;
    }
    if (threadIdx.x == 0) {
      const size_t k = (size_t)b * bv.S + s;
      bv.hscale[k] = c.tv.hself_scale[ts];
      bv.tF[k] = c.tv.tFself[ts];
      bv.tH[k] = c.tv.tHself[ts];
      bv.maxgF[k] = 0.0; bv.maxgH[k] = 0.0; bv.dev[k] = 0.0;
    }
  }
}

// ------------------------------------------------------------------ molecule-type setup
// per type sphere: constants (initMyConstants, src/expcenter.cpp:469-505), self
// surface charges (src/molecule.cpp:787-810), fixed-charge expansions and their
// Dirichlet/Neumann terms (src/expcenter.cpp:513-552, 1041-1060)
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_setup1_kernel(Ctx c, double *scr, long long scr_stride)
{
  extern __shared__ double2 dsm[];
  __shared__ double red[PBSAM_TEAM];
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const Tab &T = c.T;
  const TypeView &tv = c.tv;
  const int ts = blockIdx.x;
  const int NP = T.NP, NP2 = NP * NP;
  Scr sc = make_scr(scr + (size_t)ts * scr_stride, NP, dsm);
  int t = 0;
  while (tv.type_off[t + 1] <= ts) t++;
  const double rad = tv.rad[ts];
  double *cst = tv.cst + (size_t)ts * CST_N * NP;
  if (tm.rank == 0) {
    double bK[34], bI[34];
    const double val = T.kappa * rad, valsqr = val * val, exp_val = exp(-1.0 * val);
    const double eps = c.prm.idiel / c.prm.sdiel;
    bessel_k(T, bK, NP + 1, val);
    bessel_i(bI, NP + 1, val);
    for (int n = 0; n < NP; n++) {
      const double DH = -exp_val * bK[n], DF = 1.0;
      const double VH = exp_val * (n * bK[n] - (2 * n + 1) * bK[n + 1]), VF = -eps * n;
      cst[CST_H1 * NP + n] = VH;
      cst[CST_F1 * NP + n] = VF + (2 * n + 1);
      cst[CST_LF1 * NP + n] = -rad * eps * n;
      cst[CST_LH1 * NP + n] = rad * (n * bI[n] + valsqr * bI[n + 1] / double(2 * n + 3));
      cst[CST_H2 * NP + n] = DH + (2 * n + 1) / bI[n];
      cst[CST_F2 * NP + n] = DF;
      cst[CST_LF2 * NP + n] = rad;
      cst[CST_LH2 * NP + n] = -rad * bI[n];
      cst[CST_INVH * NP + n] = bI[n] * (T.CONST3[n]);
      cst[CST_CHGH * NP + n] = T.CONST2[n] / bI[n];
    }
  }
  tm.sync();
  const double *pts = tv.spx + 3 * (size_t)tv.spx_off[ts];
  const int npt = tv.spx_off[ts + 1] - tv.spx_off[ts];
  const double dA = 4.0 * PB_PI / double(tv.nspx[ts]);
  double totF[1], tot[1];
  surface_q2<1>(tm, T, sc, pts, npt, dA, tv.Fself + (size_t)ts * NP2, T.CONST2, tv.qFself + tv.spx_off[ts],
                tv.Hself + (size_t)ts * NP2, cst + CST_CHGH * NP, tv.qHself + tv.spx_off[ts], 0, 1, totF, tot, red);
  const double tF = totF[0];
  if (tm.rank == 0) { tv.tFself[ts] = tF; tv.tHself[ts] = tot[0]; }
  // fixed charges split into inside (multipole) / outside (local) sets, scaled by 1/eps_in
  const int q0 = tv.chg_off[t], nq = tv.chg_off[t + 1] - q0;
  double *win = sc.misc, *wout = sc.misc + nq;   // misc holds 4096 + S*S doubles (nq checked on the host)
  const double *cs = tv.cen + 3 * ts;
  for (int k = tm.rank; k < nq; k += tm.size) {
    const double *p = tv.chg_pos + 3 * (size_t)(q0 + k);
    const double dx = p[0] - cs[0], dy = p[1] - cs[1], dz = p[2] - cs[2];
    const double cq = tv.chg[q0 + k] / c.prm.idiel;
    const bool in = (dx * dx + dy * dy + dz * dz) < rad * rad;
    win[k] = in ? cq : 0.0;
    wout[k] = in ? 0.0 : cq;
  }
  tm.sync();
  double *Efix = sc.E(10), *Lfix = sc.E(11);
  numeric_expand<1>(tm, T, sc, tv.chg_pos + 3 * (size_t)q0, nq, cs, win, false, false, NP, rad, Efix);
  numeric_expand<1>(tm, T, sc, tv.chg_pos + 3 * (size_t)q0, nq, cs, wout, true, false, NP, rad, Lfix);
  // multipole of the charges assigned to this sphere (CExpCenter::setFixedCharges, src/expcenter.cpp:88-103)
  for (int k = tm.rank; k < nq; k += tm.size)
    win[k] = (tv.chg_lab[q0 + k] == ts - tv.type_off[t]) ? tv.chg[q0 + k] / c.prm.idiel : 0.0;
  tm.sync();
  numeric_expand<1>(tm, T, sc, tv.chg_pos + 3 * (size_t)q0, nq, cs, win, false, false, NP, rad,
                    tv.Eass + (size_t)ts * NP2);
  const double eps = c.prm.idiel / c.prm.sdiel;
  for (int k = tm.rank; k < NP2; k += tm.size) {
    int n = (int)sqrt((double)k);
    while (n * n > k) n--;
    while ((n + 1) * (n + 1) <= k) n++;
    const double DE = 1.0, DL = rad, VE = eps * (n + 1), VL = -eps * n * rad;
    tv.Dfix[(size_t)ts * NP2 + k] = DE * Efix[k] + DL * Lfix[k];
    tv.Vfix[(size_t)ts * NP2 + k] = VE * Efix[k] + VL * Lfix[k];
  }
}

// per type sphere: intra-molecular self local expansions (computeMolTypeValues,
// src/molecule.cpp:544-696)
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_setup2_kernel(Ctx c, double *scr, long long scr_stride)
{
  extern __shared__ double2 dsm[];
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const Tab &T = c.T;
  const TypeView &tv = c.tv;
  const int ts = blockIdx.x;
  const int NP = T.NP, NP2 = NP * NP;
  Scr sc = make_scr(scr + (size_t)ts * scr_stride, NP, dsm);
  int t = 0;
  while (tv.type_off[t + 1] <= ts) t++;
  const int t0 = tv.type_off[t], ns = tv.type_off[t + 1] - t0, ki = ts - t0;
  const double ri = tv.rad[ts];
  double *LFf = tv.LFfar + (size_t)ts * NP2, *LHf = tv.LHfar + (size_t)ts * NP2;
  double *LFi = tv.LFintra + (size_t)ts * NP2, *LHi = tv.LHintra + (size_t)ts * NP2;
  double *a = sc.E(10), *bq = sc.E(11);
  tzero(tm, LFf, NP2);
  tzero(tm, LHf, NP2);
  tm.sync();
  const int nb = tv.near_off[ts], ne = tv.near_off[ts + 1];
  const double *ci = tv.cen + 3 * ts;
  // far field (every sphere of the type not on the near list), analytic at full order
  for (int kj = 0; kj < ns; kj++) {
    if (kj == ki) continue;
    bool isnear = false;
    for (int e = nb; e < ne; e++) if (tv.near[e] == kj) isnear = true;
    if (isnear) continue;
    PairXf X;
    table_pair(tm, T, tv, sc, intra_pair(tv, ts, ki, kj), NP, NP, tv.rad[t0 + kj], ri, X);
    MultiVec V;
    V.n = 2;
    V.in[0] = tv.Fself + (size_t)(t0 + kj) * NP2; V.out[0] = a; V.useF[0] = true;
    V.in[1] = tv.Hself + (size_t)(t0 + kj) * NP2; V.out[1] = bq; V.useF[1] = false;
    pair_apply_multi(tm, T, sc, X, V, false);
    for (int i = tm.rank; i < NP2; i += tm.size) { LFf[i] += a[i]; LHf[i] += bq[i]; }
    tm.sync();
  }
  tcopy(tm, LFi, LFf, NP2);
  tcopy(tm, LHi, LHf, NP2);
  tm.sync();
  for (int e = nb; e < ne; e++) {
    const int kj = tv.near[e];
    const int tj = t0 + kj;
    const double *cj = tv.cen + 3 * tj;
    const double P[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
    const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
    const double rj = tv.rad[tj];
    const double sep = rho - ri - rj;
    if (sep > 0 && !(sep < c.prm.min_sep_numeric)) {
      PairXf X;
      table_pair(tm, T, tv, sc, intra_pair(tv, ts, ki, kj), NP, NP, rj, ri, X);
      MultiVec V;
      V.n = 2;
      V.in[0] = tv.Fself + (size_t)tj * NP2; V.out[0] = a; V.useF[0] = true;
      V.in[1] = tv.Hself + (size_t)tj * NP2; V.out[1] = bq; V.useF[1] = false;
      pair_apply_multi(tm, T, sc, X, V, false);
    } else {
      const int pF = compute_order(NP, rho, tv.tFself[tj], rj), pH = compute_order(NP, rho, tv.tHself[tj], rj);
      const double *pts = tv.spx + 3 * (size_t)tv.spx_off[tj];
      const int npt = tv.spx_off[tj + 1] - tv.spx_off[tj];
      numeric_expand2<1>(tm, T, sc, pts, npt, P, ri, NumSet{tv.qFself + tv.spx_off[tj], true, false, pF, a},
                         NumSet{tv.qHself + tv.spx_off[tj], true, true, pH, bq});
    }
    for (int i = tm.rank; i < NP2; i += tm.size) { LFi[i] += a[i]; LHi[i] += bq[i]; }
    tm.sync();
  }
}

// per intra pair entry e: rotation and translation coefficients at the full pole
// order (CXFormAIntra::reset, src/xforms.cpp:213-227), kept as the prefixes the
// apply reads (rotation n < NP, translation l < NP); entries of pairs that are
// re-expanded numerically are left unused.
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_setup3_kernel(Ctx c, int e0, int ne, double *scr, long long stride)
{
  extern __shared__ double2 dsm[];
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const Tab &T = c.T;
  const TypeView &tv = c.tv;
  const int NP = T.NP;
  const int e = e0 + blockIdx.x;
  if (blockIdx.x >= ne) return;
  const int NN = 2 * NP - 1;
  double *sh = scr + (size_t)blockIdx.x * stride;
  double *TH = sh + 4 * NP * NP, *kbuf = TH + tr_off(NN);
  double2 *lvA = dsm, *lvB = dsm + NN * NN;
  int ts = 0;
  while (tv.pair_off[ts + 1] <= e) ts++;
  int t = 0;
  while (tv.type_off[t + 1] <= ts) t++;
  const int ki = ts - tv.type_off[t], j = e - tv.pair_off[ts];
  const int tj = tv.type_off[t] + (j < ki ? j : j + 1);
  const double *ci = tv.cen + 3 * ts, *cj = tv.cen + 3 * tj;
  const double P[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
  const Sph S = cart2sph(P[0], P[1], P[2]);
  const double sep = S.rho - tv.rad[ts] - tv.rad[tj];
  if (!(sep > 0 && !(sep < c.prm.min_sep_numeric))) return;
  RotState rs;
  rot_compute(tm, T, S.theta, S.phi, PB_PI, NP, false, rs, tv.pR + (size_t)e * rot_off(NP), nullptr, sh, lvA, lvB);
  if (tm.rank == 0) {
    double *v = tv.pS + 16 * (size_t)e;
    v[0] = rs.sing ? 1.0 : 0.0; v[1] = rs.cost; v[2] = rs.sint; v[3] = rs.cott; v[4] = rs.xi;
    v[5] = rs.exphi.x; v[6] = rs.exphi.y; v[7] = rs.exxi.x; v[8] = rs.exxi.y;
  }
  TransState ts1;
  trans_compute(tm, T, S.rho, T.kappa, NP, tv.rad[tj], tv.rad[ts], false, ts1, TH, nullptr, kbuf);
  for (int i = tm.rank; i < tr_off(NP); i += tm.size) tv.pTH[(size_t)e * tr_off(NP) + i] = TH[i];
  tm.sync();
  trans_compute(tm, T, S.rho, 0.0, NP, tv.rad[tj], tv.rad[ts], false, ts1, TH, nullptr, kbuf);
  for (int i = tm.rank; i < tr_off(NP); i += tm.size) tv.pTF[(size_t)e * tr_off(NP) + i] = TH[i];
}


// Near-field operators of the exact form.  For intra near entry e (target type sphere
// u, source v = near[e]) the full-order maps LF_u += N_F F_v and LH_u += N_H H_v
// (NP2 x NP2, row-major).  Numeric pairs (kind 1): column j is the numeric expansion
// about u (numeric_expand2) of the surface charges (surface_q2) of a unit F_j (H_j) of
// v; both steps are linear and a truncation order p only drops output degrees >= p,
// so the rows of degree < p give the forward's expansion at that order.  Analytic
// pairs (kind 0): column j is the intra table transform (rotation, coaxial
// translation, rotation back) of a unit coefficient at full order; rotations keep
// degrees apart and the translation coefficients of degrees < p do not depend on p,
// so the block of degrees < p is the transform at order p.  One CTA per slot.
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_nummat_kernel(Ctx c, const int *slot_e, const int *slot_u, int s0,
                                                                  int ns, double *scr, long long stride, double *qw,
                                                                  long long qstride, double *Nmat)
{
  extern __shared__ double2 dsm[];
  __shared__ double red[PBSAM_TEAM];
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const int k = blockIdx.x;
  if (k >= ns) return;
  const Tab &T = c.T;
  const TypeView &tv = c.tv;
  const int NP = T.NP, NP2 = NP * NP;
  const int slot = s0 + k, e = slot_e[slot], u = slot_u[slot], kind = tv.nkind[slot];
  Scr sc = make_scr(scr + (size_t)k * stride, NP, dsm);
  int t = 0;
  while (tv.type_off[t + 1] <= u) t++;
  const int v = tv.type_off[t] + tv.near[e];
  const double *cu = tv.cen + 3 * u, *cv = tv.cen + 3 * v;
  const double P[3] = {cu[0] - cv[0], cu[1] - cv[1], cu[2] - cv[2]};
  const double *pts = tv.spx + 3 * (size_t)tv.spx_off[v];
  const int npt = tv.spx_off[v + 1] - tv.spx_off[v];
  const double dA = 4 * PB_PI / double(tv.nspx[v]);
  const double *cstv = tv.cst + (size_t)v * CST_N * NP;
  double *unit = sc.E(12), *outF = sc.E(10), *outH = sc.E(11);
  double *qF = qw + (size_t)k * qstride, *qH = qF + qstride / 2;
  double *NF = Nmat + (size_t)slot * 2 * NP2 * NP2, *NH = NF + (size_t)NP2 * NP2;
  tzero(tm, unit, NP2);
  tm.sync();
  for (int j = 0; j < NP2; j++) {
    if (tm.rank == 0) {
      unit[j] = 1.0;
      if (j > 0) unit[j - 1] = 0.0;
    }
    tm.sync();
    if (kind == 0) {
      // analytic pair: the intra table transform at full order (table_pair)
      PairXf X;
      table_pair(tm, T, tv, sc, intra_pair(tv, u, u - tv.type_off[t], tv.near[e]), NP, NP, tv.rad[v], tv.rad[u], X);
      MultiVec V;
      V.n = 2;
      V.in[0] = unit; V.out[0] = outF; V.useF[0] = true;
      V.in[1] = unit; V.out[1] = outH; V.useF[1] = false;
      pair_apply_multi(tm, T, sc, X, V, false);
    } else {
      double t1[1], t2[1];
      surface_q2<1>(tm, T, sc, pts, npt, dA, unit, T.CONST2, qF, unit, cstv + CST_CHGH * NP, qH, 0, 1, t1, t2, red);
      tm.sync();
      numeric_expand2<1>(tm, T, sc, pts, npt, P, tv.rad[u], NumSet{qF, true, false, NP, outF},
                         NumSet{qH, true, true, NP, outH});
    }
    tm.sync();
    for (int r = tm.rank; r < NP2; r += tm.size) {
      NF[(size_t)r * NP2 + j] = outF[r];
      NH[(size_t)r * NP2 + j] = outH[r];
    }
    tm.sync();
  }
}

}  // namespace pbsam
