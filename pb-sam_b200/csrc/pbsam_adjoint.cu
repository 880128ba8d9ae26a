// Exact form of the polarization solve and its adjoint (backward pass).
//
// The reference iterates each sphere's inner F/H fixed point
// (CSolExpCenter::solveFH, src/expcenter.cpp:1079-1135) to a tolerance or a cap;
// on the synthetic and golden molecules of this project the iteration matrix of
// that fixed point has spectral radius slightly above one (1.05-1.1), so the
// iterates drift once they have come close and the result depends on
// SOLVE_MAX_CT.  Its outer sweeps update a sphere only while its last change was
// above a tenth of the largest (src/molecule.cpp:2057), which can leave a sphere
// out of date.  The exact form solves the same equations to their fixed point:
//
//   * per sphere type, the inner fixed point is solved once for all right-hand
//     sides: G = A^-1 diag(C3 M, CI M), with A the fixed-point operator, M the
//     IMat and C3, CI the degree scalings; (F, H) = G (fb, hb) then costs one
//     2p^2 x 2p^2 product per solve instead of up to SOLVE_MAX_CT pairs of p^2 x p^2
//     IMat products (pbsam_direct_kernel, Gauss-Jordan elimination);
//   * every polarized sphere is swept until the root-mean-square relative change is
//     below exact_tol (1e-14 by default), so the state is the fixed point of the reference's equations (the first
//     round from self values, its rotated H kept for the later rounds, the
//     intra-molecular coupling, as polarize_mutual, src/molecule.cpp:1988-2263);
//   * the forces and torques are the exact negative gradient of the lab-frame
//     interaction energy of that state (pbsam_energy_kernel, lab = 1), computed by
//     the adjoint below in one backward sweep instead of the reference's
//     per-molecule, per-coordinate gradient solves (src/molecule.cpp:2081-2228).
//
// The backward pass transposes every linear step of the forward with the
// truncation orders and surface point sets held at their converged values.  Two
// identities keep it in the forward's own kernels: in the inner product weighted
// by W (1 for the m = 0 entry of a degree, 2 for the Re/Im entries of m > 0) the
// molecule rotations are orthogonal and the pair re-expansions are reciprocal, so
// R^T = W R^-1 W^-1 and T(b<-a)^T = W T(a<-b) W^-1 (checked to rounding in the
// oracle).  The numeric near field is transposed explicitly: its surface-charge
// map becomes a projection on the source sphere's points and its charge sum an
// evaluation of the target expansion at the points.
//
// Included by pbsam_api.cu after pbsam_kernels.cu.
namespace pbsam {

// ------------------------------------------------------------------ direct inner operator
// The exact form's point angles: (cos t, sin t, cos phi, sin phi) of every exposed
// point (relative to its sphere's centre), as surface_q2 computes them per call.
__global__ void pbsam_spang_kernel(TypeView tv, int TP, double *out)
{
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= TP) return;
  const double *pt = tv.spx + 3 * (size_t)h;
  const Sph s = cart2sph(pt[0], pt[1], pt[2]);
  double st, ct, sf, cf;
  sincos(s.theta, &st, &ct);
  sincos(s.phi, &sf, &cf);
  out[4 * (size_t)h] = ct;
  out[4 * (size_t)h + 1] = st;
  out[4 * (size_t)h + 2] = cf;
  out[4 * (size_t)h + 3] = sf;
}

// One CTA per type sphere ts0 + blockIdx.x: [A | Bd] (n x 2n, n = 2 NP2) reduced to
// [I | G] by Gauss-Jordan elimination with partial pivoting in the CTA's work block;
// G is copied to tv.Gdir.  Fixed point (src/expcenter.cpp:1079-1135):
//   F = C3 M (fb + cH1 H + cF1 F),  H = CI M (hb + cH2 H + cF2 F)
// so A = [[I - C3 M cF1, -C3 M cH1], [-CI M cF2, I - CI M cH2]], Bd = diag(C3 M, CI M).
// A zero pivot sets *err (a singular fixed point; the type cannot use the exact form).
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_direct_kernel(Tab T, TypeView tv, int ts0, double *work, int *err)
{
  __shared__ double rv[PBSAM_TEAM];
  __shared__ int ri[PBSAM_TEAM];
  __shared__ double s_piv;
  __shared__ int s_row;
  const int ts = ts0 + blockIdx.x;
  const int NP = T.NP, NP2 = NP * NP, n = 2 * NP2, w2 = 2 * n;
  const int ld = imat_ld(NP2);
  const double *M = tv.imat + (size_t)ts * imat_stride(NP2);
  const double *cst = tv.cst + (size_t)ts * CST_N * NP;
  double *W = work + (size_t)blockIdx.x * n * w2;
  auto degf = [](int k) {
    int d = (int)sqrt((double)k);
    while (d * d > k) d--;
    while ((d + 1) * (d + 1) <= k) d++;
    return d;
  };
  for (long long u = threadIdx.x; u < (long long)n * w2; u += blockDim.x) {
    const int r = (int)(u / w2), c = (int)(u % w2);
    const bool rH = r >= NP2, cH = (c % n) >= NP2;
    const int i = rH ? r - NP2 : r, kk = (c % n) - (cH ? NP2 : 0);
    const double m = M[(size_t)i * ld + kk];
    const double rs = rH ? cst[CST_INVH * NP + degf(i)] : T.CONST3[degf(i)];
    double v;
    if (c < n) {
      const double cc = rH ? (cH ? cst[CST_H2 * NP + degf(kk)] : cst[CST_F2 * NP + degf(kk)])
                           : (cH ? cst[CST_H1 * NP + degf(kk)] : cst[CST_F1 * NP + degf(kk)]);
      v = -rs * m * cc + ((r == c) ? 1.0 : 0.0);
    } else {
      v = (rH == cH) ? rs * m : 0.0;
    }
    W[u] = v;
  }
  __syncthreads();
  for (int c = 0; c < n; c++) {
    // pivot: the largest |W[r][c]| over r >= c, the lowest row on ties
    double best = -1.0;
    int br = c;
    for (int r = c + threadIdx.x; r < n; r += blockDim.x) {
      const double a = fabs(W[(size_t)r * w2 + c]);
      if (a > best) { best = a; br = r; }
    }
    rv[threadIdx.x] = best;
    ri[threadIdx.x] = br;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        const double a = rv[threadIdx.x + o];
        const int b = ri[threadIdx.x + o];
        if (a > rv[threadIdx.x] || (a == rv[threadIdx.x] && b < ri[threadIdx.x])) { rv[threadIdx.x] = a; ri[threadIdx.x] = b; }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) { s_row = ri[0]; s_piv = W[(size_t)ri[0] * w2 + c]; }
    __syncthreads();
    if (!(fabs(s_piv) > 1e-300)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      return;
    }
    const int pr = s_row;
    if (pr != c)
      for (int j = c + threadIdx.x; j < w2; j += blockDim.x) {
        const double t = W[(size_t)c * w2 + j];
        W[(size_t)c * w2 + j] = W[(size_t)pr * w2 + j];
        W[(size_t)pr * w2 + j] = t;
      }
    __syncthreads();
    const double ip = 1.0 / s_piv;
    for (int j = c + threadIdx.x; j < w2; j += blockDim.x) W[(size_t)c * w2 + j] *= ip;
    __syncthreads();
    // eliminate column c from every other row; a warp per row keeps the row's
    // factor in a register while it updates the row
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nwp = blockDim.x >> 5;
    for (int r = wp; r < n; r += nwp) {
      if (r == c) continue;
      const double f = W[(size_t)r * w2 + c];
      if (f == 0.0) continue;
      __syncwarp();
      for (int j = c + lane; j < w2; j += 32) W[(size_t)r * w2 + j] -= f * W[(size_t)c * w2 + j];
    }
    __syncthreads();
  }
  double *G = const_cast<double *>(tv.Gdir) + (size_t)ts * n * n;
  for (long long u = threadIdx.x; u < (long long)n * n; u += blockDim.x) {
    const int r = (int)(u / n), c = (int)(u % n);
    G[u] = W[(size_t)r * w2 + n + c];
  }
}

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ int deg_of(int k)
{
  int d = (int)sqrt((double)k);
  while (d * d > k) d--;
  while ((d + 1) * (d + 1) <= k) d++;
  return d;
}
// W weight of packed entry k (1 for m = 0, 2 for the Re/Im entries of m > 0)
__device__ __forceinline__ double wgt(int k) { const int d = deg_of(k); return (k == d * d) ? 1.0 : 2.0; }

__device__ double team_dot(const Team &tm, const double *a, const double *b, int n, double *red)
{
  double s = 0.0;
  for (int k = tm.rank; k < n; k += tm.size) s += a[k] * b[k];
  return team_sum(tm, s, red);
}

// Generator of a lab-frame rotation about axis c applied to a packed expansion
// (d/de of the rotation by angle e, at e = 0).  Within degree n: about z the
// (Re, Im) pair of order m turns by m; about x and y order m couples to m +- 1 with
// the half ladder coefficients c_m = sqrt((n - m)(n + m + 1)) / 2, the m = 0 entry
// taking 2 c_0 (its weight is 1 against 2 for the others).
__device__ void rot_gen(const Team &tm, int c, const double *v, double *o, int P)
{
  for (int k = tm.rank; k < P * P; k += tm.size) {
    const int n = deg_of(k), b = n * n, mm = k - b;
    if (n == 0) { o[k] = 0.0; continue; }
    auto cm = [&](int m) { return 0.5 * sqrt((double)(n - m) * (n + m + 1)); };
    auto re = [&](int m) { return m == 0 ? b : b + 2 * m - 1; };
    auto im = [&](int m) { return b + 2 * m; };
    double r = 0.0;
    if (mm == 0) {
      r = (c == 0) ? 2 * cm(0) * v[im(1)] : (c == 1) ? -2 * cm(0) * v[re(1)] : 0.0;
    } else {
      const int m = (mm + 1) / 2;
      const bool isre = (mm & 1) != 0;
      if (c == 2) r = isre ? -m * v[im(m)] : m * v[re(m)];
      else if (c == 0) {
        if (isre) { if (m >= 2) r += cm(m - 1) * v[im(m - 1)]; if (m < n) r += cm(m) * v[im(m + 1)]; }
        else { r -= cm(m - 1) * v[re(m - 1)]; if (m < n) r -= cm(m) * v[re(m + 1)]; }
      } else {
        if (isre) { r += cm(m - 1) * v[re(m - 1)]; if (m < n) r -= cm(m) * v[re(m + 1)]; }
        else { if (m >= 2) r += cm(m - 1) * v[im(m - 1)]; if (m < n) r -= cm(m) * v[im(m + 1)]; }
      }
    }
    o[k] = r;
  }
}

// out = W * R(v / W): the transpose of the molecule rotation in direction bFor,
// which is the rotation in the other direction between W and 1/W
__device__ void rot_T(const Team &tm, const RotState &rs, const double *v, double *tmp, double *out, int P, bool bFor)
{
  for (int k = tm.rank; k < P * P; k += tm.size) tmp[k] = v[k] / wgt(k);
  tm.sync();
  rot_apply_xi(tm, rs, tmp, out, P, !bFor, P);
  tm.sync();
  for (int k = tm.rank; k < P * P; k += tm.size) out[k] *= wgt(k);
  tm.sync();
}

// The inner solve transposed: (gfb, ghb) = G^T (gF, gH), then
// dU/dLF = cLF1 gfb + cLF2 ghb and dU/dLH = cLH1 gfb + cLH2 ghb.
__device__ void solve_direct_T(const Team &tm, const Tab &T, const TypeView &tv, const Scr &sc, int ts, const double *gF,
                               const double *gH, double *gLF, double *gLH)
{
  const int NP = T.NP, NP2 = NP * NP, n2 = 2 * NP2;
  const double *cst = tv.cst + (size_t)ts * CST_N * NP;
  const double *G = tv.Gdir + (size_t)ts * n2 * n2;
  double *x = sc.xs, *y = sc.sol;
  for (int k = tm.rank; k < NP2; k += tm.size) { x[k] = gF[k]; x[NP2 + k] = gH[k]; }
  tm.sync();
  {
    const double *Ms[1] = {G}, *xs[1] = {x};
    const int nr[1] = {n2};
    cols_apply<1>(tm, Ms, nr, nr, n2, xs, sc.tile, (int)(dyn_region_bytes(NP) / sizeof(double)),
                  [&](int, int j, double v) { y[j] = v; });
  }
  for (int k = tm.rank; k < NP2; k += tm.size) {
    const int n = deg_of(k);
    gLF[k] = cst[CST_LF1 * NP + n] * y[k] + cst[CST_LF2 * NP + n] * y[NP2 + k];
    gLH[k] = cst[CST_LH1 * NP + n] * y[k] + cst[CST_LH2 * NP + n] * y[NP2 + k];
  }
  tm.sync();
}

// phi[h] = sum_k w_k * (local-expansion basis k of a unit charge at pts[h] - shift),
// the value at each point of the local expansion w about the target (the transpose
// of the charge sum of numeric_expand2 with local = true); P degrees of w are used
__device__ void local_eval(const Team &tm, const Tab &T, const double *pts, int N, const double *shift, double scale,
                           bool kappa, int P, const double *w, double *phi)
{
  double rad[64];
  for (int h = tm.rank; h < N; h += tm.size) {
    const Sph s = cart2sph(pts[3 * h] - shift[0], pts[3 * h + 1] - shift[1], pts[3 * h + 2] - shift[2]);
    radial_factors(T, s.rho, 1.0, true, kappa, P, scale, rad);
    double st, ct;
    sincos(s.theta, &st, &ct);
    double acc = 0.0;
    for (int m = 0; m < P; m++)
      sh_column(T, ct, st, s.phi, m, P, [&](int n, double re, double im) {
        if (m == 0) acc += rad[n] * w[IDX(n)] * re;
        else acc += rad[n] * (w[IDX(n) + 2 * m - 1] * re + w[IDX(n) + 2 * m] * im);
      });
    phi[h] = acc;
  }
  tm.sync();
}

// pose terms of one inter-molecular re-expansion target kt <- source ks: dU/dP = gP
// with P = c_tgt - c_src moves the two molecules' positions and turns their sphere
// centres (c = pos + R cen)
__device__ void add_pose_grad(const Team &tm, const Sys &y, int kt, int ks, const double *gP)
{
  if (tm.rank != 0) return;
  const BatchView &bv = y.c->bv;
  const int it = y.mol(kt), is = y.mol(ks);
  double *dp = bv.dpos + (size_t)y.b * bv.nmol * 3, *dr = bv.drot + (size_t)y.b * bv.nmol * 3;
  const double *ct = y.cenRot(kt), *cs = y.cenRot(ks);
  for (int d = 0; d < 3; d++) { dp[3 * it + d] += gP[d]; dp[3 * is + d] -= gP[d]; }
  dr[3 * it + 0] += ct[1] * gP[2] - ct[2] * gP[1];
  dr[3 * it + 1] += ct[2] * gP[0] - ct[0] * gP[2];
  dr[3 * it + 2] += ct[0] * gP[1] - ct[1] * gP[0];
  dr[3 * is + 0] -= cs[1] * gP[2] - cs[2] * gP[1];
  dr[3 * is + 1] -= cs[2] * gP[0] - cs[0] * gP[2];
  dr[3 * is + 2] -= cs[0] * gP[1] - cs[1] * gP[0];
}
// dU/domega_i += sign * <g, J_c v> for c = x, y, z
__device__ void add_rot_grad(const Team &tm, const Sys &y, int i, const double *g, const double *v, double sign,
                             double *tmp)
{
  const int NP2 = y.NP2;
  double d[3];
  for (int c = 0; c < 3; c++) {
    rot_gen(tm, c, v, tmp, y.NP);
    tm.sync();
    d[c] = team_dot(tm, g, tmp, NP2, y.red);
  }
  if (tm.rank == 0) {
    double *dr = y.c->bv.drot + ((size_t)y.b * y.c->bv.nmol + i) * 3;
    for (int c = 0; c < 3; c++) dr[c] += sign * d[c];
  }
  tm.sync();
}

// One inter-molecular re-expansion target kt <- source ks at order p (screened),
// transposed: gsrc += T^T g = W T(ks <- kt)(g / W), with its pose terms
// <g, dT/dP v>, v the source expansion of the forward; fwd (optional) receives T v.
__device__ void pair_adjoint(const Team &tm, const Sys &y, int kt, int ks, int p, const double *v, const double *g,
                             double *gsrc, double *fwd = nullptr)
{
  const Tab &T = y.c->T;
  const Scr &sc = y.sc;
  const int NP2 = y.NP2;
  double ct[3], cs[3];
  y.cen_lab(kt, ct);
  y.cen_lab(ks, cs);
  double P[3] = {ct[0] - cs[0], ct[1] - cs[1], ct[2] - cs[2]};
  min_image(y.c->prm.box, P);
  const double Pm[3] = {-P[0], -P[1], -P[2]};
  PairXf X;
  prep_pair(tm, T, sc, P, p, 0, y.rad(ks), y.rad(kt), true, X);
  if (fwd) pair_apply(tm, T, sc, X, false, v, fwd);
  double *G = sc.G(1);
  pair_apply_grad(tm, T, sc, X, v, G);
  double gP[3];
  for (int c = 0; c < 3; c++) gP[c] = team_dot(tm, g, G + (size_t)c * NP2, NP2, y.red);
  add_pose_grad(tm, y, kt, ks, gP);
  double *gw = sc.E(12), *o = sc.E(13);
  for (int k = tm.rank; k < NP2; k += tm.size) gw[k] = g[k] / wgt(k);
  tm.sync();
  prep_pair(tm, T, sc, Pm, p, 0, y.rad(kt), y.rad(ks), false, X);
  pair_apply(tm, T, sc, X, false, gw, o);
  for (int k = tm.rank; k < NP2; k += tm.size) gsrc[k] += wgt(k) * o[k];
  tm.sync();
}

__device__ __forceinline__ double warp_dot(const WarpTeam &tw, const double *a, const double *b, int n)
{
  double s = 0.0;
  for (int k = tw.rank; k < n; k += tw.size) s += a[k] * b[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// One pair (si <- sj) of the energy adjoint transformed by a single warp with its own
// scratch ws (pair_adjoint's arithmetic): part += a . T Hlab_sj (this warp's share of
// dU/dHlab_si), gHl_sj += W T(sj <- si)(wi / W), and the pose terms <wi, dT/dP Hlab_sj>
// summed on lane 0 into pose[9]: d/dpos_i (3), d/domega_i (3), d/domega_j (3).
__device__ __noinline__ void energy_pair_warp(const WarpTeam &tw, const Sys &y, const Scr &ws, int si, int sj, int p,
                                              const double *Hj, const double *wi, const double *a, double *gHj,
                                              double *part, double *pose)
{
  const Tab &T = y.c->T;
  const int NP2 = y.NP2;
  double ct[3], cs[3];
  y.cen_lab(si, ct);
  y.cen_lab(sj, cs);
  double P[3] = {ct[0] - cs[0], ct[1] - cs[1], ct[2] - cs[2]};
  min_image(y.c->prm.box, P);
  const double Pm[3] = {-P[0], -P[1], -P[2]};
  PairXf X;
  prep_pair(tw, T, ws, P, p, 0, y.rad(sj), y.rad(si), true, X);
  double *fwd = ws.misc + NP2, *gw = ws.misc + 2 * NP2;
  pair_apply(tw, T, ws, X, false, Hj, fwd);
  double *G = ws.G(0);
  pair_apply_grad(tw, T, ws, X, Hj, G);
  double gP[3];
  for (int c = 0; c < 3; c++) gP[c] = warp_dot(tw, wi, G + (size_t)c * NP2, NP2);
  if (tw.rank == 0) {
    const double *rt = y.cenRot(si), *rs = y.cenRot(sj);
    for (int d = 0; d < 3; d++) pose[d] += gP[d];
    pose[3] += rt[1] * gP[2] - rt[2] * gP[1];
    pose[4] += rt[2] * gP[0] - rt[0] * gP[2];
    pose[5] += rt[0] * gP[1] - rt[1] * gP[0];
    pose[6] -= rs[1] * gP[2] - rs[2] * gP[1];
    pose[7] -= rs[2] * gP[0] - rs[0] * gP[2];
    pose[8] -= rs[0] * gP[1] - rs[1] * gP[0];
  }
  for (int k = tw.rank; k < NP2; k += tw.size) {
    part[k] += a[k] * fwd[k];
    gw[k] = wi[k] / wgt(k);
  }
  tw.sync();
  prep_pair(tw, T, ws, Pm, p, 0, y.rad(si), y.rad(sj), false, X);
  double *o = ws.G(0);
  pair_apply(tw, T, ws, X, false, gw, o);
  for (int k = tw.rank; k < NP2; k += tw.size) gHj[k] += wgt(k) * o[k];
  tw.sync();
}

// molecule rotation state of molecule i (the forward prepares it only for molecules
// with inter-molecular work; the energy needs every molecule)
__device__ RotState mol_rot(const Team &tm, const Sys &y, int i)
{
  const BatchView &bv = y.c->bv;
  if (!bv.interX[(size_t)y.b * bv.nmol + i]) {
    const double *q = bv.quat + 4 * ((size_t)y.b * bv.nmol + i);
    double qn[4];
    const double in = 1.0 / sqrt((q[1] * q[1] + q[2] * q[2] + q[3] * q[3]) + q[0] * q[0]);
    qn[0] = q[0] * in; qn[1] = q[1] * in; qn[2] = q[2] * in; qn[3] = q[3] * in;
    double th, ph, xi;
    quat_angles(qn, th, ph, xi);
    RotState rs;
    double2 *Rm = bv.molR + ((size_t)y.b * bv.nmol + i) * rot_off(2 * y.NP - 1);
    rot_compute(tm, y.c->T, th, ph, xi, y.NP, false, rs, Rm, nullptr, y.sc.sh, y.sc.lvA, y.sc.lvB);
    if (tm.rank == 0) {
      double *v = bv.molRS + ((size_t)y.b * bv.nmol + i) * 16;
      v[0] = rs.sing ? 1.0 : 0.0; v[1] = rs.cost; v[2] = rs.sint; v[3] = rs.cott; v[4] = rs.xi;
      v[5] = rs.exphi.x; v[6] = rs.exphi.y; v[7] = rs.exxi.x; v[8] = rs.exxi.y;
    }
    tm.sync();
  }
  return y.molrot(i);
}

// entry of type sphere kv (index within the type) in the near list of type sphere tsu, or -1
__device__ __forceinline__ int near_entry(const TypeView &tv, int tsu, int kv)
{
  for (int e = tv.near_off[tsu]; e < tv.near_off[tsu + 1]; e++)
    if (tv.near[e] == kv) return e;
  return -1;
}

__device__ __forceinline__ bool polarized(const Sys &y, int s)
{
  return y.c->bv.interX[(size_t)y.b * y.c->bv.nmol + y.mol(s)] && y.nipol(s) > 0;
}

// The backward pass of one system (a crew of one CTA) on the converged exact-form
// state: dU/dpos and dU/domega (lab frame) of the lab-frame energy into bv.dpos /
// bv.drot.  Returns false if the transposed sweeps hit max_pol_rounds.
__device__ __noinline__ bool backward_body(const Team &tm, const Sys &y)
{
  const Ctx &c = *y.c;
  const BatchView &bv = c.bv;
  const Tab &T = c.T;
  const Scr &sc = y.sc;
  const int S = bv.S, nmol = bv.nmol, NP = y.NP, NP2 = y.NP2, b = y.b;
  // adjoint state in the gradient work set (the exact form has no gradient phase)
  auto slot = [&](double *base, int s, int k) { return base + ((size_t)b * S + s) * 3 * NP2 + (size_t)k * NP2; };
  auto lamF = [&](int s) { return slot(bv.gFw, s, 0); };
  auto lamH = [&](int s) { return slot(bv.gFw, s, 1); };
  auto muF = [&](int s) { return slot(bv.gFw, s, 2); };
  auto muH = [&](int s) { return slot(bv.gHw, s, 0); };
  auto gHl = [&](int s) { return slot(bv.gHw, s, 1); };
  auto gHrot = [&](int s) { return slot(bv.gHw, s, 2); };
  auto gHsr = [&](int s) { return slot(bv.gHrotw, s, 0); };
  auto Hlab = [&](int s) { return bv.Hlab + ((size_t)b * S + s) * NP2; };
  double *t0 = sc.E(3), *t1 = sc.E(4), *t2 = sc.E(5), *t3 = sc.E(6), *t4 = sc.E(7), *t5 = sc.E(8), *t6 = sc.E(9);
  for (int t = tm.rank; t < nmol * 3; t += tm.size) {
    bv.dpos[(size_t)b * nmol * 3 + t] = 0.0;
    bv.drot[(size_t)b * nmol * 3 + t] = 0.0;
  }
  for (int s = 0; s < S; s++) {
    tzero(tm, gHl(s), NP2); tzero(tm, gHrot(s), NP2); tzero(tm, gHsr(s), NP2);
  }
  tm.sync();
  // ---- lab-frame H of every sphere
  for (int i = 0; i < nmol; i++) {
    const RotState mr = mol_rot(tm, y, i);
    for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
      rot_apply_xi(tm, mr, y.H(s), Hlab(s), NP, true, NP);
      tm.sync();
    }
  }
  // ---- the energy: U = sum_{i<j} sum_{si, sj} <a_si . Hlab_si, T(si <- sj) Hlab_sj>
  // At pole orders up to PBSAM_WARP_MAX_NP the pairs of order <= PBSAM_WARP_P are
  // dealt round-robin to the CTA's warps, each transforming its pairs alone (a pair
  // at p = 10 is too narrow to keep 512 threads busy); their shares of dU/dHlab_si
  // and of the pose terms are added in warp order.  The other pairs are transformed
  // one by one by the whole CTA.
  PhaseClock pe{y.tph, 0};
  pe.start(tm);
  const bool warps = NP <= PBSAM_WARP_MAX_NP;
  const int lane = tm.rank & 31, w = tm.rank >> 5, nw = tm.size >> 5;
  const WarpTeam tw{lane, 32};
  const Scr ws = warps ? warp_scr(wscr_of(bv, b, 0, w), NP) : sc;
  auto pair_order_E = [&](int si, int sj) {
    double ci[3], cj[3];
    y.cen_lab(si, ci);
    y.cen_lab(sj, cj);
    double dd[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
    min_image(c.prm.box, dd);
    const double rho = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
    const int pi2j = compute_order(NP, rho, bv.tH[y.sc1(si)], y.rad(si));
    const int pj2i = compute_order(NP, rho, bv.tH[y.sc1(sj)], y.rad(sj));
    return pi2j < pj2i ? pi2j : pj2i;
  };
  for (int i = 0; i < nmol; i++)
    for (int j = i + 1; j < nmol; j++) {
      double pose[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // this warp's pose terms (lane 0)
      for (int si = bv.mol_off[i]; si < bv.mol_off[i + 1]; si++) {
        const double fact = 1.0 / (bv.hscale[y.sc1(si)] * y.rad(si));
        double *a = t0, *wi = t1;
        for (int k = tm.rank; k < NP2; k += tm.size) {
          a[k] = wgt(k) * pow(fact, (double)deg_of(k));
          wi[k] = a[k] * Hlab(si)[k];
        }
        tm.sync();
        if (warps) {
          double *part = ws.misc;
          tzero(tw, part, NP2);
          tw.sync();
          int q = 0;
          for (int sj = bv.mol_off[j]; sj < bv.mol_off[j + 1]; sj++) {
            const int p = pair_order_E(si, sj);
            if (p > PBSAM_WARP_P) continue;
            if ((q++ % nw) != w) continue;
            energy_pair_warp(tw, y, ws, si, sj, p, Hlab(sj), wi, a, gHl(sj), part, pose);
          }
          tm.sync();
          const size_t moff = (size_t)(warp_scr(wscr_of(bv, b, 0, 0), NP).misc - wscr_of(bv, b, 0, 0));
          for (int k = tm.rank; k < NP2; k += tm.size) {
            double v = 0.0;
            for (int u = 0; u < nw; u++) v += wscr_of(bv, b, 0, u)[moff + k];
            gHl(si)[k] += v;
          }
          tm.sync();
        }
        for (int sj = bv.mol_off[j]; sj < bv.mol_off[j + 1]; sj++) {
          const int p = pair_order_E(si, sj);
          if (warps && p <= PBSAM_WARP_P) continue;
          pair_adjoint(tm, y, si, sj, p, Hlab(sj), wi, gHl(sj), t2);
          for (int k = tm.rank; k < NP2; k += tm.size) gHl(si)[k] += a[k] * t2[k];
          tm.sync();
        }
      }
      if (warps) {
        // the warps' pose terms in warp order
        double *dp = bv.dpos + (size_t)b * nmol * 3, *dr = bv.drot + (size_t)b * nmol * 3;
        for (int u = 0; u < nw; u++) {
          if (w == u && lane == 0)
            for (int d = 0; d < 3; d++) {
              dp[3 * i + d] += pose[d];
              dp[3 * j + d] -= pose[d];
              dr[3 * i + d] += pose[3 + d];
              dr[3 * j + d] += pose[6 + d];
            }
          tm.sync();
        }
      }
    }
  pe.stop(tm, PH_GX_INTER);
  // ---- Hlab = RF H: rotation terms, then dU/dH in the molecule frame
  for (int i = 0; i < nmol; i++) {
    const RotState mr = y.molrot(i);
    for (int s = bv.mol_off[i]; s < bv.mol_off[i + 1]; s++) {
      add_rot_grad(tm, y, i, gHl(s), Hlab(s), 1.0, t2);
      rot_T(tm, mr, gHl(s), t2, t3, NP, true);
      tcopy(tm, gHl(s), t3, NP2);
      tm.sync();
    }
  }
  // ---- the intra-molecular fixed point, transposed: lambda_v = g_v + sum_u A_uv^T mu_u,
  // mu_u = dU/d(LF_u, LH_u) = (direct solve)^T lambda_u; swept in reverse sphere order
  for (int s = 0; s < S; s++) {
    if (!polarized(y, s)) continue;
    tzero(tm, lamF(s), NP2);
    tcopy(tm, lamH(s), gHl(s), NP2);
    tm.sync();
    solve_direct_T(tm, T, c.tv, sc, y.ts(s), lamF(s), lamH(s), muF(s), muH(s));
  }
  PhaseClock pt{y.tph, 0};
  pt.start(tm);
  const double tol2 = c.prm.exact_tol * c.prm.exact_tol;
  bool conv = false;
  for (int sweep = 0; sweep < c.prm.max_pol_rounds && !conv; sweep++) {
    double dn = 0.0, nn = 0.0;
    for (int v = S - 1; v >= 0; v--) {
      if (!polarized(y, v)) continue;
      const int i = y.mol(v), mo = bv.mol_off[i], tsv = y.ts(v);
      double *nF = t2, *nH = t3;
      tzero(tm, nF, NP2);
      tcopy(tm, nH, gHl(v), NP2);
      tm.sync();
      for (int e = c.tv.near_off[tsv]; e < c.tv.near_off[tsv + 1]; e++) {
        const int u = mo + c.tv.near[e];
        if (!polarized(y, u)) continue;
        // the forward map v -> u (reexpand_intra_near of target u over its neighbour v)
        const double *cu = y.cen(u), *cv = y.cen(v);
        const double P[3] = {cu[0] - cv[0], cu[1] - cv[1], cu[2] - cv[2]};
        const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
        const double sep = rho - y.rad(u) - y.rad(v);
        const int pF = compute_order(NP, rho, bv.tF[y.sc1(v)], y.rad(v));
        const int pH = compute_order(NP, rho, bv.tH[y.sc1(v)], y.rad(v));
        double *oF = t6, *oH = sc.E(10);
        const bool analytic = sep > 0 && !(sep < c.prm.min_sep_numeric);
        const int ent = c.tv.nslot ? near_entry(c.tv, y.ts(u), v - mo) : -1;
        const int slot = ent >= 0 ? c.tv.nslot[ent] : -1;
        if (slot >= 0 && c.tv.nkind[slot] == (analytic ? 0 : 1)) {
          // the precomputed operators of the forward map v -> u, transposed
          const double *NF = c.tv.Nmat + (size_t)slot * 2 * NP2 * NP2;
          num_apply2_T(tm, NF, NF + (size_t)NP2 * NP2, pF, pH, analytic ? pF : NP, analytic ? pH : NP, muF(u),
                       muH(u), nF, nH, NP2, sc.tile, (int)(dyn_region_bytes(NP) / sizeof(double)));
        } else if (analytic) {
          // analytic: T(u <- v)^T = W T(v <- u) W^-1, from the intra table of target v
          double *wF = t4, *wH = t5;
          for (int k = tm.rank; k < NP2; k += tm.size) { wF[k] = muF(u)[k] / wgt(k); wH[k] = muH(u)[k] / wgt(k); }
          tm.sync();
          PairXf X;
          table_pair(tm, T, c.tv, sc, intra_pair(c.tv, tsv, v - mo, u - mo), pH, pF, y.rad(u), y.rad(v), X);
          MultiVec V;
          V.n = 2;
          V.in[0] = wF; V.out[0] = oF; V.useF[0] = true;
          V.in[1] = wH; V.out[1] = oH; V.useF[1] = false;
          pair_apply_multi(tm, T, sc, X, V, false);
          for (int k = tm.rank; k < NP2; k += tm.size) { nF[k] += wgt(k) * oF[k]; nH[k] += wgt(k) * oH[k]; }
          tm.sync();
        } else {
          // numeric: the expansion at u of v's surface charges q = dA W c_n E . Y
          // (surface_q2) summed over v's points (numeric_expand2, local); transposed:
          // mu_u evaluated at the points, projected on v's harmonics, scaled by dA W c_n
          const double dA = 4 * PB_PI / double(c.tv.nspx[tsv]);
          const double zero[3] = {0.0, 0.0, 0.0};
          const double *cstv = c.tv.cst + (size_t)tsv * CST_N * NP;
          double *phiF = y.gFp(v), *phiH = y.gHp(v);   // per-point work (no gradient charges here)
          local_eval(tm, T, y.spx(v), y.npts(v), P, y.rad(u), false, pF, muF(u), phiF);
          local_eval(tm, T, y.spx(v), y.npts(v), P, y.rad(u), true, pH, muH(u), phiH);
          numeric_expand2<1>(tm, T, sc, y.spx(v), y.npts(v), zero, y.rad(v), NumSet{phiF, false, false, NP, oF},
                             NumSet{phiH, false, false, NP, oH});
          tm.sync();
          for (int k = tm.rank; k < NP2; k += tm.size) {
            const int n = deg_of(k);
            nF[k] += dA * wgt(k) * T.CONST2[n] * oF[k];
            nH[k] += dA * wgt(k) * cstv[CST_CHGH * NP + n] * oH[k];
          }
          tm.sync();
        }
      }
      double ld = 0.0, ln = 0.0;
      for (int k = tm.rank; k < NP2; k += tm.size) {
        const double a = nF[k] - lamF(v)[k], bb = nH[k] - lamH(v)[k];
        ld += a * a + bb * bb;
        ln += nF[k] * nF[k] + nH[k] * nH[k];
      }
      double sd, sn;
      team_sum2(tm, ld, ln, y.red, sd, sn);
      dn += sd;
      nn += sn;
      const double om = c.prm.exact_relax;   // over-relaxed as the forward sweeps
      for (int k = tm.rank; k < NP2; k += tm.size) {
        lamF(v)[k] += om * (nF[k] - lamF(v)[k]);
        lamH(v)[k] += om * (nH[k] - lamH(v)[k]);
      }
      tm.sync();
      solve_direct_T(tm, T, c.tv, sc, tsv, lamF(v), lamH(v), muF(v), muH(v));
    }
    conv = !(dn > tol2 * nn);
  }
  pt.stop(tm, PH_GX_ANALYTIC);
  PhaseClock ps{y.tph, 0};
  ps.start(tm);
  // ---- stage 2: LS = RB(sum over interPol neighbours T(u <- s2) Hrot_s2)
  for (int u = 0; u < S; u++) {
    if (!polarized(y, u)) continue;
    const int i = y.mol(u);
    const RotState mr = y.molrot(i);
    double *LSrot = t2, *gLSrot = t3;
    rot_apply_xi(tm, mr, y.LS(u), LSrot, NP, true, NP);     // RB^-1 LS
    tm.sync();
    rot_T(tm, mr, muH(u), t4, gLSrot, NP, false);            // RB^T mu_H
    add_rot_grad(tm, y, i, gLSrot, LSrot, -1.0, t4);
    const int *lst = y.ipol(u);
    for (int e = 0; e < y.nipol(u); e++) {
      const int s2 = lst[e];
      double cu[3], c2[3];
      y.cen_lab(u, cu);
      y.cen_lab(s2, c2);
      double dd[3] = {cu[0] - c2[0], cu[1] - c2[1], cu[2] - c2[2]};
      min_image(c.prm.box, dd);
      const double rho = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
      const int p = compute_order(NP, rho, bv.tH[y.sc1(s2)], y.rad(s2));
      pair_adjoint(tm, y, u, s2, p, y.Hrot(s2), gLSrot, gHrot(s2));
    }
  }
  // ---- stage 1: Hrot = RF H1, H1 solved from LS1 = RB(sum T(u <- s2) HselfRot_s2)
  for (int u = 0; u < S; u++) {
    if (!polarized(y, u)) continue;
    const int i = y.mol(u);
    const RotState mr = y.molrot(i);
    add_rot_grad(tm, y, i, gHrot(u), y.Hrot(u), 1.0, t2);
    double *gH1 = t3, *zF = t4, *g1F = t5, *g1H = t6;
    rot_T(tm, mr, gHrot(u), t2, gH1, NP, true);
    tzero(tm, zF, NP2);
    tm.sync();
    solve_direct_T(tm, T, c.tv, sc, y.ts(u), zF, gH1, g1F, g1H);
    // the first-round LS, recomputed (the later rounds overwrote it)
    double *LSrot1 = sc.E(10), *tL = sc.E(11);
    tzero(tm, LSrot1, NP2);
    tm.sync();
    const int *lst = y.ipol(u);
    for (int e = 0; e < y.nipol(u); e++) {
      const int s2 = lst[e];
      double cu[3], c2[3];
      y.cen_lab(u, cu);
      y.cen_lab(s2, c2);
      double P[3] = {cu[0] - c2[0], cu[1] - c2[1], cu[2] - c2[2]};
      min_image(c.prm.box, P);
      const double rho = sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]);
      const int p = compute_order(NP, rho, c.tv.tHself[y.ts(s2)], y.rad(s2));
      PairXf X;
      prep_pair(tm, T, sc, P, p, 0, y.rad(s2), y.rad(u), false, X);
      pair_apply(tm, T, sc, X, false, y.HselfRot(s2), tL);
      add_vec_into(tm, LSrot1, tL, NP2);
    }
    double *gLSrot1 = t2;
    rot_T(tm, mr, g1H, t4, gLSrot1, NP, false);
    add_rot_grad(tm, y, i, gLSrot1, LSrot1, -1.0, t4);
    for (int e = 0; e < y.nipol(u); e++) {
      const int s2 = lst[e];
      double cu[3], c2[3];
      y.cen_lab(u, cu);
      y.cen_lab(s2, c2);
      double dd[3] = {cu[0] - c2[0], cu[1] - c2[1], cu[2] - c2[2]};
      min_image(c.prm.box, dd);
      const double rho = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
      const int p = compute_order(NP, rho, c.tv.tHself[y.ts(s2)], y.rad(s2));
      pair_adjoint(tm, y, u, s2, p, y.HselfRot(s2), gLSrot1, gHsr(s2));
    }
  }
  // ---- HselfRot = RF Hself
  for (int s = 0; s < S; s++) {
    const int i = y.mol(s);
    if (!bv.interX[(size_t)b * nmol + i] || (y.nipol(s) == 0 && y.niact(s) == 0)) continue;
    add_rot_grad(tm, y, i, gHsr(s), y.HselfRot(s), 1.0, t2);
  }
  ps.stop(tm, PH_GX_NUMERIC);
  return conv;
}

// dL/dpos, dL/dquat and dL/domega from the stored dU/dpos, dU/domega and a per-system
// seed dL/dU: dU/dq = 2 (0, dU/domega) q for the unit quaternion q (the derivative
// along q' = (1, omega/2) q, tangent to the unit sphere).
__global__ void pbsam_backward_out_kernel(BatchView bv, const double *seed, double *dpos, double *dquat,
                                          double *drot)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= bv.B * bv.nmol) return;
  const int b = t / bv.nmol;
  const double sd = seed ? seed[b] : 1.0;
  const double *p = bv.dpos + 3 * (size_t)t, *r = bv.drot + 3 * (size_t)t;
  if (dpos) for (int d = 0; d < 3; d++) dpos[3 * (size_t)t + d] = sd * p[d];
  if (drot) for (int d = 0; d < 3; d++) drot[3 * (size_t)t + d] = sd * r[d];
  if (dquat) {
    const double *q = bv.quat + 4 * (size_t)t;
    const double in = 1.0 / sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    const double w = q[0] * in, x = q[1] * in, y = q[2] * in, z = q[3] * in;
    const double gx = 2 * sd * r[0], gy = 2 * sd * r[1], gz = 2 * sd * r[2];
    // (0, g) * q, Hamilton product
    dquat[4 * (size_t)t + 0] = -(gx * x + gy * y + gz * z);
    dquat[4 * (size_t)t + 1] = gx * w + gy * z - gz * y;
    dquat[4 * (size_t)t + 2] = gy * w + gz * x - gx * z;
    dquat[4 * (size_t)t + 3] = gz * w + gx * y - gy * x;
  }
}

}  // namespace pbsam
