// Molecule-type preparation on the GPU: the surface-integral matrices (IMat,
// the reference's `pbsam mat`) and self-polarization (`pbsam spol`).
// Included by pbsam_api.cu after pbsam_kernels.cu.
namespace pbsam {

// ------------------------------------------------------------------ IMat
// Yt[c * K + h] = real spherical-harmonic component c (packed layout, P degrees)
// at quadrature point h (points relative to the sphere centre).
__global__ void imat_sh_kernel(Tab T, const double *pts, int K, int P, double *Yt)
{
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= K) return;
  const Sph s = cart2sph(pts[3 * h], pts[3 * h + 1], pts[3 * h + 2]);
  double st, ct;
  sincos(s.theta, &st, &ct);
  for (int m = 0; m < P; m++) {
    sh_column(T, ct, st, s.phi, m, P, [&](int n, double re, double im) {
      if (m == 0) Yt[(size_t)IDX(n) * K + h] = re;
      else {
        Yt[(size_t)(IDX(n) + 2 * m - 1) * K + h] = re;
        Yt[(size_t)(IDX(n) + 2 * m) * K + h] = im;
      }
    });
  }
}

// G[i][j] += sum_h Yt[i][h] Yt[j][h]  (N x N, 64 x 64 tiles, 4 x 4 per thread)
#define GT 64
#define GK 16
__global__ void __launch_bounds__(256) gram_kernel(const double *Yt, int K, int N, double *G)
{
  __shared__ double A[GK][GT + 1], B[GK][GT + 1];
  const int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4];
  for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
  for (int k0 = 0; k0 < K; k0 += GK) {
    for (int u = threadIdx.x; u < GT * GK; u += blockDim.x) {
      const int r = u / GK, kk = u % GK;
      const int gi = i0 + r, gj = j0 + r, gk = k0 + kk;
      A[kk][r] = (gi < N && gk < K) ? Yt[(size_t)gi * K + gk] : 0.0;
      B[kk][r] = (gj < N && gk < K) ? Yt[(size_t)gj * K + gk] : 0.0;
    }
    __syncthreads();
    for (int kk = 0; kk < GK; kk++) {
      double a[4], b[4];
      for (int q = 0; q < 4; q++) { a[q] = A[kk][ty + 16 * q]; b[q] = B[kk][tx + 16 * q]; }
      for (int p = 0; p < 4; p++) for (int q = 0; q < 4; q++) acc[p][q] += a[p] * b[q];
    }
    __syncthreads();
  }
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) {
      const int gi = i0 + ty + 16 * p, gj = j0 + tx + 16 * q;
      if (gi < N && gj < N) G[(size_t)gi * N + gj] += acc[p][q];
    }
}

// Simpson-weighted Gram of the m = 0 components (src/expcenter.cpp:715-724):
// weight 1/3 at the first point of the list, then 2/3 (even index) or 4/3 (odd).
__global__ void gram_simpson_kernel(const double *Yt, int K, int P, long long h0, double *Gs)
{
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= P * P) return;
  const int n = u / P, l = u % P;
  const double *yn = Yt + (size_t)IDX(n) * K, *yl = Yt + (size_t)IDX(l) * K;
  double s = 0.0;
  for (int h = 0; h < K; h++) {
    const long long hh = h0 + h;
    const double w = (hh > 0) ? ((hh % 2 == 0) ? 2.0 / 3.0 : 4.0 / 3.0) : 1.0 / 3.0;
    s += w * yn[h] * yl[h];
  }
  Gs[u] += s;
}

// IMat (P^2 x P^2, column-major) from the Gram (build_IMatE, src/expcenter.cpp:910-1033,
// with computeIntegralE / computeIntegralB scaling, src/expcenter.cpp:738-773, 858-899)
__global__ void imat_assemble_kernel(Tab T, const double *G, const double *Gs, int P, double dA, int buried,
                                     double *IM)
{
  const int N = P * P;
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= (long long)N * N) return;
  const int col = (int)(u / N), row = (int)(u % N);
  int n = (int)sqrt((double)row);
  while (n * n > row) n--;
  while ((n + 1) * (n + 1) <= row) n++;
  int l = (int)sqrt((double)col);
  while (l * l > col) l--;
  while ((l + 1) * (l + 1) <= col) l++;
  const int mr = row - n * n, mc = col - l * l;
  const int m = (mr + 1) / 2, s = (mc + 1) / 2;
  const bool rim = (mr > 0 && mr % 2 == 0), cim = (mc > 0 && mc % 2 == 0);
  double v = G[(size_t)row * N + col];
  if (m == 0 && s == 0 && (n + l) % 2 == 0) v = Gs[n * P + l];
  double y;
  if (!buried) y = v * dA;
  else if (n == l && m == s) {
    const double delta = 1.0 / T.CONST2[l];
    if (rim == cim) y = ((m == 0) ? delta : 0.5 * delta) - dA * v;
    else y = v * (-dA);
  } else y = v * (-dA);
  const double c = (s == 0) ? 1.0 : 2.0;
  IM[u] = (c * T.CONST2[n]) * y;
}

// ------------------------------------------------------------------ self-polarization
// polarize_self (src/molecule.cpp:1898-1979) for a system of one molecule, starting
// from F = 0 and H = the multipole expansion of the charges assigned to each
// sphere (src/expcenter.cpp:88-103, 541-545, 576-587).
__device__ void selfpol_body(const Team &tm, const Ctx &c, const Crew &cw, int b, void *dsm, double *red,
                             const double *Eass, int max_rounds, int *rounds_out)
{
  const BatchView &bv = c.bv;
  Sys y;
  y.c = &c; y.b = b; y.NP = c.T.NP; y.NP2 = y.NP * y.NP; y.S = bv.S;
  y.cw = cw;
  y.sc = make_scr(scr_of(bv, b, 0), y.NP, dsm);
  y.red = red;
  y.tph = bv.tphase + (size_t)b * PH_N;
  const Tab &T = c.T;
  const int S = bv.S, NP2 = y.NP2;
  if (tm.rank == 0) for (int k = 0; k < PH_N; k++) y.tph[k] = 0.0;
  int *st = y.stats();
  if (tm.rank == 0) for (int k = 0; k < 8; k++) st[k] = 0;
  for (int s = 0; s < S; s++) {
    const int ts = y.ts(s);
    for (int i = tm.rank; i < NP2; i += tm.size) {
      y.H(s)[i] = Eass[(size_t)ts * NP2 + i];
      y.F(s)[i] = 0.0;
      y.LS(s)[i] = 0.0;
    }
    for (int i = tm.rank; i < y.npts(s); i += tm.size) y.qF(s)[i] = 0.0;
    tm.sync();
    const double *cst = c.tv.cst + (size_t)ts * CST_N * y.NP;
    const double dA = 4 * PB_PI / double(c.tv.nspx[ts]);
    double tot[1];
    crew_surface_q2<1>(tm, y.cw, T, y.sc, y.red, y.spx(s), y.npts(s), dA, y.H(s), cst + CST_CHGH * y.NP, y.qH(s), tot,
                       nullptr, nullptr, nullptr, nullptr);
    if (tm.rank == 0) { bv.tH[y.sc1(s)] = tot[0]; bv.tF[y.sc1(s)] = 0.0; bv.dev[y.sc1(s)] = 0.0; }
    tm.sync();
  }
  const double tol2 = c.prm.max_polar_dev * c.prm.max_polar_dev;
  double maxdev = 0.0;
  for (int s = 0; s < S; s++) {
    reexpand_intra_near(tm, y, s);
    const double d = solve_surface(tm, y, s, false);
    if (maxdev < d) maxdev = d;
  }
  int ct = 1;
  while (maxdev > tol2 && ct < max_rounds) {
    double mn = 0.0;
    for (int s = 0; s < S; s++) {
      double d = bv.dev[y.sc1(s)];
      if (d > 0.1 * maxdev || ct % 5 == 0) {
        reexpand_intra_near(tm, y, s);
        d = solve_surface(tm, y, s, false);
      }
      if (mn < d) mn = d;
    }
    maxdev = mn;
    ct++;
  }
  if (tm.rank == 0) rounds_out[b] = ct;
}

// Grid: one crew of cluster-size CTAs per system (a plain launch is a crew of one).
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_selfpol_kernel(Ctx c, const double *Eass, int max_rounds,
                                                                  int *rounds_out)
{
  extern __shared__ double2 dsm[];
  __shared__ double red[PBSAM_TEAM];
  __shared__ CrewCmd cmd;
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  cg::cluster_group cl = cg::this_cluster();
  const Crew cw{(int)cl.block_rank(), (int)cl.num_blocks(), &cmd};
  const int b = blockIdx.x / cw.size;
  if (b >= c.bv.B) return;
  if (cw.rank != 0) {
    crew_serve(tm, helper_sys(c, cw, b, dsm, red));
    return;
  }
  selfpol_body(tm, c, cw, b, dsm, red, Eass, max_rounds, rounds_out);
  crew_finish(tm, cw);
}

}  // namespace pbsam
