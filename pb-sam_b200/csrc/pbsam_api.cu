// Host side of the C ABI (include/pbsam_b200.h): constant tables, input file
// readers, exposed-surface-point generation, device storage of molecule types
// and systems, and kernel launches.  Single translation unit with the kernels.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <algorithm>
#include <utility>
#include <vector>

#include "pbsam_b200.h"
#include "pbsam_kernels.cu"
#include "pbsam_setup.cu"
#include "pbsam_bd.cu"
#include "pbsam_adjoint.cu"

using namespace pbsam;

static thread_local std::string g_err;
static int fail(int code, const std::string &msg) { g_err = msg; return code; }
#define CK(x)                                                                                  \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess) return fail(PBSAM_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

extern "C" const char *pbsam_last_error(void) { return g_err.c_str(); }

// ------------------------------------------------------------------ host tables
// The formulas of src/expansion.cpp:39-96, src/rotcoeff.cpp:15-33, 949-983,
// src/transcoeff.cpp:15-38, src/expcenter.cpp:186-210; zeta has 2NP columns
// (the reference's table writes one column past its declared width).
struct HostTab {
  int NP;
  double kappa;
  std::vector<double> buf;
  size_t oC1, oC2, oC3, oC4, oC6, oZ, oE, oA, oB, oG, oD, oQ, oK2, oK3;
  void build(int np, double kap)
  {
    NP = np; kappa = kap;
    const int N2 = 2 * NP;
    size_t off = 0;
    auto take = [&](size_t n) { size_t o = off; off += n; return o; };
    oC1 = take(N2 * N2); oC2 = take(N2 * N2); oC3 = take(N2 * N2); oC4 = take(N2); oC6 = take(N2);
    oZ = take(N2 * N2); oE = take(N2 * (4 * NP - 1)); oA = take(N2 * NP); oB = take(N2 * NP);
    oG = take(N2 * (2 * NP - 1)); oD = take(N2 * (2 * NP - 1)); oQ = take((2 * NP - 1) * NP * 2);
    oK2 = take(NP); oK3 = take(NP);
    buf.assign(off, 0.0);
    double *C1 = &buf[oC1], *C2 = &buf[oC2], *C3 = &buf[oC3], *C4 = &buf[oC4], *C6 = &buf[oC6];
    std::vector<double> temp(4 * NP);
    temp[0] = 1.0;
    for (int i = 1; i < 4 * NP; i++) temp[i] = temp[i - 1] * sqrt((double)i);
    for (int n = 0; n < N2; n++)
      for (int m = 0; m <= n; m++) {
        C1[n * N2 + m] = (2 * n - 1) / (double)(n - m);
        C2[n * N2 + m] = (n + m - 1) / (double)(n - m);
        C3[n * N2 + m] = temp[n - m] / temp[n + m];
      }
    C6[0] = 1.0; C6[1] = 1.0;
    for (int n = 2; n < N2; n++) C6[n] = C6[n - 1] * (2 * n - 1);
    for (int n = 0; n < N2; n++) C4[n] = 1.0 / ((2 * n - 1) * (2 * n - 3));
    auto ZETA = [&](int n, int m) -> double & { return buf[oZ + n * N2 + m]; };
    auto ETA = [&](int n, int m) -> double & { return buf[oE + n * (4 * NP - 1) + 2 * NP - 1 + m]; };
    for (int n = 0; n < N2; n++)
      for (int m = 0; m <= n; m++) ZETA(n, m) = sqrt((double)(n + m + 1) * (n - m + 1) / ((2 * n + 1) * (2 * n + 3)));
    for (int n = 0; n < N2; n++)
      for (int m = 0; m <= n; m++) {
        ETA(n, m) = sqrt((double)(n - m - 1) * (n - m) / ((2 * n + 1) * (2 * n - 1)));
        if (m != 0) ETA(n, -m) = -sqrt((double)(n + m - 1) * (n + m) / ((2 * n + 1) * (2 * n - 1)));
      }
    // singular-rotation derivative coefficients from the degenerate harmonics at theta = 0
    {
      const int nn = 2 * NP - 1;
      std::vector<double> SH(nn, 0.0);
      if (nn > 1) SH[1] = -1;
      if (nn > 2) SH[2] = -1.0 * 3;
      for (int l = 3; l < nn; l++) SH[l] = (1.0 * (2 * l - 1) * SH[l - 1] - l * SH[l - 2]) / (l - 1);
      for (int l = 1; l < nn; l++) SH[l] *= (-C3[l * N2 + 1]);
      auto Q = [&](int n, int m, int k) -> double & { return buf[oQ + (n * NP + m) * 2 + k]; };
      for (int n = 1; n < nn; n++) { Q(n, 0, 0) = 0.0; Q(n, 0, 1) = SH[n]; }
      for (int n = 2; n < nn; n++) {
        Q(n - 1, 1, 0) = (ETA(n, -1) * Q(n, 0, 1) + ZETA(n - 1, 0)) / ETA(n, 0);
        Q(n - 1, 1, 1) = (n > 2) ? (ETA(n, 1) / ETA(n, 0)) * Q(n, 0, 1) : 0.0;
      }
      for (int m = 1; m < NP - 1; m++)
        for (int n = m + 2; n < 2 * NP - m - 1; n++) {
          Q(n - 1, m + 1, 0) = (ETA(n, m - 1) * Q(n, m, 0) + ZETA(n - 1, m)) / ETA(n, m);
          Q(n - 1, m + 1, 1) = (n > m + 2) ? (ETA(n, m + 1) / ETA(n, m)) * Q(n, m, 1) : 0.0;
        }
    }
    const double kapsqr = (kappa == 0 ? 0 : 1.0);
    for (int n = 0; n < N2; n++)
      for (int m = 0; m < NP; m++) {
        double &A = buf[oA + n * NP + m], &B = buf[oB + n * NP + m];
        double &G = buf[oG + n * (2 * NP - 1) + NP - 1 + m], &D = buf[oD + n * (2 * NP - 1) + NP - 1 + m];
        A = sqrt((double)(n + m + 1) * (n - m + 1));
        B = kapsqr * A / ((2 * n + 1) * (2 * n + 3));
        G = sqrt((double)(n - m - 1) * (n - m));
        D = kapsqr * G / ((2 * n + 1) * (2 * n - 1));
        if (m != 0) {
          double &Gm = buf[oG + n * (2 * NP - 1) + NP - 1 - m], &Dm = buf[oD + n * (2 * NP - 1) + NP - 1 - m];
          Gm = -sqrt((double)(n + m - 1) * (n + m));
          Dm = kapsqr * Gm / ((2 * n + 1) * (2 * n - 1));
        }
      }
    for (int l = 0; l < NP; l++) { buf[oK2 + l] = (2 * l + 1) / (4.0 * M_PI); buf[oK3 + l] = 1 / (double)(2 * l + 1); }
  }
  Tab view(const double *d) const
  {
    Tab t;
    t.NP = NP; t.kappa = kappa;
    t.C1 = d + oC1; t.C2 = d + oC2; t.C3 = d + oC3; t.C4 = d + oC4; t.C6 = d + oC6;
    t.zeta = d + oZ; t.eta = d + oE; t.alpha = d + oA; t.beta = d + oB; t.gam = d + oG; t.del = d + oD;
    t.Q = d + oQ; t.CONST2 = d + oK2; t.CONST3 = d + oK3;
    return t;
  }
};

// ------------------------------------------------------------------ molecule types (host copy)
struct HostType {
  int ns = 0;
  double maxR = 0;
  std::vector<double> cen, rad;       // molecule frame (sphere centres minus their mean)
  std::vector<double> spx;            // exposed points, per sphere, relative to its centre
  std::vector<int> spx_cnt, nspx;
  std::vector<std::vector<int> > near;
  std::vector<double> fself, hself, hscale, imat;
  std::vector<double> chg_pos, chg;   // relative to the molecule centre
  std::vector<int> chg_lab;           // sphere each charge is assigned to
};

struct pbsam_context {
  pbsam_params prm;
  int device = 0;
  HostTab ht;
  double *dtab = nullptr;
  Tab T;
  std::vector<HostType> types;
  bool finalized = false;
  TypeView tv;
  std::vector<void *> tbufs;
  int live_systems = 0;
};

struct pbsam_system {
  pbsam_context *ctx = nullptr;
  Ctx c;
  int B = 0, nmol = 0;
  std::vector<void *> bufs;
  cudaStream_t stream = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  int crew = 1;            // CTAs (one cluster) per system in the force kernel
  // adaptive crews (cluster_size == -1): systems grouped by the cost of their last
  // evaluation, one launch per crew size on side streams
  bool adaptive = false;
  int *h_stats = nullptr, *h_list = nullptr, *d_list = nullptr;   // pinned host / device
  cudaEvent_t ev_stats = nullptr, ev_fork = nullptr, ev_join[5] = {};
  cudaStream_t gs[5] = {};
  bool stats_pending = false;
  std::vector<int> gsize, gcount;    // per launch: crew size, systems (lists concatenated in d_list)
  struct BDHost *bd = nullptr;       // Brownian-dynamics state (pbsam_system_bd_init)
};
static void bd_free(pbsam_system *s);

// Crew sizes from the last evaluation's inner-iteration counts: every system starts
// with one CTA, the one with the largest cost per CTA doubles (up to 16) while the
// crews fit in the SMs.  Returns per system its crew size.
static std::vector<int> plan_crews(const int *its, int B, int n_sm)
{
  std::vector<int> C(B, 1);
  int total = B;
  for (;;) {
    int best = -1;
    double bc = -1.0;
    for (int b = 0; b < B; b++) {
      if (C[b] >= PBSAM_MAX_CREW) continue;
      const double v = (its[b] + 1.0) / C[b];
      if (v > bc) { bc = v; best = b; }
    }
    if (best < 0 || total + C[best] > n_sm) break;
    total += C[best];
    C[best] *= 2;
  }
  return C;
}

extern "C" void pbsam_params_default(pbsam_params *p)
{
  p->poles = 10; p->salt = 0.05; p->idiel = 4.0; p->sdiel = 78.0; p->temperature = 298.15;
  p->max_polar_dev = 1e-2; p->solve_tol = 1e-8; p->solve_max_ct = 100; p->max_pol_rounds = 1000;
  p->inter_cutoff = 10; p->interact_cutoff = 100; p->intra_cutoff = 30; p->min_sep_numeric = 5;
  p->num_points_x = 10000;
  p->cluster_size = 0;
  p->exact = 0;
  p->box_length = 0.0;
  p->exact_tables = 1;
  p->exact_tol = 1e-14;
  p->exact_relax = 1.0;
}

static double kappa_of(const pbsam_params &p)
{
  const double AVO = 6.0221415e23, ECHG = 1.60217646e-19, EPS0 = 8.854187817e-12;
  const double KBOLTZ = 1.3806503e-23, ANG = 1e-10, LIT = 1e-3;
  return ANG * sqrt((2 * p.salt * AVO / LIT * ECHG * ECHG) / (p.sdiel * EPS0 * KBOLTZ * p.temperature));
}

extern "C" int pbsam_context_create(const pbsam_params *prm, int device, pbsam_context **out)
{
  if (!prm || !out) return fail(PBSAM_E_BADARG, "null argument");
  if (prm->poles < 1 || prm->poles > 32) return fail(PBSAM_E_BADARG, "poles must be in [1, 32]");
  if (prm->cluster_size < -1 || prm->cluster_size > PBSAM_MAX_CREW)
    return fail(PBSAM_E_BADARG, "cluster_size must be -1 (adaptive), 0 (automatic) or 1..16");
  if (prm->exact != 0 && prm->exact != 1) return fail(PBSAM_E_BADARG, "exact must be 0 or 1");
  if (prm->exact_tables != 0 && prm->exact_tables != 1) return fail(PBSAM_E_BADARG, "exact_tables must be 0 or 1");
  if (!(prm->exact_tol > 0.0 && prm->exact_tol < 1.0)) return fail(PBSAM_E_BADARG, "exact_tol must be in (0, 1)");
  if (!(prm->exact_relax > 0.0 && prm->exact_relax < 2.0)) return fail(PBSAM_E_BADARG, "exact_relax must be in (0, 2)");
  if (!(prm->box_length >= 0.0) || !std::isfinite(prm->box_length))
    return fail(PBSAM_E_BADARG, "box_length must be 0 (no periodic box) or a positive edge");
  if (prm->exact && prm->poles > 32) return fail(PBSAM_E_BADARG, "the exact form supports pole orders up to 32");
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(PBSAM_E_BADARG, "no such CUDA device");
  CK(cudaSetDevice(device));
  CK(cudaDeviceSetLimit(cudaLimitStackSize, 8192));
  pbsam_context *c = new pbsam_context();
  c->prm = *prm;
  c->device = device;
  c->ht.build(prm->poles, kappa_of(*prm));
  cudaError_t e = cudaMalloc(&c->dtab, c->ht.buf.size() * sizeof(double));
  if (e != cudaSuccess) { delete c; return fail(PBSAM_E_CUDA, cudaGetErrorString(e)); }
  e = cudaMemcpy(c->dtab, c->ht.buf.data(), c->ht.buf.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(c->dtab); delete c; return fail(PBSAM_E_CUDA, cudaGetErrorString(e)); }
  c->T = c->ht.view(c->dtab);
  *out = c;
  return PBSAM_OK;
}

extern "C" int pbsam_context_kappa(const pbsam_context *c, double *kappa)
{
  if (!c || !kappa) return fail(PBSAM_E_BADARG, "null argument");
  *kappa = c->ht.kappa;
  return PBSAM_OK;
}

extern "C" int pbsam_context_destroy(pbsam_context *c)
{
  if (!c) return PBSAM_OK;
  if (c->live_systems > 0) return fail(PBSAM_E_STATE, "systems still alive");
  cudaSetDevice(c->device);
  for (void *p : c->tbufs) cudaFree(p);
  cudaFree(c->dtab);
  delete c;
  return PBSAM_OK;
}

// ------------------------------------------------------------------ input files
// PQR as read by src/readutil.cpp:285-355 (CEN at byte 18, x y z q r from byte 31)
static bool read_pqr(const char *fname, std::vector<double> &pos, std::vector<double> &ch, std::vector<double> &rad,
                     std::vector<double> &cen)
{
  FILE *f = fopen(fname, "r");
  if (!f) return false;
  char buf[512];
  while (fgets(buf, sizeof buf, f)) {
    if (strncmp(buf, "ATOM", 4) != 0 || strlen(buf) < 32) continue;
    double x, y, z, c, r;
    if (sscanf(buf + 31, "%lf %lf %lf %lf %lf", &x, &y, &z, &c, &r) != 5) continue;
    if (strncmp(buf + 18, "CEN", 3) == 0) { rad.push_back(r); cen.push_back(x); cen.push_back(y); cen.push_back(z); }
    else { pos.push_back(x); pos.push_back(y); pos.push_back(z); ch.push_back(c); }
  }
  fclose(f);
  return true;
}
// IMat binary: int p, then p^4 doubles; a larger p is truncated as src/readutil.cpp:399-435
static bool read_imat(const char *fname, int NP, double *mat)
{
  FILE *f = fopen(fname, "rb");
  if (!f) return false;
  int p = 0;
  if (fread(&p, sizeof(int), 1, f) != 1 || p < NP) { fclose(f); return false; }
  const long psq = (long)NP * NP;
  bool ok = true;
  if (p == NP) ok = fread(mat, sizeof(double), psq * psq, f) == (size_t)(psq * psq);
  else {
    const long matlen = (long)p * p;
    for (long j = 0; j < psq && ok; j++) {
      ok = fread(mat + j * psq, sizeof(double), psq, f) == (size_t)psq;
      fseek(f, (matlen - psq) * (long)sizeof(double), SEEK_CUR);
    }
  }
  fclose(f);
  return ok;
}
// expansion text file: p, scale, rcut, coefficients (src/readutil.cpp:564-598)
static bool read_exp(const char *fname, int NP, double *V, double &scale)
{
  std::ifstream fin(fname);
  if (!fin) return false;
  int pr = 0;
  double rcut = 0;
  fin >> pr >> scale >> rcut;
  if (!fin) return false;
  for (int k = 0; k < NP * NP; k++) V[k] = 0.0;
  const int n = (pr < NP) ? pr * pr : NP * NP;
  for (int k = 0; k < n; k++) fin >> V[k];
  return (bool)fin;
}

// exposed surface points (src/molecule.cpp:756-780, 877-894, 948-994, 2272-2294)
static void make_surface_points(const pbsam_params &prm, HostType &t, const std::vector<double> &cen_abs)
{
  const int ns = t.ns;
  t.spx.clear(); t.spx_cnt.assign(ns, 0); t.nspx.assign(ns, 0);
  for (int k = 0; k < ns; k++) {
    std::vector<int> neigh;
    for (int j = 0; j < ns; j++) {
      if (j == k) continue;
      const double sr = t.rad[k] + t.rad[j];
      const double dx = cen_abs[3 * k] - cen_abs[3 * j], dy = cen_abs[3 * k + 1] - cen_abs[3 * j + 1],
                   dz = cen_abs[3 * k + 2] - cen_abs[3 * j + 2];
      if (dx * dx + dy * dy + dz * dz < sr * sr) neigh.push_back(j);
    }
    const int Nin = prm.num_points_x;
    const double cutoff = 1.5, maxrad = 10, gradient = Nin / ((maxrad - cutoff) * (maxrad - cutoff));
    int N;
    if (t.rad[k] < cutoff) N = 200;
    else { N = int(200 + gradient * (t.rad[k] - cutoff) * (t.rad[k] - cutoff)); if (N > Nin) N = Nin; }
    std::vector<double> th(N), ph(N);
    for (int i = 1; i <= N; i++) {
      const double h = -1.0 + 2.0 * (i - 1.0) / (N - 1.0);
      th[i - 1] = acos(h);
      if (i == 1 || i == N) ph[i - 1] = 0;
      else ph[i - 1] = (ph[i - 2] + 3.6 / sqrt(N * (1.0 - h * h)));
      while (ph[i - 1] > 2 * M_PI) ph[i - 1] -= 2 * M_PI;
      while (ph[i - 1] < -2 * M_PI) ph[i - 1] += 2 * M_PI;
    }
    for (int n = 0; n < N; n++) {
      const double px = t.rad[k] * (1 * sin(th[n]) * cos(ph[n])), py = t.rad[k] * (1 * sin(th[n]) * sin(ph[n])),
                   pz = t.rad[k] * (1 * cos(th[n]));
      bool inside = false;
      for (int j : neigh) {
        const double dx = px + cen_abs[3 * k] - cen_abs[3 * j], dy = py + cen_abs[3 * k + 1] - cen_abs[3 * j + 1],
                     dz = pz + cen_abs[3 * k + 2] - cen_abs[3 * j + 2];
        if (dx * dx + dy * dy + dz * dz < t.rad[j] * t.rad[j]) { inside = true; break; }
      }
      if (!inside) { t.spx.push_back(px); t.spx.push_back(py); t.spx.push_back(pz); t.spx_cnt[k]++; }
    }
    t.nspx[k] = N;
  }
}

static int add_type(pbsam_context *c, HostType &&t0, const std::vector<double> &cen_abs)
{
  HostType t = std::move(t0);
  const int ns = t.ns;
  // molecule centre = mean sphere centre (src/BDnam.cpp:68-70)
  double rc[3] = {0, 0, 0};
  for (int k = 0; k < ns; k++) for (int d = 0; d < 3; d++) rc[d] += cen_abs[3 * k + d];
  const double inv = 1.0 / ns;
  for (int d = 0; d < 3; d++) rc[d] *= inv;
  t.cen.resize(3 * ns);
  t.maxR = 0;
  for (int k = 0; k < ns; k++) {
    for (int d = 0; d < 3; d++) t.cen[3 * k + d] = cen_abs[3 * k + d] - rc[d];
    const double r = sqrt(t.cen[3 * k] * t.cen[3 * k] + t.cen[3 * k + 1] * t.cen[3 * k + 1] + t.cen[3 * k + 2] * t.cen[3 * k + 2]) + t.rad[k];
    if (r > t.maxR) t.maxR = r;
  }
  for (size_t q = 0; q < t.chg.size(); q++) for (int d = 0; d < 3; d++) t.chg_pos[3 * q + d] -= rc[d];
  make_surface_points(c->prm, t, cen_abs);
  // assign each charge to the first sphere that contains it (src/molecule.cpp:1001-1023)
  t.chg_lab.assign(t.chg.size(), -1);
  for (size_t q = 0; q < t.chg.size(); q++) {
    for (int k = 0; k < ns; k++) {
      const double dx = t.chg_pos[3 * q] - t.cen[3 * k], dy = t.chg_pos[3 * q + 1] - t.cen[3 * k + 1],
                   dz = t.chg_pos[3 * q + 2] - t.cen[3 * k + 2];
      if (sqrt(dx * dx + dy * dy + dz * dz) + 0.0 <= t.rad[k]) { t.chg_lab[q] = k; break; }
    }
    if (t.chg_lab[q] < 0) return fail(PBSAM_E_BADARG, "a charge lies outside every sphere");
  }
  // intra near lists (src/molecule.cpp:500-535)
  t.near.assign(ns, std::vector<int>());
  for (int kj = 0; kj < ns; kj++)
    for (int ki = 0; ki < kj; ki++) {
      const double dx = t.cen[3 * ki] - t.cen[3 * kj], dy = t.cen[3 * ki + 1] - t.cen[3 * kj + 1], dz = t.cen[3 * ki + 2] - t.cen[3 * kj + 2];
      const double rho = sqrt(dx * dx + dy * dy + dz * dz);
      if (rho < (t.rad[ki] + t.rad[kj] + c->prm.intra_cutoff)) { t.near[ki].push_back(kj); t.near[kj].push_back(ki); }
    }
  c->types.push_back(std::move(t));
  return (int)c->types.size() - 1;
}
static bool all_finite(const std::vector<double> &v)
{
  for (double x : v)
    if (!std::isfinite(x)) return false;
  return true;
}

static int add_type_checked(pbsam_context *c, HostType &&t, const std::vector<double> &cen_abs, int *type_id)
{
  // a non-finite input would only surface as NaN forces much later
  if (!all_finite(cen_abs) || !all_finite(t.rad) || !all_finite(t.chg_pos) || !all_finite(t.chg))
    return fail(PBSAM_E_BADARG, "non-finite sphere centre, radius or charge");
  for (double r : t.rad)
    if (!(r > 0.0)) return fail(PBSAM_E_BADARG, "sphere radius must be positive");
  if (!all_finite(t.imat)) return fail(PBSAM_E_BADARG, "non-finite IMat entry");
  if (!all_finite(t.fself) || !all_finite(t.hself) || !all_finite(t.hscale))
    return fail(PBSAM_E_BADARG, "non-finite self-polarized expansion");
  const int r = add_type(c, std::move(t), cen_abs);
  if (r < 0) return r;
  *type_id = r;
  return PBSAM_OK;
}

extern "C" int pbsam_moltype_load(pbsam_context *c, const char *pqr, const char *imat_dir, const char *exp_dir,
                                  const char *exp_name, int *type_id)
{
  if (!c || !pqr || !imat_dir || !exp_dir || !exp_name || !type_id) return fail(PBSAM_E_BADARG, "null argument");
  if (c->finalized) return fail(PBSAM_E_STATE, "molecule types are frozen once a system exists");
  const int NP = c->prm.poles;
  HostType t;
  std::vector<double> cen_abs;
  if (!read_pqr(pqr, t.chg_pos, t.chg, t.rad, cen_abs)) return fail(PBSAM_E_IO, std::string("cannot read ") + pqr);
  t.ns = (int)t.rad.size();
  if (t.ns == 0) return fail(PBSAM_E_IO, std::string("no CEN spheres in ") + pqr);
  const long NP2 = (long)NP * NP;
  t.imat.resize((size_t)t.ns * NP2 * NP2);
  t.fself.resize((size_t)t.ns * NP2);
  t.hself.resize((size_t)t.ns * NP2);
  t.hscale.resize(t.ns);
  char fn[4096];
  for (int k = 0; k < t.ns; k++) {
    snprintf(fn, sizeof fn, "%s/imat.sp%d.out.bin", imat_dir, k);
    if (!read_imat(fn, NP, t.imat.data() + (size_t)k * NP2 * NP2)) return fail(PBSAM_E_IO, std::string("cannot read ") + fn);
    double sc;
    snprintf(fn, sizeof fn, "%s/%s.%d.F.exp", exp_dir, exp_name, k);
    if (!read_exp(fn, NP, t.fself.data() + (size_t)k * NP2, sc)) return fail(PBSAM_E_IO, std::string("cannot read ") + fn);
    snprintf(fn, sizeof fn, "%s/%s.%d.H.exp", exp_dir, exp_name, k);
    if (!read_exp(fn, NP, t.hself.data() + (size_t)k * NP2, t.hscale[k])) return fail(PBSAM_E_IO, std::string("cannot read ") + fn);
  }
  return add_type_checked(c, std::move(t), cen_abs, type_id);
}

extern "C" int pbsam_moltype_create(pbsam_context *c, int n_sph, const double *centres, const double *radii, int n_chg,
                                    const double *chg_pos, const double *chg, const double *imats, const double *fself,
                                    const double *hself, const double *hself_scale, int *type_id)
{
  if (!c || n_sph <= 0 || n_chg < 0 || !centres || !radii || !imats || !fself || !hself || !hself_scale || !type_id ||
      (n_chg > 0 && (!chg_pos || !chg)))
    return fail(PBSAM_E_BADARG, "bad argument");
  if (c->finalized) return fail(PBSAM_E_STATE, "molecule types are frozen once a system exists");
  const long NP2 = (long)c->prm.poles * c->prm.poles;
  HostType t;
  t.ns = n_sph;
  t.rad.assign(radii, radii + n_sph);
  t.chg_pos.assign(chg_pos, chg_pos + 3 * n_chg);
  t.chg.assign(chg, chg + n_chg);
  t.imat.assign(imats, imats + (size_t)n_sph * NP2 * NP2);
  t.fself.assign(fself, fself + (size_t)n_sph * NP2);
  t.hself.assign(hself, hself + (size_t)n_sph * NP2);
  t.hscale.assign(hself_scale, hself_scale + n_sph);
  std::vector<double> cen_abs(centres, centres + 3 * n_sph);
  return add_type_checked(c, std::move(t), cen_abs, type_id);
}

extern "C" int pbsam_moltype_info(const pbsam_context *c, int id, int *n_sph, int *n_points)
{
  if (!c || id < 0 || id >= (int)c->types.size()) return fail(PBSAM_E_BADARG, "bad type id");
  if (n_sph) *n_sph = c->types[id].ns;
  if (n_points) *n_points = (int)(c->types[id].spx.size() / 3);
  return PBSAM_OK;
}

template <class T>
static int dalloc(std::vector<void *> &bufs, T **p, size_t n)
{
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) return fail(PBSAM_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  bufs.push_back((void *)*p);
  e = cudaMemset(*p, 0, n * sizeof(T));
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, cudaGetErrorString(e));
  return PBSAM_OK;
}
template <class T>
static int dput(std::vector<void *> &bufs, const T **p, const std::vector<T> &h)
{
  T *d;
  int r = dalloc(bufs, &d, h.size());
  if (r) return r;
  if (!h.empty()) CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  *p = d;
  return PBSAM_OK;
}
#define TRY(x) do { int r_ = (x); if (r_) return r_; } while (0)

// Launch n_sys crews of C CTAs (a thread-block cluster per system when C > 1).
template <class... Exp, class... Act>
static cudaError_t launch_crews(void (*kern)(Exp...), int n_sys, int C, size_t smem, cudaStream_t st, Act &&...args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(n_sys * C));
  cfg.blockDim = dim3(PBSAM_TEAM);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  if (C > 1) {
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Act>(args)...);
}

// CTAs per system: the requested size, or the largest of 16, 8, 4, 2 at which all
// n_sys crews are resident at once (cluster occupancy), else 1.
template <class K>
static int pick_crew(K kern, int n_sys, size_t smem, int requested)
{
  if (requested > 0) return requested;
  for (int C : {16, 8, 4, 2}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(n_sys * C));
    cfg.blockDim = dim3(PBSAM_TEAM);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (const void *)kern, &cfg) == cudaSuccess && n >= n_sys) return C;
    cudaGetLastError();
  }
  return 1;
}

// opt every team kernel into the dynamic shared memory it needs
static int set_smem_attrs(int NP)
{
  const int smem = (int)team_smem_bytes(NP);
  CK(cudaFuncSetAttribute(pbsam_forces_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)forces_smem_bytes(NP)));
  // clusters of up to 16 CTAs (beyond the portable 8)
  CK(cudaFuncSetAttribute(pbsam_forces_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  CK(cudaFuncSetAttribute(pbsam_selfpol_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  CK(cudaFuncSetAttribute(pbsam_energy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(pbsam_setup1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(pbsam_setup2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(pbsam_setup3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(pbsam_selfpol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  CK(cudaFuncSetAttribute(pbsam_nummat_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  return PBSAM_OK;
}

// upload all molecule types and run the per-type setup kernels
// Exact form: the near-field operators of the intra near pairs (pbsam_nummat_kernel):
// of every pair when they fit in 4 GB, else of the numeric pairs alone when those fit,
// else none (tv.nslot and tv.Nmat stay null and the kernels transform the pairs as
// the plain drop-in does).  A pair that the device classifies otherwise than this host
// test (a separation within rounding of 0 or min_sep_numeric) finds an operator of the
// other kind and is transformed the plain way too.
static int build_numeric_operators(std::vector<void *> &B, pbsam_context *c, TypeView &tv, Ctx cx, int NP,
                                   const std::vector<int> &type_off, const std::vector<int> &near_off,
                                   const std::vector<int> &near, const std::vector<int> &spx_off,
                                   const std::vector<double> &cen, const std::vector<double> &rad)
{
  const long long NP2 = (long long)NP * NP;
  const int TS = type_off.back();
  const size_t per = (size_t)2 * NP2 * NP2 * sizeof(double), budget = 4ULL << 30;
  std::vector<int> nslot, slot_e, slot_u, slot_k;
  int maxpts = 1;
  for (int with_analytic = 1; with_analytic >= 0; with_analytic--) {
    nslot.assign(near.size(), -1);
    slot_e.clear(); slot_u.clear(); slot_k.clear();
    for (int ts = 0, t = 0; ts < TS; ts++) {
      while (type_off[t + 1] <= ts) t++;
      for (int e = near_off[ts]; e < near_off[ts + 1]; e++) {
        const int v = type_off[t] + near[e];
        const double P[3] = {cen[3 * ts] - cen[3 * v], cen[3 * ts + 1] - cen[3 * v + 1], cen[3 * ts + 2] - cen[3 * v + 2]};
        const double sep = std::sqrt(P[0] * P[0] + P[1] * P[1] + P[2] * P[2]) - rad[ts] - rad[v];
        const bool analytic = sep > 0 && !(sep < c->prm.min_sep_numeric);
        if (analytic && !with_analytic) continue;
        nslot[e] = (int)slot_e.size();
        slot_e.push_back(e);
        slot_u.push_back(ts);
        slot_k.push_back(analytic ? 0 : 1);
        if (!analytic) maxpts = std::max(maxpts, spx_off[v + 1] - spx_off[v]);
      }
    }
    if (per * slot_e.size() <= budget) break;
  }
  if (slot_e.empty() || per * slot_e.size() > budget) return PBSAM_OK;
  double *N = nullptr;
  TRY(dalloc(B, &N, slot_e.size() * 2 * NP2 * NP2));
  const int *dslot = nullptr, *dkind = nullptr, *de = nullptr, *du = nullptr;
  TRY(dput(B, &dslot, nslot));
  TRY(dput(B, &dkind, slot_k));
  std::vector<void *> tmp;
  auto release = [&]() { for (void *q : tmp) cudaFree(q); };
  int r = dput(tmp, &de, slot_e);
  if (!r) r = dput(tmp, &du, slot_u);
  const int CH = 256, ns = (int)slot_e.size();
  const long long stride = scr_doubles(NP, 1), qstride = 2 * ((maxpts + 1) & ~1LL);
  double *scr = nullptr, *qw = nullptr;
  if (!r) r = dalloc(tmp, &scr, (size_t)stride * CH);
  if (!r) r = dalloc(tmp, &qw, (size_t)qstride * CH);
  if (r) { release(); return r; }
  tv.Nmat = N;
  tv.nslot = dslot;
  tv.nkind = dkind;
  cx.tv = tv;
  cudaError_t e = cudaSuccess;
  for (int s0 = 0; e == cudaSuccess && s0 < ns; s0 += CH) {
    const int n = ns - s0 < CH ? ns - s0 : CH;
    pbsam_nummat_kernel<<<n, PBSAM_TEAM, team_smem_bytes(NP)>>>(cx, de, du, s0, n, scr, stride, qw, qstride, N);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  release();
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("numeric near-field operators: ") + cudaGetErrorString(e));
  return PBSAM_OK;
}

static int finalize_types(pbsam_context *c)
{
  if (c->finalized) return PBSAM_OK;
  if (c->types.empty()) return fail(PBSAM_E_STATE, "no molecule types");
  CK(cudaSetDevice(c->device));
  const int NP = c->prm.poles;
  const long NP2 = (long)NP * NP;
  std::vector<int> type_off(1, 0), spx_off(1, 0), nspx, near_off(1, 0), near, chg_off(1, 0), chg_lab, pair_off(1, 0);
  std::vector<double> maxR, cen, rad, spx, Fs, Hs, hsc, imat, chg_pos, chg;
  int maxq = 0, maxns = 0;
  for (auto &t : c->types) {
    type_off.push_back(type_off.back() + t.ns);
    maxR.push_back(t.maxR);
    cen.insert(cen.end(), t.cen.begin(), t.cen.end());
    rad.insert(rad.end(), t.rad.begin(), t.rad.end());
    for (int k = 0; k < t.ns; k++) {
      spx_off.push_back(spx_off.back() + t.spx_cnt[k]);
      nspx.push_back(t.nspx[k]);
      near_off.push_back(near_off.back() + (int)t.near[k].size());
      near.insert(near.end(), t.near[k].begin(), t.near[k].end());
      pair_off.push_back(pair_off.back() + t.ns - 1);
    }
    spx.insert(spx.end(), t.spx.begin(), t.spx.end());
    Fs.insert(Fs.end(), t.fself.begin(), t.fself.end());
    Hs.insert(Hs.end(), t.hself.begin(), t.hself.end());
    hsc.insert(hsc.end(), t.hscale.begin(), t.hscale.end());
    {
      const size_t base = imat.size(), stride = imat_stride((int)NP2);
      imat.resize(base + (size_t)t.ns * stride, 0.0);
      for (int k = 0; k < t.ns; k++) {
        const double *src = t.imat.data() + (size_t)k * NP2 * NP2;
        double *dst = imat.data() + base + (size_t)k * stride;
        const long ld = imat_ld((int)NP2);
        for (long r = 0; r < NP2; r++)
          for (long cc = 0; cc < NP2; cc++) dst[r * ld + cc] = src[cc * NP2 + r];
      }
    }
    chg_off.push_back(chg_off.back() + (int)t.chg.size());
    chg_pos.insert(chg_pos.end(), t.chg_pos.begin(), t.chg_pos.end());
    chg.insert(chg.end(), t.chg.begin(), t.chg.end());
    chg_lab.insert(chg_lab.end(), t.chg_lab.begin(), t.chg_lab.end());
    if ((int)t.chg.size() > maxq) maxq = (int)t.chg.size();
    if (t.ns > maxns) maxns = t.ns;
  }
  TypeView &tv = c->tv;
  auto &B = c->tbufs;
  tv.ntypes = (int)c->types.size();
  tv.TS = type_off.back();
  const int TS = tv.TS, TP = spx_off.back();
  TRY(dput(B, &tv.type_off, type_off)); TRY(dput(B, &tv.maxR, maxR)); TRY(dput(B, &tv.cen, cen));
  TRY(dput(B, &tv.rad, rad)); TRY(dput(B, &tv.spx_off, spx_off)); TRY(dput(B, &tv.spx, spx));
  TRY(dput(B, &tv.nspx, nspx)); TRY(dput(B, &tv.Fself, Fs)); TRY(dput(B, &tv.Hself, Hs));
  TRY(dput(B, &tv.hself_scale, hsc)); TRY(dput(B, &tv.near_off, near_off)); TRY(dput(B, &tv.near, near));
  TRY(dput(B, &tv.imat, imat));
  TRY(dput(B, &tv.chg_off, chg_off)); TRY(dput(B, &tv.chg_pos, chg_pos));
  TRY(dput(B, &tv.chg, chg));
  TRY(dput(B, &tv.chg_lab, chg_lab));
  TRY(dput(B, &tv.pair_off, pair_off));
  TRY(dalloc(B, &tv.Eass, TS * NP2));
  const int TE = pair_off.back();   // ordered intra pairs of all types
  TRY(dalloc(B, &tv.pR, (size_t)TE * rot_off(NP)));
  TRY(dalloc(B, &tv.pTH, (size_t)TE * tr_off(NP)));
  TRY(dalloc(B, &tv.pTF, (size_t)TE * tr_off(NP)));
  TRY(dalloc(B, &tv.pS, (size_t)TE * 16));
  TRY(dalloc(B, &tv.qFself, TP)); TRY(dalloc(B, &tv.qHself, TP));
  TRY(dalloc(B, &tv.tFself, TS)); TRY(dalloc(B, &tv.tHself, TS));
  TRY(dalloc(B, &tv.LFintra, TS * NP2)); TRY(dalloc(B, &tv.LHintra, TS * NP2));
  TRY(dalloc(B, &tv.LFfar, TS * NP2)); TRY(dalloc(B, &tv.LHfar, TS * NP2));
  TRY(dalloc(B, &tv.Dfix, TS * NP2)); TRY(dalloc(B, &tv.Vfix, TS * NP2));
  TRY(dalloc(B, &tv.cst, (size_t)TS * CST_N * NP));
  // setup scratch: one team per type sphere; misc must hold 2 weights per charge
  long long Sm = maxns;
  while (4096 + Sm * Sm < 2LL * maxq) Sm++;
  const long long stride = scr_doubles(NP, Sm);
  double *scr;
  if (cudaMalloc(&scr, (size_t)stride * TS * sizeof(double)) != cudaSuccess)
    return fail(PBSAM_E_NOMEM, "setup scratch");
  Ctx cx;
  memset(&cx, 0, sizeof cx);
  cx.T = c->T;
  cx.tv = tv;
  cx.prm.idiel = c->prm.idiel; cx.prm.sdiel = c->prm.sdiel;
  cx.prm.min_sep_numeric = c->prm.min_sep_numeric;
  TRY(set_smem_attrs(NP));
  const size_t smem = team_smem_bytes(NP);
  pbsam_setup1_kernel<<<TS, PBSAM_TEAM, smem>>>(cx, scr, stride);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  // intra pair tables, in chunks of CH entries (slim per-block scratch)
  const int CH = 512;
  const long long s3 = 4LL * NP * NP + tr_off(2 * NP - 1) + 2 * NP + 8;
  double *scr3 = nullptr;
  if (e == cudaSuccess && TE > 0) e = cudaMalloc(&scr3, (size_t)s3 * CH * sizeof(double));
  for (int e0 = 0; e == cudaSuccess && e0 < TE; e0 += CH) {
    const int ne = (TE - e0 < CH) ? TE - e0 : CH;
    pbsam_setup3_kernel<<<ne, PBSAM_TEAM, smem>>>(cx, e0, ne, scr3, s3);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (scr3) cudaFree(scr3);
  if (e == cudaSuccess) { pbsam_setup2_kernel<<<TS, PBSAM_TEAM, smem>>>(cx, scr, stride); e = cudaGetLastError(); }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(scr);
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("setup kernels: ") + cudaGetErrorString(e));
  if (c->prm.exact) {
    // exact form: the inner fixed point of every type sphere solved once for all
    // right-hand sides (pbsam_direct_kernel), in chunks whose elimination blocks
    // take at most about 2 GB
    const long long n = 2 * NP2;
    double *G = nullptr;
    TRY(dalloc(B, &G, (size_t)TS * n * n));
    tv.Gdir = G;
    const size_t blk = (size_t)n * 2 * n * sizeof(double);
    int chunk = (int)std::max<size_t>(1, (size_t)(2ULL << 30) / blk);
    if (chunk > TS) chunk = TS;
    double *work = nullptr;
    int *derr = nullptr;
    if (cudaMalloc(&work, blk * chunk) != cudaSuccess) return fail(PBSAM_E_NOMEM, "exact-form elimination blocks");
    if (cudaMalloc(&derr, sizeof(int)) != cudaSuccess) { cudaFree(work); return fail(PBSAM_E_NOMEM, "flag"); }
    cudaMemset(derr, 0, sizeof(int));
    for (int t0 = 0; e == cudaSuccess && t0 < TS; t0 += chunk) {
      const int nb = TS - t0 < chunk ? TS - t0 : chunk;
      pbsam_direct_kernel<<<nb, PBSAM_TEAM>>>(c->T, tv, t0, work, derr);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(work);
    cudaFree(derr);
    if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("exact-form operators: ") + cudaGetErrorString(e));
    if (herr) return fail(PBSAM_E_BADARG, "a sphere's inner fixed point is singular; the exact form cannot be used");
    if (c->prm.exact_tables) TRY(build_numeric_operators(B, c, tv, cx, NP, type_off, near_off, near, spx_off, cen, rad));
    // the exposed points' angles (32 bytes a point), read by the surface charges
    if (c->prm.exact_tables && TP > 0) {
      double *A = nullptr;
      TRY(dalloc(B, &A, (size_t)TP * 4));
      pbsam_spang_kernel<<<(TP + 255) / 256, 256>>>(tv, TP, A);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaDeviceSynchronize();
      if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("surface point angles: ") + cudaGetErrorString(e));
      tv.spang = A;
    }
  }
  c->finalized = true;
  return PBSAM_OK;
}

extern "C" int pbsam_system_create(pbsam_context *c, int n_systems, int n_mol, const int *mol_types, pbsam_system **out)
{
  if (!c || n_systems <= 0 || n_mol <= 0 || n_mol > 64 || !mol_types || !out) return fail(PBSAM_E_BADARG, "bad argument");
  for (int i = 0; i < n_mol; i++)
    if (mol_types[i] < 0 || mol_types[i] >= (int)c->types.size()) return fail(PBSAM_E_BADARG, "bad molecule type");
  TRY(finalize_types(c));
  CK(cudaSetDevice(c->device));
  const int NP = c->prm.poles;
  const long NP2 = (long)NP * NP;
  pbsam_system *s = new pbsam_system();
  s->ctx = c;
  s->B = n_systems; s->nmol = n_mol;
  std::vector<int> mol_off(1, 0), sph_ts, sph_mol, pt_off(1, 0), toff(1, 0);
  for (auto &t : c->types) toff.push_back(toff.back() + t.ns);
  for (int i = 0; i < n_mol; i++) {
    const HostType &t = c->types[mol_types[i]];
    for (int k = 0; k < t.ns; k++) {
      sph_ts.push_back(toff[mol_types[i]] + k);
      sph_mol.push_back(i);
      pt_off.push_back(pt_off.back() + t.spx_cnt[k]);
    }
    mol_off.push_back(mol_off.back() + t.ns);
  }
  const int S = mol_off.back(), SP = pt_off.back();
  const long long B = n_systems;
  BatchView &bv = s->c.bv;
  auto &Bf = s->bufs;
  bv.B = n_systems; bv.nmol = n_mol; bv.S = S; bv.SP = SP;
  std::vector<int> mt(mol_types, mol_types + n_mol);
  int r = 0;
  auto chk = [&](int rr) { if (rr && !r) r = rr; };
  chk(dput(Bf, &bv.mol_type, mt)); chk(dput(Bf, &bv.mol_off, mol_off)); chk(dput(Bf, &bv.sph_ts, sph_ts));
  chk(dput(Bf, &bv.sph_mol, sph_mol)); chk(dput(Bf, &bv.pt_off, pt_off));
  double *pos, *quat;
  chk(dalloc(Bf, &pos, B * n_mol * 3)); chk(dalloc(Bf, &quat, B * n_mol * 4));
  bv.pos = pos; bv.quat = quat;
  bv.fmask = nullptr;
  chk(dalloc(Bf, &bv.F, B * S * NP2)); chk(dalloc(Bf, &bv.H, B * S * NP2)); chk(dalloc(Bf, &bv.Hrot, B * S * NP2));
  chk(dalloc(Bf, &bv.HselfRot, B * S * NP2)); chk(dalloc(Bf, &bv.LS, B * S * NP2));
  chk(dalloc(Bf, &bv.LFS, B * S * NP2)); chk(dalloc(Bf, &bv.LHS, B * S * NP2));
  chk(dalloc(Bf, &bv.hscale, B * S)); chk(dalloc(Bf, &bv.tF, B * S)); chk(dalloc(Bf, &bv.tH, B * S));
  chk(dalloc(Bf, &bv.maxgF, B * S)); chk(dalloc(Bf, &bv.maxgH, B * S)); chk(dalloc(Bf, &bv.dev, B * S));
  chk(dalloc(Bf, &bv.qF, B * SP)); chk(dalloc(Bf, &bv.qH, B * SP));
  chk(dalloc(Bf, &bv.gFp, B * SP * 3)); chk(dalloc(Bf, &bv.gHp, B * SP * 3));
  chk(dalloc(Bf, &bv.gLHN, B * S * 3 * NP2)); chk(dalloc(Bf, &bv.gH, B * S * 3 * NP2));
  chk(dalloc(Bf, &bv.cenRot, B * S * 3));
  chk(dalloc(Bf, &bv.Hlab, B * S * NP2));
  chk(dalloc(Bf, &bv.ipol, B * S * S)); chk(dalloc(Bf, &bv.ipol_n, B * S));
  chk(dalloc(Bf, &bv.iact, B * S * S)); chk(dalloc(Bf, &bv.iact_n, B * S));
  chk(dalloc(Bf, &bv.interMol, B * n_mol * S)); chk(dalloc(Bf, &bv.interMol_n, B * n_mol));
  chk(dalloc(Bf, &bv.intraPol, B * n_mol * S)); chk(dalloc(Bf, &bv.intraPol_n, B * n_mol));
  chk(dalloc(Bf, &bv.intraAct, B * n_mol * S)); chk(dalloc(Bf, &bv.intraAct_n, B * n_mol));
  chk(dalloc(Bf, &bv.interX, B * n_mol));
  chk(dalloc(Bf, &bv.gFw, B * S * 3 * NP2)); chk(dalloc(Bf, &bv.gHw, B * S * 3 * NP2));
  chk(dalloc(Bf, &bv.gHrotw, B * S * 3 * NP2)); chk(dalloc(Bf, &bv.tGw, B * S * 3 * NP2));
  chk(dalloc(Bf, &bv.gkey, B * S)); chk(dalloc(Bf, &bv.dgrad, B * S));
  chk(dalloc(Bf, &bv.molR, (size_t)B * n_mol * rot_off(2 * NP - 1)));
  chk(dalloc(Bf, &bv.molRS, B * n_mol * 16));
  chk(dalloc(Bf, &bv.sep, B * S * S));
  // the exact form runs one CTA per system (its backward pass is not shared by a crew)
  s->adaptive = c->prm.cluster_size < 0 && !c->prm.exact;
  s->crew = c->prm.exact ? 1 : pick_crew(pbsam_forces_kernel, B, forces_smem_bytes(NP), s->adaptive ? 0 : c->prm.cluster_size);
  bv.crew = s->adaptive ? PBSAM_MAX_CREW : s->crew;   // scratch blocks per system: the largest crew it may get
  bv.scr_stride = scr_doubles(NP, S);
  chk(dalloc(Bf, &bv.scr, (size_t)B * bv.crew * bv.scr_stride));
  bv.wscr_stride = NP <= PBSAM_WARP_MAX_NP ? warp_scr_doubles(NP) : 0;   // no warp transforms above
  chk(dalloc(Bf, &bv.wscr, (size_t)B * bv.crew * PBSAM_WARPS * bv.wscr_stride));
  chk(dalloc(Bf, &bv.dorder, (size_t)B * bv.crew * S));
  if (s->adaptive) chk(dalloc(Bf, &s->d_list, B));
  chk(dalloc(Bf, &bv.force, B * n_mol * 3)); chk(dalloc(Bf, &bv.torque, B * n_mol * 3));
  chk(dalloc(Bf, &bv.dpos, B * n_mol * 3)); chk(dalloc(Bf, &bv.drot, B * n_mol * 3));
  chk(dalloc(Bf, &bv.energy, B)); chk(dalloc(Bf, &bv.status, B)); chk(dalloc(Bf, &bv.stats, B * 8));
  chk(dalloc(Bf, &bv.tphase, B * PH_N));
  if (r) {
    for (void *p : Bf) cudaFree(p);
    delete s;
    return r;
  }
  s->c.T = c->T;
  s->c.tv = c->tv;
  SolveParams &p = s->c.prm;
  p.max_polar_dev = c->prm.max_polar_dev; p.solve_tol = c->prm.solve_tol; p.solve_max_ct = c->prm.solve_max_ct;
  p.max_pol_rounds = c->prm.max_pol_rounds; p.inter_cut = c->prm.inter_cutoff; p.interact_cut = c->prm.interact_cutoff;
  p.min_sep_numeric = c->prm.min_sep_numeric; p.idiel = c->prm.idiel; p.sdiel = c->prm.sdiel;
  p.exact = c->prm.exact;
  p.exact_tol = c->prm.exact_tol;
  p.exact_relax = c->prm.exact_relax;
  p.box = c->prm.box_length;
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  if (s->adaptive) {
    if (cudaMallocHost(&s->h_stats, (size_t)B * 8 * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&s->h_list, (size_t)B * sizeof(int)) != cudaSuccess)
      r = fail(PBSAM_E_NOMEM, "pinned host buffers");
    cudaEventCreateWithFlags(&s->ev_stats, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming);
    for (int g = 0; g < 5; g++) {
      cudaEventCreateWithFlags(&s->ev_join[g], cudaEventDisableTiming);
      cudaStreamCreateWithFlags(&s->gs[g], cudaStreamNonBlocking);
    }
  }
  c->live_systems++;
  if (r) {
    pbsam_system_destroy(s);
    return r;
  }
  *out = s;
  return pbsam_system_reset(s);
}

extern "C" int pbsam_system_reset(pbsam_system *s)
{
  if (!s) return fail(PBSAM_E_BADARG, "null system");
  CK(cudaSetDevice(s->ctx->device));
  pbsam_init_kernel<<<s->B, PBSAM_TEAM, 0, s->stream>>>(s->c);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->stream));
  return PBSAM_OK;
}

extern "C" int pbsam_system_destroy(pbsam_system *s)
{
  if (!s) return PBSAM_OK;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->stream);
  for (void *p : s->bufs) cudaFree(p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->adaptive) {
    for (int g = 0; g < 5; g++) {
      if (s->gs[g]) { cudaStreamSynchronize(s->gs[g]); cudaStreamDestroy(s->gs[g]); }
      if (s->ev_join[g]) cudaEventDestroy(s->ev_join[g]);
    }
    if (s->ev_stats) cudaEventDestroy(s->ev_stats);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    if (s->h_stats) cudaFreeHost(s->h_stats);
    if (s->h_list) cudaFreeHost(s->h_list);
  }
  bd_free(s);
  s->ctx->live_systems--;
  delete s;
  return PBSAM_OK;
}

extern "C" int pbsam_system_set_stream(pbsam_system *s, void *stream)
{
  if (!s) return fail(PBSAM_E_BADARG, "null system");
  s->stream = (cudaStream_t)stream;
  return PBSAM_OK;
}

extern "C" int pbsam_system_set_poses(pbsam_system *s, const double *pos, const double *quat, int on_device)
{
  if (!s || !pos || !quat) return fail(PBSAM_E_BADARG, "null argument");
  CK(cudaSetDevice(s->ctx->device));
  const size_t n = (size_t)s->B * s->nmol;
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CK(cudaMemcpyAsync((void *)s->c.bv.pos, pos, n * 3 * sizeof(double), k, s->stream));
  CK(cudaMemcpyAsync((void *)s->c.bv.quat, quat, n * 4 * sizeof(double), k, s->stream));
  if (!on_device) CK(cudaStreamSynchronize(s->stream));
  return PBSAM_OK;
}

extern "C" int pbsam_system_compute_forces(pbsam_system *s, double *force, double *torque, int *status, int on_device)
{
  if (!s) return fail(PBSAM_E_BADARG, "null system");
  CK(cudaSetDevice(s->ctx->device));
  const size_t smem = forces_smem_bytes(s->ctx->prm.poles);
  if (s->adaptive && s->stats_pending) {
    // regroup from the last evaluation's costs, every call: wait for the counters of
    // the previous evaluation, so that the plan depends on the counts alone and not
    // on how far the GPU has got when the host asks
    CK(cudaEventSynchronize(s->ev_stats));
    s->stats_pending = false;
    std::vector<int> its(s->B);
    for (int b = 0; b < s->B; b++) its[b] = s->h_stats[8 * b + 1];
    int n_sm = 0;
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, s->ctx->device));
    const std::vector<int> C = plan_crews(its.data(), s->B, n_sm - n_sm / 16);
    std::vector<int> gsize, gcount, list;
    for (int size : {16, 8, 4, 2, 1}) {
      int cnt = 0;
      for (int b = 0; b < s->B; b++)
        if (C[b] == size) { list.push_back(b); cnt++; }
      if (cnt) { gsize.push_back(size); gcount.push_back(cnt); }
    }
    bool same = (gsize == s->gsize && gcount == s->gcount);
    for (int i = 0; same && i < s->B; i++) same = (s->h_list[i] == list[i]);
    if (!same) {
      CK(cudaStreamSynchronize(s->stream));      // the previous list upload has completed
      for (int i = 0; i < s->B; i++) s->h_list[i] = list[i];
      CK(cudaMemcpyAsync(s->d_list, s->h_list, s->B * sizeof(int), cudaMemcpyHostToDevice, s->stream));
      s->gsize = gsize;
      s->gcount = gcount;
    }
  }
  CK(cudaEventRecord(s->ev0, s->stream));
  if (!s->adaptive || s->gsize.empty()) {
    CK(launch_crews(pbsam_forces_kernel, s->B, s->crew, smem, s->stream, s->c, (const int *)nullptr));
  } else {
    // one launch per crew size on side streams, heaviest first, joined back
    CK(cudaEventRecord(s->ev_fork, s->stream));
    int off = 0;
    for (size_t g = 0; g < s->gsize.size(); g++) {
      CK(cudaStreamWaitEvent(s->gs[g], s->ev_fork, 0));
      CK(launch_crews(pbsam_forces_kernel, s->gcount[g], s->gsize[g], smem, s->gs[g], s->c,
                      (const int *)(s->d_list + off)));
      CK(cudaEventRecord(s->ev_join[g], s->gs[g]));
      off += s->gcount[g];
    }
    for (size_t g = 0; g < s->gsize.size(); g++) CK(cudaStreamWaitEvent(s->stream, s->ev_join[g], 0));
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(s->ev1, s->stream));
  if (s->adaptive && !s->stats_pending) {
    CK(cudaMemcpyAsync(s->h_stats, s->c.bv.stats, (size_t)s->B * 8 * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaEventRecord(s->ev_stats, s->stream));
    s->stats_pending = true;
  }
  const size_t n = (size_t)s->B * s->nmol * 3;
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (force) CK(cudaMemcpyAsync(force, s->c.bv.force, n * sizeof(double), k, s->stream));
  if (torque) CK(cudaMemcpyAsync(torque, s->c.bv.torque, n * sizeof(double), k, s->stream));
  if (status) CK(cudaMemcpyAsync(status, s->c.bv.status, s->B * sizeof(int), k, s->stream));
  if (!on_device) {
    CK(cudaStreamSynchronize(s->stream));
    CK(cudaEventElapsedTime(&s->last_ms, s->ev0, s->ev1));
  }
  return PBSAM_OK;
}

static int energy_launch(pbsam_system *s, double *energy, int on_device, int lab)
{
  if (!s || !energy) return fail(PBSAM_E_BADARG, "null argument");
  CK(cudaSetDevice(s->ctx->device));
  pbsam_energy_kernel<<<s->B, PBSAM_TEAM, team_smem_bytes(s->ctx->prm.poles), s->stream>>>(s->c, lab);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(energy, s->c.bv.energy, s->B * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s->stream));
  if (!on_device) CK(cudaStreamSynchronize(s->stream));
  return PBSAM_OK;
}

extern "C" int pbsam_system_compute_energy(pbsam_system *s, double *energy, int on_device)
{
  return energy_launch(s, energy, on_device, 0);
}

extern "C" int pbsam_system_compute_energy_lab(pbsam_system *s, double *energy, int on_device)
{
  return energy_launch(s, energy, on_device, 1);
}

extern "C" int pbsam_system_backward(pbsam_system *s, const double *seed, double *dpos, double *dquat, double *drot,
                                     int on_device)
{
  if (!s) return fail(PBSAM_E_BADARG, "null system");
  if (!s->ctx->prm.exact) return fail(PBSAM_E_STATE, "the backward pass needs a context made with exact = 1");
  CK(cudaSetDevice(s->ctx->device));
  const size_t n = (size_t)s->B * s->nmol;
  std::vector<void *> tmp;
  auto cleanup = [&]() { for (void *p : tmp) cudaFree(p); };
  double *dseed = nullptr, *dp = nullptr, *dq = nullptr, *dr = nullptr;
  if (seed) {
    if (on_device) dseed = (double *)seed;
    else {
      if (cudaMalloc(&dseed, s->B * sizeof(double)) != cudaSuccess) return fail(PBSAM_E_NOMEM, "seed");
      tmp.push_back(dseed);
      if (cudaMemcpyAsync(dseed, seed, s->B * sizeof(double), cudaMemcpyHostToDevice, s->stream) != cudaSuccess) {
        cleanup();
        return fail(PBSAM_E_CUDA, "seed copy");
      }
    }
  }
  auto out = [&](double *user, size_t len, double **dev) -> int {
    if (!user) { *dev = nullptr; return PBSAM_OK; }
    if (on_device) { *dev = user; return PBSAM_OK; }
    if (cudaMalloc(dev, len * sizeof(double)) != cudaSuccess) return fail(PBSAM_E_NOMEM, "backward output");
    tmp.push_back(*dev);
    return PBSAM_OK;
  };
  int r = out(dpos, 3 * n, &dp);
  if (!r) r = out(dquat, 4 * n, &dq);
  if (!r) r = out(drot, 3 * n, &dr);
  if (r) { cudaStreamSynchronize(s->stream); cleanup(); return r; }
  pbsam_backward_out_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s->stream>>>(s->c.bv, dseed, dp, dq, dr);
  cudaError_t e = cudaGetLastError();
  if (!on_device) {
    if (e == cudaSuccess && dpos) e = cudaMemcpyAsync(dpos, dp, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && dquat) e = cudaMemcpyAsync(dquat, dq, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess && drot) e = cudaMemcpyAsync(drot, dr, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  }
  cudaError_t e2 = cudaStreamSynchronize(s->stream);
  if (e == cudaSuccess) e = e2;
  cleanup();
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("backward: ") + cudaGetErrorString(e));
  return PBSAM_OK;
}

extern "C" int pbsam_system_potential(pbsam_system *s, int n_points, const double *points, int per_system, int lab,
                                      double *pot, int on_device)
{
  if (!s || n_points <= 0 || !points || !pot) return fail(PBSAM_E_BADARG, "bad argument");
  CK(cudaSetDevice(s->ctx->device));
  const size_t np = (size_t)n_points * (per_system ? s->B : 1), no = (size_t)n_points * s->B;
  const double *dpts = points;
  double *dpot = pot, *tp = nullptr, *to = nullptr;
  if (!on_device) {
    if (cudaMalloc(&tp, np * 3 * sizeof(double)) != cudaSuccess) return fail(PBSAM_E_NOMEM, "points");
    if (cudaMalloc(&to, no * sizeof(double)) != cudaSuccess) { cudaFree(tp); return fail(PBSAM_E_NOMEM, "potential"); }
    dpts = tp;
    dpot = to;
  }
  cudaError_t e = cudaSuccess;
  if (!on_device) e = cudaMemcpyAsync(tp, points, np * 3 * sizeof(double), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess && lab) {
    pbsam_hlab_kernel<<<s->B, PBSAM_TEAM, team_smem_bytes(s->ctx->prm.poles), s->stream>>>(s->c);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    pbsam_potential_kernel<<<(unsigned)((no + 127) / 128), 128, 0, s->stream>>>(s->c, n_points, dpts, per_system ? 1 : 0,
                                                                                 lab ? 1 : 0, dpot);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && !on_device) e = cudaMemcpyAsync(pot, to, no * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  const cudaError_t e2 = cudaStreamSynchronize(s->stream);
  if (e == cudaSuccess) e = e2;
  if (tp) cudaFree(tp);
  if (to) cudaFree(to);
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("potential: ") + cudaGetErrorString(e));
  return PBSAM_OK;
}

extern "C" int pbsam_system_stats(const pbsam_system *s, int *stats)
{
  if (!s || !stats) return fail(PBSAM_E_BADARG, "null argument");
  CK(cudaSetDevice(s->ctx->device));
  CK(cudaMemcpy(stats, s->c.bv.stats, (size_t)s->B * 8 * sizeof(int), cudaMemcpyDeviceToHost));
  return PBSAM_OK;
}

extern "C" int pbsam_system_last_kernel_ms(const pbsam_system *s, double *ms)
{
  if (!s || !ms) return fail(PBSAM_E_BADARG, "null argument");
  *ms = s->last_ms;
  return PBSAM_OK;
}

// ------------------------------------------------------------------ IMat builder
// Surface-integral matrices of a molecule's spheres (pbsam mat: CMolecule IMat
// constructor, src/molecule.cpp:279-346, getSpherePoints, src/molecule.cpp:901-939,
// build_IMatE, src/expcenter.cpp:910-1033).  centres are absolute; imats receives
// n_sph * p^4 doubles (column-major p^2 x p^2 per sphere).
extern "C" int pbsam_imat_build(pbsam_context *c, int n_sph, const double *centres, const double *radii, int n_points,
                                double *imats)
{
  if (!c || n_sph <= 0 || !centres || !radii || n_points < 3 || !imats) return fail(PBSAM_E_BADARG, "bad argument");
  CK(cudaSetDevice(c->device));
  const int P = c->prm.poles, N = P * P;
  // molecule-centred coordinates as the reference prepares them
  double rc[3] = {0, 0, 0};
  for (int k = 0; k < n_sph; k++) for (int d = 0; d < 3; d++) rc[d] += centres[3 * k + d];
  const double inv = 1.0 / n_sph;
  for (int d = 0; d < 3; d++) rc[d] *= inv;
  std::vector<double> cr(3 * n_sph);
  for (int k = 0; k < n_sph; k++) for (int d = 0; d < 3; d++) cr[3 * k + d] = centres[3 * k + d] - rc[d];
  // unit-sphere spiral shared by every sphere (src/molecule.cpp:2272-2294)
  std::vector<double> qx(n_points), qy(n_points), qz(n_points);
  {
    const int Np = n_points;
    double phprev = 0;
    for (int i = 1; i <= Np; i++) {
      const double h = -1.0 + 2.0 * (i - 1.0) / (Np - 1.0);
      const double th = acos(h);
      double ph = (i == 1 || i == Np) ? 0 : (phprev + 3.6 / sqrt(Np * (1.0 - h * h)));
      while (ph > 2 * M_PI) ph -= 2 * M_PI;
      while (ph < -2 * M_PI) ph += 2 * M_PI;
      phprev = ph;
      qx[i - 1] = 1 * sin(th) * cos(ph); qy[i - 1] = 1 * sin(th) * sin(ph); qz[i - 1] = 1 * cos(th);
    }
  }
  const int KC = 16384;
  double *dY = nullptr, *dG = nullptr, *dGs = nullptr, *dIM = nullptr, *dP = nullptr;
  std::vector<void *> tmp;
  auto cleanup = [&]() { for (void *p : tmp) cudaFree(p); };
  if (cudaMalloc(&dY, (size_t)KC * N * sizeof(double)) != cudaSuccess) { cleanup(); return fail(PBSAM_E_NOMEM, "imat Y"); }
  tmp.push_back(dY);
  if (cudaMalloc(&dG, (size_t)N * N * sizeof(double)) != cudaSuccess) { cleanup(); return fail(PBSAM_E_NOMEM, "imat G"); }
  tmp.push_back(dG);
  if (cudaMalloc(&dIM, (size_t)N * N * sizeof(double)) != cudaSuccess) { cleanup(); return fail(PBSAM_E_NOMEM, "imat"); }
  tmp.push_back(dIM);
  if (cudaMalloc(&dGs, (size_t)P * P * sizeof(double)) != cudaSuccess) { cleanup(); return fail(PBSAM_E_NOMEM, "imat Gs"); }
  tmp.push_back(dGs);
  if (cudaMalloc(&dP, (size_t)n_points * 3 * sizeof(double)) != cudaSuccess) { cleanup(); return fail(PBSAM_E_NOMEM, "imat pts"); }
  tmp.push_back(dP);
  const double dA = 4 * M_PI / (double)(n_points - 1);
  for (int k = 0; k < n_sph; k++) {
    std::vector<int> neigh;
    for (int j = 0; j < n_sph; j++) {
      if (j == k) continue;
      const double sr = radii[k] + radii[j];
      const double dx = centres[3 * k] - centres[3 * j], dy = centres[3 * k + 1] - centres[3 * j + 1],
                   dz = centres[3 * k + 2] - centres[3 * j + 2];
      if (dx * dx + dy * dy + dz * dz < sr * sr) neigh.push_back(j);
    }
    std::vector<double> E, Bp;
    for (int i = 0; i < n_points; i++) {
      const double px = radii[k] * qx[i], py = radii[k] * qy[i], pz = radii[k] * qz[i];
      bool buried = false;
      for (int j : neigh) {
        const double dx = (px + cr[3 * k]) - cr[3 * j], dy = (py + cr[3 * k + 1]) - cr[3 * j + 1],
                     dz = (pz + cr[3 * k + 2]) - cr[3 * j + 2];
        if (dx * dx + dy * dy + dz * dz < radii[j] * radii[j] * 1.0) { buried = true; break; }
      }
      std::vector<double> &dst = buried ? Bp : E;
      dst.push_back(px); dst.push_back(py); dst.push_back(pz);
    }
    const int npe = (int)E.size() / 3, npb = (int)Bp.size() / 3;
    const int buried = (npe <= npb) ? 0 : 1;
    const std::vector<double> &pts = buried ? Bp : E;
    const int K = (int)pts.size() / 3;
    CK(cudaMemset(dG, 0, (size_t)N * N * sizeof(double)));
    CK(cudaMemset(dGs, 0, (size_t)P * P * sizeof(double)));
    if (K > 0) CK(cudaMemcpy(dP, pts.data(), pts.size() * sizeof(double), cudaMemcpyHostToDevice));
    for (int h0 = 0; h0 < K; h0 += KC) {
      const int kc = (K - h0 < KC) ? K - h0 : KC;
      imat_sh_kernel<<<(kc + 127) / 128, 128>>>(c->T, dP + 3 * (size_t)h0, kc, P, dY);
      dim3 g((N + GT - 1) / GT, (N + GT - 1) / GT);
      gram_kernel<<<g, 256>>>(dY, kc, N, dG);
      gram_simpson_kernel<<<(P * P + 127) / 128, 128>>>(dY, kc, P, h0, dGs);
      CK(cudaGetLastError());
    }
    const long long tot = (long long)N * N;
    imat_assemble_kernel<<<(unsigned)((tot + 255) / 256), 256>>>(c->T, dG, dGs, P, dA, buried, dIM);
    CK(cudaGetLastError());
    CK(cudaMemcpy(imats + (size_t)k * N * N, dIM, (size_t)N * N * sizeof(double), cudaMemcpyDeviceToHost));
  }
  cleanup();
  return PBSAM_OK;
}

// ------------------------------------------------------------------ self-polarization
// pbsam spol (src/selfp_makemat.cpp:37-118, CMolecule::polarize_self,
// src/molecule.cpp:1898-1979) for molecule type type_id (its own F/H inputs are
// ignored).  Outputs are rounded as the reference writes them to .exp files
// (8 significant digits, |x| < 1e-15 -> 0, src/readutil.cpp:541-556,
// src/expansion.cpp:913-929): fself/hself[n_sph * p^2], hself_scale[n_sph].
static double round8(double x)
{
  if (fabs(x) < 1e-15) return 0.0;
  char b[64];
  snprintf(b, sizeof b, "%.8g", x);
  return strtod(b, nullptr);
}

extern "C" int pbsam_selfpol(pbsam_context *c, int type_id, int max_rounds, double *fself, double *hself,
                             double *hself_scale, int *rounds)
{
  if (!c || type_id < 0 || type_id >= (int)c->types.size() || !fself || !hself || !hself_scale || max_rounds < 1)
    return fail(PBSAM_E_BADARG, "bad argument");
  pbsam_system *s = nullptr;
  const int mt[1] = {type_id};
  TRY(pbsam_system_create(c, 1, 1, mt, &s));
  int *drounds = nullptr;
  if (cudaMalloc(&drounds, sizeof(int)) != cudaSuccess) { pbsam_system_destroy(s); return fail(PBSAM_E_NOMEM, "rounds"); }
  cudaError_t e = launch_crews(pbsam_selfpol_kernel, 1, s->crew, team_smem_bytes(c->prm.poles), s->stream, s->c,
                               (const double *)c->tv.Eass, max_rounds, drounds);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  const int ns = c->types[type_id].ns, NP2 = c->prm.poles * c->prm.poles;
  std::vector<double> F((size_t)ns * NP2), H((size_t)ns * NP2);
  int r = 0;
  if (e == cudaSuccess) e = cudaMemcpy(F.data(), s->c.bv.F, F.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(H.data(), s->c.bv.H, H.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&r, drounds, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(drounds);
  pbsam_system_destroy(s);
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("self-polarization: ") + cudaGetErrorString(e));
  for (size_t i = 0; i < F.size(); i++) { fself[i] = round8(F[i]); hself[i] = round8(H[i]); }
  for (int k = 0; k < ns; k++) hself_scale[k] = round8(1.0 / c->types[type_id].rad[k]);
  if (rounds) *rounds = r;
  return PBSAM_OK;
}

extern "C" int pbsam_system_phase_ms(const pbsam_system *s, double *ms)
{
  if (!s || !ms) return fail(PBSAM_E_BADARG, "null argument");
  CK(cudaSetDevice(s->ctx->device));
  CK(cudaMemcpy(ms, s->c.bv.tphase, (size_t)s->B * PH_N * sizeof(double), cudaMemcpyDeviceToHost));
  for (int i = 0; i < s->B * PH_N; i++) ms[i] *= 1e-6;
  return PBSAM_OK;
}

// Brownian dynamics on the force path (uses the helpers above)
#include "pbsam_bd_host.cu"
#include "pbsam_group.cu"

// fixed-buffer variant of the IMat builder (uses the helpers above)
#include "pbsam_static_imat.cu"

// measured device rates for the roofline (uses the helpers above)
#include "pbsam_probe.cu"
#include "pbsam_expan.cu"

// bdm restart configurations (host only): readConfigWithMolType (src/readutil.cpp:835-886)
// and CMolecule::saveConfig (src/molecule.cpp:255-269), one molecule per line,
// "x y z qw qx qy qz type".  The reader takes whitespace-separated fields, eight per
// molecule; a file that ends inside a molecule is refused rather than cut short.
extern "C" int pbsam_config_read(const char *path, int max_mol, int *n_mol, double *pos, double *quat, int *moltype)
{
  if (!path || !n_mol || max_mol < 0) return fail(PBSAM_E_BADARG, "bad argument");
  std::ifstream in(path);
  if (!in) return fail(PBSAM_E_IO, std::string("cannot open configuration ") + path);
  int n = 0;
  double v[7];
  while (in >> v[0]) {
    int t;
    for (int k = 1; k < 7; k++)
      if (!(in >> v[k])) return fail(PBSAM_E_IO, std::string("configuration ends inside a molecule: ") + path);
    if (!(in >> t)) return fail(PBSAM_E_IO, std::string("configuration ends inside a molecule: ") + path);
    if (n < max_mol) {
      if (pos) for (int k = 0; k < 3; k++) pos[3 * n + k] = v[k];
      if (quat) for (int k = 0; k < 4; k++) quat[4 * n + k] = v[3 + k];
      if (moltype) moltype[n] = t;
    }
    n++;
  }
  if (!in.eof()) return fail(PBSAM_E_IO, std::string("configuration has a field that is not a number: ") + path);
  *n_mol = n;
  if (n > max_mol) return fail(PBSAM_E_BADARG, "the configuration holds more molecules than max_mol");
  return PBSAM_OK;
}

extern "C" int pbsam_config_write(const char *path, int n_mol, const double *pos, const double *quat,
                                  const int *moltype)
{
  if (!path || n_mol < 0 || (n_mol > 0 && (!pos || !quat || !moltype))) return fail(PBSAM_E_BADARG, "bad argument");
  FILE *f = std::fopen(path, "w");
  if (!f) return fail(PBSAM_E_IO, std::string("cannot write configuration ") + path);
  for (int i = 0; i < n_mol; i++)
    std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %d\n", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2],
                 quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3], moltype[i]);
  const bool ok = std::fclose(f) == 0;
  return ok ? PBSAM_OK : fail(PBSAM_E_IO, std::string("writing configuration ") + path);
}

extern "C" int pbsam_system_get_forces(pbsam_system *s, double *force, double *torque, int *status, int on_device)
{
  if (!s) return fail(PBSAM_E_BADARG, "null system");
  CK(cudaSetDevice(s->ctx->device));
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t n = (size_t)s->B * s->nmol * 3;
  if (force) CK(cudaMemcpyAsync(force, s->c.bv.force, n * sizeof(double), k, s->stream));
  if (torque) CK(cudaMemcpyAsync(torque, s->c.bv.torque, n * sizeof(double), k, s->stream));
  if (status) CK(cudaMemcpyAsync(status, s->c.bv.status, (size_t)s->B * sizeof(int), k, s->stream));
  if (!on_device) CK(cudaStreamSynchronize(s->stream));
  return PBSAM_OK;
}
