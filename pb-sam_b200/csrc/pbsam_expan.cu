// Single-expansion operations, batched: the rotation, coaxial translation and pair
// re-expansion of the reference's CRotCoeff (src/rotcoeff.h:10-266), CTransCoeff
// (src/transcoeff.h:9-182) and CXFormA (src/xforms.h:58-104), for callers that drive
// expansions one by one (the C++ classes of pb-sam_b200/cpp/pbsam_b200.hpp).  One CTA
// per item, each with its own scratch block; the same device routines as the force
// kernel.  Included by pbsam_api.cu.
namespace pbsam {

enum { EXPAN_ROTATE = 0, EXPAN_TRANSLATE = 1, EXPAN_REEXPAND = 2 };

// Item i0 + blockIdx.x of a batch.  args per item: rotate (theta, phi, xi), translate
// (rho, scale_in, scale_out), re-expand (P = c_tgt - c_src, scale_src, scale_tgt).
// f1, f2: rotate (with_xi, forward), translate (screened, deriv), re-expand (screened, -).
__global__ void __launch_bounds__(PBSAM_TEAM) pbsam_expan_kernel(Tab T, int op, int i0, int n, const double *args,
                                                                 int p, int f1, int f2, const double *in, double *out,
                                                                 double *grad, double *scr, long long stride)
{
  extern __shared__ double2 dsm[];
  const Team tm{(int)threadIdx.x, (int)blockDim.x};
  const int i = i0 + blockIdx.x;
  if (i >= n) return;
  const int NP = T.NP, NP2 = NP * NP;
  Scr sc = make_scr(scr + (size_t)blockIdx.x * stride, NP, dsm);
  const double *x = in + (size_t)i * NP2;
  double *y = out + (size_t)i * NP2;
  if (op == EXPAN_ROTATE) {
    const double *a = args + 3 * (size_t)i;
    RotState rs;
    rot_compute(tm, T, a[0], a[1], a[2], p, false, rs, sc.R, nullptr, sc.sh, sc.lvA, sc.lvB);
    tm.sync();
    if (f1) rot_apply_xi(tm, rs, x, y, p, f2 != 0, NP);
    else rot_apply(tm, rs, x, y, p, f2 != 0, NP);
    tm.sync();
  } else if (op == EXPAN_TRANSLATE) {
    const double *a = args + 3 * (size_t)i;
    TransState ts;
    trans_compute(tm, T, a[0], f1 ? T.kappa : 0.0, p, a[1], a[2], f2 != 0, ts, sc.TH, sc.dTH, sc.kbuf);
    if (tm.rank == 0) {
      sc.fact[0] = 1.0;
      for (int k = 1; k < NP; k++) sc.fact[k] = sc.fact[k - 1] * (a[2] / a[1]);
    }
    tm.sync();
    for (int k = tm.rank; k < NP2; k += tm.size) y[k] = 0.0;
    tm.sync();
    trans_apply(tm, ts, sc.fact, x, y, f2 != 0, p);
    tm.sync();
  } else {
    const double *a = args + 5 * (size_t)i;
    PairXf X;
    prep_pair(tm, T, sc, a, p, f1 ? 0 : p, a[3], a[4], grad != nullptr && f1, X);
    pair_apply(tm, T, sc, X, !f1, x, y);
    if (grad && f1) pair_apply_grad(tm, T, sc, X, x, grad + (size_t)i * 3 * NP2);
  }
}

}  // namespace pbsam

// one batch of single-expansion operations: n items in waves of at most CH CTAs
static int expan_batch(pbsam_context *c, int op, int n, const double *args, int nargs, int p, int f1, int f2,
                       const double *in, double *out, double *grad, int on_device)
{
  if (!c || n < 0 || !args || !in || !out) return fail(PBSAM_E_BADARG, "null argument");
  if (n == 0) return PBSAM_OK;
  const int NP = c->prm.poles, NP2 = NP * NP;
  if (p < 1 || p > NP) return fail(PBSAM_E_BADARG, "order p must be in 1..poles");
  for (long long k = 0; !on_device && k < (long long)n * nargs; k++)
    if (!std::isfinite(args[k])) return fail(PBSAM_E_BADARG, "non-finite transform argument");
  CK(cudaSetDevice(c->device));
  TRY(set_smem_attrs(NP));
  CK(cudaFuncSetAttribute(pbsam::pbsam_expan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)team_smem_bytes(NP)));
  std::vector<void *> tmp;
  auto release = [&]() { for (void *q : tmp) cudaFree(q); };
  const double *da = args, *dx = in;
  double *dy = out, *dg = grad;
  int r = 0;
  if (!on_device) {
    double *a = nullptr, *x = nullptr, *y = nullptr, *g = nullptr;
    r = dalloc(tmp, &a, (size_t)n * nargs);
    if (!r) r = dalloc(tmp, &x, (size_t)n * NP2);
    if (!r) r = dalloc(tmp, &y, (size_t)n * NP2);
    if (!r && grad) r = dalloc(tmp, &g, (size_t)n * 3 * NP2);
    if (r) { release(); return r; }
    cudaError_t e = cudaMemcpy(a, args, (size_t)n * nargs * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(x, in, (size_t)n * NP2 * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { release(); return fail(PBSAM_E_CUDA, cudaGetErrorString(e)); }
    da = a; dx = x; dy = y; dg = g;
  }
  const int CH = 148;
  const long long stride = scr_doubles(NP, 1);
  double *scr = nullptr;
  r = dalloc(tmp, &scr, (size_t)stride * CH);
  if (r) { release(); return r; }
  cudaError_t e = cudaSuccess;
  for (int i0 = 0; e == cudaSuccess && i0 < n; i0 += CH) {
    const int nb = n - i0 < CH ? n - i0 : CH;
    pbsam::pbsam_expan_kernel<<<nb, PBSAM_TEAM, team_smem_bytes(NP)>>>(c->T, op, i0, n, da, p, f1, f2, dx, dy, dg,
                                                                         scr, stride);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess && !on_device) {
    e = cudaMemcpy(out, dy, (size_t)n * NP2 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && grad) e = cudaMemcpy(grad, dg, (size_t)n * 3 * NP2 * sizeof(double), cudaMemcpyDeviceToHost);
  }
  release();
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("expansion batch: ") + cudaGetErrorString(e));
  return PBSAM_OK;
}

extern "C" int pbsam_expan_rotate(pbsam_context *c, int n, const double *rot, int p, int with_xi, int forward,
                                  const double *in, double *out, int on_device)
{
  return expan_batch(c, pbsam::EXPAN_ROTATE, n, rot, 3, p, with_xi != 0, forward != 0, in, out, nullptr, on_device);
}

extern "C" int pbsam_expan_translate(pbsam_context *c, int n, const double *args, int p, int screened, int deriv,
                                     const double *in, double *out, int on_device)
{
  if (!on_device && args)
    for (int i = 0; i < n; i++)
      if (!(args[3 * i] > 0.0 && args[3 * i + 1] > 0.0 && args[3 * i + 2] > 0.0))
        return fail(PBSAM_E_BADARG, "translation distance and scales must be positive");
  return expan_batch(c, pbsam::EXPAN_TRANSLATE, n, args, 3, p, screened != 0, deriv != 0, in, out, nullptr, on_device);
}

extern "C" int pbsam_expan_reexpand(pbsam_context *c, int n, const double *args, int p, int screened,
                                    const double *in, double *out, double *grad, int on_device)
{
  if (grad && !screened) return fail(PBSAM_E_BADARG, "the gradient is that of the screened (H) re-expansion");
  if (!on_device && args)
    for (int i = 0; i < n; i++) {
      const double *a = args + 5 * (size_t)i;
      if (!(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] > 0.0) || !(a[3] > 0.0 && a[4] > 0.0))
        return fail(PBSAM_E_BADARG, "re-expansion needs distinct centres and positive scales");
    }
  return expan_batch(c, pbsam::EXPAN_REEXPAND, n, args, 5, p, screened != 0, 0, in, out, grad, on_device);
}

extern "C" int pbsam_quat_angles(const double *q, double *angles)
{
  if (!q || !angles) return fail(PBSAM_E_BADARG, "null argument");
  const double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(n > 0.0) || !std::isfinite(n)) return fail(PBSAM_E_BADARG, "zero or non-finite quaternion");
  const double qn[4] = {q[0] / n, q[1] / n, q[2] / n, q[3] / n};
  pbsam::quat_angles(qn, angles[0], angles[1], angles[2]);
  return PBSAM_OK;
}
