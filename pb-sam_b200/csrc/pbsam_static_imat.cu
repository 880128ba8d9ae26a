// IMat builder that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they build a molecule type: hosts
// whose own pool allocator owns all device memory (a second allocator in the
// process would fragment it or fail), and services whose device footprint must be
// fixed once the library is loaded, so that no call can fail for lack of memory
// mid-run.  pbsam_imat_build_static serves them: it runs the same kernels as
// pbsam_imat_build, but its work buffers live in one file-scope device array of
// fixed size instead of memory allocated per call.
//
// Limits: pole order p <= PBSAM_STATIC_IMAT_MAX_POLES (the p^2 x p^2 Gram and IMat
// buffers must fit); the quadrature points stream through the array in chunks of
// PBSAM_STATIC_IMAT_CHUNK, so n_points is not limited by it; at most
// PBSAM_STATIC_IMAT_MAX_NEIGH spheres may overlap any one sphere.
//
// The array is shared by every call in the process on that device and keeps what
// the last call left in it: each call clears the Gram accumulators it sums into
// before use, and everything else is written before it is read.  Two calls whose
// work overlaps on the GPU (different host threads, or different streams) race on
// the array; callers serialise them.
//
// Included at the end of pbsam_api.cu (one translation unit).
namespace pbsam {

#define PBSAM_STATIC_IMAT_MAX_POLES 16
#define PBSAM_STATIC_IMAT_CHUNK 1024
#define PBSAM_STATIC_IMAT_MAX_NEIGH 256

// layout: [Gram N*N][IMat N*N][Simpson Gram P*P][harmonics CHUNK*N][points CHUNK*3], N = P^2
#define PBSAM_STATIC_IMAT_NMAX (PBSAM_STATIC_IMAT_MAX_POLES * PBSAM_STATIC_IMAT_MAX_POLES)
#define PBSAM_STATIC_IMAT_DOUBLES                                                                              \
  (2 * PBSAM_STATIC_IMAT_NMAX * PBSAM_STATIC_IMAT_NMAX + PBSAM_STATIC_IMAT_MAX_POLES * PBSAM_STATIC_IMAT_MAX_POLES + \
   PBSAM_STATIC_IMAT_CHUNK * PBSAM_STATIC_IMAT_NMAX + PBSAM_STATIC_IMAT_CHUNK * 3)

// 3.2 MB per device that loads the library, held until the process exits
static __device__ __align__(256) double g_static_imat_scratch[PBSAM_STATIC_IMAT_DOUBLES];

// device address of the array, looked up on the first call on each device with
// that device current (host code cannot use the symbol's name as a device pointer)
// and kept for the life of the process; the lookup is guarded so that host threads
// making their first calls at once do not race on the cache.  A cudaDeviceReset of a
// device invalidates the kept address together with every other handle of this
// library on that device.
static double *g_static_imat_ptr[64];
static std::mutex g_static_imat_mu;

static int static_imat_scratch(int device, double **out)
{
  if (device < 0 || device >= 64) return fail(PBSAM_E_BADARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_static_imat_mu);
  if (!g_static_imat_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_imat_scratch);
    if (e != cudaSuccess || !p)
      return fail(PBSAM_E_CUDA, std::string("static IMat scratch address: ") + cudaGetErrorString(e));
    g_static_imat_ptr[device] = (double *)p;
  }
  *out = g_static_imat_ptr[device];
  return PBSAM_OK;
}

}  // namespace pbsam

// unit-sphere spiral point i (1-based) of n, continuing from the previous angle
// (src/molecule.cpp:2272-2294), the same arithmetic as pbsam_imat_build
static inline void static_imat_spiral(int i, int n, double &phprev, double &x, double &y, double &z)
{
  const double h = -1.0 + 2.0 * (i - 1.0) / (n - 1.0);
  const double th = acos(h);
  double ph = (i == 1 || i == n) ? 0 : (phprev + 3.6 / sqrt(n * (1.0 - h * h)));
  while (ph > 2 * M_PI) ph -= 2 * M_PI;
  while (ph < -2 * M_PI) ph += 2 * M_PI;
  phprev = ph;
  x = 1 * sin(th) * cos(ph); y = 1 * sin(th) * sin(ph); z = 1 * cos(th);
}

extern "C" int pbsam_imat_build_static(pbsam_context *c, int n_sph, const double *centres, const double *radii,
                                       int n_points, double *imats)
{
  using namespace pbsam;
  if (!c || n_sph <= 0 || !centres || !radii || n_points < 3 || !imats) return fail(PBSAM_E_BADARG, "bad argument");
  const int P = c->prm.poles, N = P * P;
  if (P > PBSAM_STATIC_IMAT_MAX_POLES)
    return fail(PBSAM_E_BADARG, "pbsam_imat_build_static: pole order " + std::to_string(P) + " exceeds the maximum " +
                                    std::to_string(PBSAM_STATIC_IMAT_MAX_POLES) +
                                    " of its fixed device buffer; use pbsam_imat_build");
  CK(cudaSetDevice(c->device));
  // the first call on a device looks up the array's device address (set-up)
  double *base = nullptr;
  {
    const int r = static_imat_scratch(c->device, &base);
    if (r) return r;
  }
  double *dG = base, *dIM = dG + (size_t)N * N, *dGs = dIM + (size_t)N * N, *dY = dGs + (size_t)P * P;
  double *dP = dY + (size_t)PBSAM_STATIC_IMAT_CHUNK * N;
  // molecule-centred coordinates as the reference prepares them
  double rc[3] = {0, 0, 0};
  for (int k = 0; k < n_sph; k++) for (int d = 0; d < 3; d++) rc[d] += centres[3 * k + d];
  const double inv = 1.0 / n_sph;
  for (int d = 0; d < 3; d++) rc[d] *= inv;
  const double dA = 4 * M_PI / (double)(n_points - 1);
  double chunk[PBSAM_STATIC_IMAT_CHUNK * 3];
  int neigh[PBSAM_STATIC_IMAT_MAX_NEIGH];
  for (int k = 0; k < n_sph; k++) {
    int nn = 0;
    for (int j = 0; j < n_sph; j++) {
      if (j == k) continue;
      const double sr = radii[k] + radii[j];
      const double dx = centres[3 * k] - centres[3 * j], dy = centres[3 * k + 1] - centres[3 * j + 1],
                   dz = centres[3 * k + 2] - centres[3 * j + 2];
      if (dx * dx + dy * dy + dz * dz < sr * sr) {
        if (nn == PBSAM_STATIC_IMAT_MAX_NEIGH)
          return fail(PBSAM_E_BADARG, "pbsam_imat_build_static: more than " +
                                          std::to_string(PBSAM_STATIC_IMAT_MAX_NEIGH) + " overlapping spheres");
        neigh[nn++] = j;
      }
    }
    // point on sphere k buried inside an overlapping neighbour?
    const double ckx = centres[3 * k] - rc[0], cky = centres[3 * k + 1] - rc[1], ckz = centres[3 * k + 2] - rc[2];
    auto buried_pt = [&](double px, double py, double pz) {
      for (int q = 0; q < nn; q++) {
        const int j = neigh[q];
        const double cjx = centres[3 * j] - rc[0], cjy = centres[3 * j + 1] - rc[1], cjz = centres[3 * j + 2] - rc[2];
        const double dx = (px + ckx) - cjx, dy = (py + cky) - cjy, dz = (pz + ckz) - cjz;
        if (dx * dx + dy * dy + dz * dz < radii[j] * radii[j] * 1.0) return true;
      }
      return false;
    };
    // first pass: count exposed and buried points (the smaller set is integrated)
    int npe = 0, npb = 0;
    {
      double phprev = 0, x, y, z;
      for (int i = 1; i <= n_points; i++) {
        static_imat_spiral(i, n_points, phprev, x, y, z);
        if (buried_pt(radii[k] * x, radii[k] * y, radii[k] * z)) npb++;
        else npe++;
      }
    }
    const int buried = (npe <= npb) ? 0 : 1;
    CK(cudaMemset(dG, 0, (size_t)N * N * sizeof(double)));
    CK(cudaMemset(dGs, 0, (size_t)P * P * sizeof(double)));
    // second pass: stream the chosen set through the fixed buffers
    double phprev = 0, x, y, z;
    int h0 = 0, kc = 0;
    auto flush = [&]() -> int {
      if (kc == 0) return PBSAM_OK;
      CK(cudaMemcpy(dP, chunk, (size_t)kc * 3 * sizeof(double), cudaMemcpyHostToDevice));
      imat_sh_kernel<<<(kc + 127) / 128, 128>>>(c->T, dP, kc, P, dY);
      dim3 g((N + GT - 1) / GT, (N + GT - 1) / GT);
      gram_kernel<<<g, 256>>>(dY, kc, N, dG);
      gram_simpson_kernel<<<(P * P + 127) / 128, 128>>>(dY, kc, P, h0, dGs);
      CK(cudaGetLastError());
      h0 += kc;
      kc = 0;
      return PBSAM_OK;
    };
    for (int i = 1; i <= n_points; i++) {
      static_imat_spiral(i, n_points, phprev, x, y, z);
      const double px = radii[k] * x, py = radii[k] * y, pz = radii[k] * z;
      if (buried_pt(px, py, pz) != (buried != 0)) continue;
      chunk[3 * kc] = px; chunk[3 * kc + 1] = py; chunk[3 * kc + 2] = pz;
      if (++kc == PBSAM_STATIC_IMAT_CHUNK) {
        const int r = flush();
        if (r) return r;
      }
    }
    {
      const int r = flush();
      if (r) return r;
    }
    const long long tot = (long long)N * N;
    imat_assemble_kernel<<<(unsigned)((tot + 255) / 256), 256>>>(c->T, dG, dGs, P, dA, buried, dIM);
    CK(cudaGetLastError());
    CK(cudaMemcpy(imats + (size_t)k * N * N, dIM, (size_t)N * N * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return PBSAM_OK;
}
