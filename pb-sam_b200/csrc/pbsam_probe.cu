// Device rates measured in place: the FP64 FMA pipe and L2-to-SM read bandwidth.
// The force kernel's IMat rows come from L2 (the IMats stay resident) and its
// arithmetic is FP64 on CUDA cores, so these two are the denominators of its
// roofline; neither is a vendor figure, both are timed here with CUDA events.
// Included by pbsam_api.cu.
namespace pbsam {

// 8 independent FMA chains per thread, n rounds: 16 flops per round per thread
__global__ void __launch_bounds__(512) probe_fp64_kernel(int n, double seed, double *out)
{
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = seed + threadIdx.x * 1e-9 + k;
  const double m = 0.999999999, c = 1e-9;
  for (int i = 0; i < n; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 12345.678) out[0] = s;   // keeps the chains alive; never true in practice
}

// every thread reads 16-byte words of an L2-resident buffer, `reps` passes
__global__ void __launch_bounds__(512) probe_l2_kernel(const double2 *buf, long long n2, int reps, double *out)
{
  double2 acc = make_double2(0.0, 0.0);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int r = 0; r < reps; r++)
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
      const double2 v = __ldcg(buf + i);
      acc.x += v.x;
      acc.y += v.y;
    }
  if (acc.x == 12345.678) out[0] = acc.y;
}

}  // namespace pbsam

// FP64 FMA rate (TFLOP/s) and L2 read bandwidth (GB/s) of a device, each the best of
// three timed launches over every SM
extern "C" int pbsam_device_peaks(int device, double *fp64_tflops, double *l2_gbs)
{
  if (!fp64_tflops || !l2_gbs) return fail(PBSAM_E_BADARG, "null argument");
  CK(cudaSetDevice(device));
  int n_sm = 0;
  CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device));
  const long long bytes = 32LL << 20;    // 32 MB: well inside L2
  double2 *buf = nullptr;
  double *out = nullptr;
  if (cudaMalloc(&buf, bytes) != cudaSuccess) return fail(PBSAM_E_NOMEM, "probe buffer");
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) { cudaFree(buf); return fail(PBSAM_E_NOMEM, "probe"); }
  cudaMemset(buf, 0, bytes);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = n_sm * 4, threads = 512, rounds = 1 << 16, reps = 16;
  float best_f = 1e30f, best_l = 1e30f;
  cudaError_t e = cudaSuccess;
  for (int t = 0; t < 4 && e == cudaSuccess; t++) {
    cudaEventRecord(e0);
    pbsam::probe_fp64_kernel<<<blocks, threads>>>(rounds, 1.0, out);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (t > 0 && ms < best_f) best_f = ms;    // the first launch warms up
    cudaEventRecord(e0);
    pbsam::probe_l2_kernel<<<blocks, threads>>>(buf, bytes / 16, reps, out);
    cudaEventRecord(e1);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (t > 0 && ms < best_l) best_l = ms;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  cudaFree(out);
  if (e != cudaSuccess) return fail(PBSAM_E_CUDA, std::string("device probe: ") + cudaGetErrorString(e));
  *fp64_tflops = 16.0 * rounds * (double)blocks * threads / (best_f * 1e-3) / 1e12;
  *l2_gbs = (double)bytes * reps / (best_l * 1e-3) / 1e9;
  return PBSAM_OK;
}
