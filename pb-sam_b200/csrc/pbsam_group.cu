// Groups of system handles: the systems of several handles, each with its own molecule
// list (sphere counts) and possibly its own context (pole order), evaluated in one
// launch, one CTA per system, in an order the group keeps: initially by the square of
// the sphere count, after pbsam_group_tune by the device time of each system's last
// evaluation, longest first, so that the longest systems start first and the short
// ones fill in behind them.  BD steps of every trajectory of every handle are one CUDA
// graph per step (group kernels for the time step, forces and moves).  Included at the
// end of pbsam_api.cu.

struct pbsam_group {
  std::vector<pbsam_system *> sys;
  int device = 0;
  int n_work = 0;
  std::vector<int2> order;              // (handle, system), in launch order
  int2 *d_work = nullptr;
  Ctx *d_ctx = nullptr;                 // per handle: its context view (forces)
  Ctx *d_ctx_bd = nullptr;              // the same with the BD force mask
  BDParams *d_bdp = nullptr;
  BDView *d_bdv = nullptr;
  size_t smem = 0, move_smem = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static void group_release(pbsam_group *g)
{
  if (g->st) cudaStreamSynchronize(g->st);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (void *p : {(void *)g->d_work, (void *)g->d_ctx, (void *)g->d_ctx_bd, (void *)g->d_bdp, (void *)g->d_bdv})
    if (p) cudaFree(p);
  if (g->ev) cudaEventDestroy(g->ev);
  if (g->st) cudaStreamDestroy(g->st);
  delete g;
}

// wait for the handles' queued work (their streams and BD streams), on the host
static int group_join_in(pbsam_group *g)
{
  for (pbsam_system *s : g->sys) {
    CK(cudaStreamSynchronize(s->stream));
    if (s->bd) CK(cudaStreamSynchronize(s->bd->st));
  }
  return PBSAM_OK;
}
// later work on every handle's stream follows the group's
static int group_join_out(pbsam_group *g)
{
  CK(cudaEventRecord(g->ev, g->st));
  for (pbsam_system *s : g->sys) CK(cudaStreamWaitEvent(s->stream, g->ev, 0));
  return PBSAM_OK;
}

static int group_upload_order(pbsam_group *g)
{
  CK(cudaMemcpy(g->d_work, g->order.data(), g->order.size() * sizeof(int2), cudaMemcpyHostToDevice));
  return PBSAM_OK;
}

extern "C" int pbsam_group_create(int n, pbsam_system *const *systems, pbsam_group **out)
{
  if (n <= 0 || !systems || !out) return fail(PBSAM_E_BADARG, "bad argument");
  for (int i = 0; i < n; i++) {
    if (!systems[i]) return fail(PBSAM_E_BADARG, "null system");
    if (systems[i]->ctx->device != systems[0]->ctx->device) return fail(PBSAM_E_BADARG, "systems on different devices");
    for (int j = 0; j < i; j++)
      if (systems[j] == systems[i]) return fail(PBSAM_E_BADARG, "a system appears twice");
  }
  pbsam_group *g = new pbsam_group();
  g->sys.assign(systems, systems + n);
  g->device = systems[0]->ctx->device;
  auto bail = [&](int rc) { group_release(g); return rc; };
  if (cudaSetDevice(g->device) != cudaSuccess) return bail(fail(PBSAM_E_CUDA, "cudaSetDevice"));
  // static order: systems of larger molecule lists first (cost about S^2)
  std::vector<std::pair<long long, int2>> w;
  for (int i = 0; i < n; i++) {
    const long long S = systems[i]->c.bv.S;
    for (int b = 0; b < systems[i]->B; b++) w.push_back({-S * S, make_int2(i, b)});
  }
  std::stable_sort(w.begin(), w.end(), [](const std::pair<long long, int2> &a, const std::pair<long long, int2> &b) {
    return a.first < b.first;
  });
  for (auto &x : w) g->order.push_back(x.second);
  g->n_work = (int)g->order.size();
  for (pbsam_system *s : g->sys) g->smem = std::max(g->smem, forces_smem_bytes(s->ctx->prm.poles));
  std::vector<Ctx> hc;
  for (pbsam_system *s : g->sys) hc.push_back(s->c);
  if (cudaMalloc(&g->d_work, g->order.size() * sizeof(int2)) != cudaSuccess ||
      cudaMalloc(&g->d_ctx, n * sizeof(Ctx)) != cudaSuccess || cudaMalloc(&g->d_ctx_bd, n * sizeof(Ctx)) != cudaSuccess ||
      cudaMalloc(&g->d_bdp, n * sizeof(BDParams)) != cudaSuccess || cudaMalloc(&g->d_bdv, n * sizeof(BDView)) != cudaSuccess)
    return bail(fail(PBSAM_E_NOMEM, "group buffers"));
  if (cudaMemcpy(g->d_ctx, hc.data(), n * sizeof(Ctx), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(PBSAM_E_CUDA, "group context copy"));
  if (group_upload_order(g)) return bail(PBSAM_E_CUDA);
  if (cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(PBSAM_E_CUDA, "group stream"));
  if (cudaFuncSetAttribute(pbsam_forces_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g->smem) !=
      cudaSuccess)
    return bail(fail(PBSAM_E_CUDA, "group kernel shared memory"));
  *out = g;
  return PBSAM_OK;
}

extern "C" int pbsam_group_destroy(pbsam_group *g)
{
  if (!g) return PBSAM_OK;
  CK(cudaSetDevice(g->device));
  group_release(g);
  return PBSAM_OK;
}

extern "C" int pbsam_group_compute_forces(pbsam_group *g)
{
  if (!g) return fail(PBSAM_E_BADARG, "null group");
  CK(cudaSetDevice(g->device));
  TRY(group_join_in(g));
  pbsam_forces_group_kernel<<<g->n_work, PBSAM_TEAM, g->smem, g->st>>>(g->d_ctx, g->d_work);
  CK(cudaGetLastError());
  TRY(group_join_out(g));
  CK(cudaStreamSynchronize(g->st));
  return PBSAM_OK;
}

// the scheduler: the device time of each system's last evaluation (its phase timer),
// longest first; systems never evaluated keep their place behind the timed ones
extern "C" int pbsam_group_tune(pbsam_group *g)
{
  if (!g) return fail(PBSAM_E_BADARG, "null group");
  CK(cudaSetDevice(g->device));
  TRY(group_join_in(g));
  std::vector<std::pair<double, int2>> w;
  for (int i = 0; i < (int)g->sys.size(); i++) {
    pbsam_system *s = g->sys[i];
    std::vector<double> ph((size_t)s->B * PH_N);
    CK(cudaMemcpy(ph.data(), s->c.bv.tphase, ph.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int b = 0; b < s->B; b++) w.push_back({-ph[(size_t)b * PH_N + PH_TOTAL], make_int2(i, b)});
  }
  std::stable_sort(w.begin(), w.end(), [](const std::pair<double, int2> &a, const std::pair<double, int2> &b) {
    return a.first < b.first;
  });
  for (size_t k = 0; k < w.size(); k++) g->order[k] = w[k].second;
  return group_upload_order(g);
}

static cudaError_t group_bd_enqueue(pbsam_group *g, cudaStream_t st)
{
  pbsam_bd_pre_group_kernel<<<g->n_work, PBSAM_BD_THREADS, 0, st>>>(g->d_ctx_bd, g->d_bdp, g->d_bdv, g->d_work);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  pbsam_forces_group_kernel<<<g->n_work, PBSAM_TEAM, g->smem, st>>>(g->d_ctx_bd, g->d_work);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  pbsam_bd_move_group_kernel<<<g->n_work, PBSAM_BD_THREADS, g->move_smem, st>>>(g->d_ctx_bd, g->d_bdp, g->d_bdv,
                                                                               g->d_work);
  return cudaGetLastError();
}

extern "C" int pbsam_group_bd_run(pbsam_group *g, int n_steps)
{
  if (!g || n_steps < 0) return fail(PBSAM_E_BADARG, "bad argument");
  CK(cudaSetDevice(g->device));
  const int n = (int)g->sys.size();
  std::vector<Ctx> hc;
  std::vector<BDParams> hp;
  std::vector<BDView> hv;
  size_t ms = 0;
  for (pbsam_system *s : g->sys) {
    if (!s->bd) return fail(PBSAM_E_STATE, "every system of the group needs pbsam_system_bd_init");
    Ctx c = s->c;
    c.bv.fmask = s->bd->v.need;
    hc.push_back(c);
    hp.push_back(s->bd->p);
    hv.push_back(s->bd->v);
    ms = std::max(ms, s->bd->move_smem);
  }
  if (n_steps == 0) return PBSAM_OK;
  TRY(group_join_in(g));
  // the views as they are now (contact lists may have been set since the last run)
  CK(cudaMemcpy(g->d_ctx_bd, hc.data(), n * sizeof(Ctx), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g->d_bdp, hp.data(), n * sizeof(BDParams), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g->d_bdv, hv.data(), n * sizeof(BDView), cudaMemcpyHostToDevice));
  if (ms > g->move_smem || !g->exec) {
    if (ms > 48 * 1024)
      CK(cudaFuncSetAttribute(pbsam_bd_move_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms));
    g->move_smem = std::max(g->move_smem, ms);
    if (g->exec) { cudaGraphExecDestroy(g->exec); g->exec = nullptr; }
    if (g->graph) { cudaGraphDestroy(g->graph); g->graph = nullptr; }
    CK(cudaStreamBeginCapture(g->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = group_bd_enqueue(g, g->st);
    cudaGraph_t gr = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(g->st, &gr);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (gr) cudaGraphDestroy(gr);
      return fail(PBSAM_E_CUDA, std::string("group BD step capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    g->graph = gr;
    CK(cudaGraphInstantiate(&g->exec, gr, 0));
  }
  for (int k = 0; k < n_steps; k++) CK(cudaGraphLaunch(g->exec, g->st));
  TRY(group_join_out(g));
  return PBSAM_OK;
}
