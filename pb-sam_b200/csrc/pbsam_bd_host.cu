// Host side of the Brownian-dynamics entry points (include/pbsam_b200.h):
// device state of the trajectories, one step as three launches, and the CUDA
// graph that replays a step.  Included at the end of pbsam_api.cu.

struct BDHost {
  BDParams p;
  BDView v;
  std::vector<void *> bufs;
  int use_graph = 0;
  size_t move_smem = 0;
  cudaStream_t st = nullptr;            // stream the steps (and the graph) run on
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

static void bd_free(pbsam_system *s)
{
  BDHost *h = s->bd;
  if (!h) return;
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->ev_in) cudaEventDestroy(h->ev_in);
  if (h->ev_out) cudaEventDestroy(h->ev_out);
  if (h->st) cudaStreamDestroy(h->st);
  for (void *p : h->bufs) cudaFree(p);
  delete h;
  s->bd = nullptr;
}

extern "C" void pbsam_bd_params_default(int mode, pbsam_bd_params *p)
{
  p->mode = mode;
  p->max_tries = 500;                       // maxc, src/BDnam.cpp:270, src/BDmulti.cpp:451
  p->force_dist = 100.0;                    // f_DIST, src/BDnam.h:25
  p->escape_dist = 500.0;                   // q_DIST, src/BDnam.h:24
  p->dt_min = 2.0;                          // src/BDnam.cpp:409-417, src/BDmulti.cpp:511-517
  p->dt_max = 1e300;
  p->dt_ref = mode == PBSAM_BD_MULTI ? 10.0 : 5.0;   // DISTCUTOFF_TIME (src/BDmulti.cpp:13) / 5 A
  p->dt_div = 15.0;
  p->fact_tr = 5.604586e2;                  // FACT2, src/BDnam.h:10
  p->ikbt = 1.0 / (1.3806503e-23 * 298.15); // IKbT, src/BDnam.h:18
  p->coul_k = 2.30708e-18;                  // COUL_K, src/BDnam.h:19
  p->seed = 0;
  p->use_graph = 1;
  p->noise = PBSAM_BD_NOISE_PHILOX;
}

extern "C" int pbsam_system_bd_init(pbsam_system *s, const pbsam_bd_params *prm, const double *dtr, const double *drot)
{
  if (!s || !prm || !dtr || !drot) return fail(PBSAM_E_BADARG, "null argument");
  if (prm->mode != PBSAM_BD_NAM && prm->mode != PBSAM_BD_MULTI) return fail(PBSAM_E_BADARG, "bad BD mode");
  if (prm->mode == PBSAM_BD_NAM && s->nmol != 2) return fail(PBSAM_E_BADARG, "NAM dynamics needs two molecules");
  if (prm->max_tries < 1 || prm->max_tries > 1000000) return fail(PBSAM_E_BADARG, "max_tries out of range");
  if (!(prm->dt_min > 0) || !(prm->dt_div > 0) || !(prm->dt_max >= prm->dt_min))
    return fail(PBSAM_E_BADARG, "bad time-step schedule");
  for (int i = 0; i < s->nmol; i++)
    if (!(dtr[i] >= 0) || !(drot[i] >= 0)) return fail(PBSAM_E_BADARG, "negative diffusion coefficient");
  CK(cudaSetDevice(s->ctx->device));
  if (s->bd) {
    CK(cudaStreamSynchronize(s->bd->st));
    bd_free(s);
  }
  BDHost *h = new BDHost();
  s->bd = h;
  BDParams &p = h->p;
  p.mode = prm->mode; p.max_tries = prm->max_tries;
  p.force_dist = prm->force_dist; p.escape_dist = prm->escape_dist;
  p.dt_min = prm->dt_min; p.dt_max = prm->dt_max; p.dt_ref = prm->dt_ref; p.dt_div = prm->dt_div;
  p.fact_tr = prm->fact_tr; p.ikbt = prm->ikbt; p.coul_k = prm->coul_k;
  p.interact_cut = s->ctx->prm.interact_cutoff;
  p.seed = prm->seed;
  if (prm->noise != PBSAM_BD_NOISE_PHILOX && prm->noise != PBSAM_BD_NOISE_DRAND48) {
    bd_free(s);
    return fail(PBSAM_E_BADARG, "bad noise kind");
  }
  p.noise = prm->noise;
  h->use_graph = prm->use_graph;
  const size_t B = s->B, nm = s->nmol, S = s->c.bv.S;
  BDView &v = h->v;
  int r = 0;
  auto chk = [&](int rr) { if (rr && !r) r = rr; };
  chk(dalloc(h->bufs, &v.status, B)); chk(dalloc(h->bufs, &v.steps, B)); chk(dalloc(h->bufs, &v.fevals, B));
  chk(dalloc(h->bufs, &v.time, B)); chk(dalloc(h->bufs, &v.dt, B)); chk(dalloc(h->bufs, &v.ctr, B));
  chk(dalloc(h->bufs, &v.lcg, B)); chk(dalloc(h->bufs, &v.nr_val, B)); chk(dalloc(h->bufs, &v.nr_saved, B));
  chk(dalloc(h->bufs, &v.rot, B * nm * 4)); chk(dalloc(h->bufs, &v.need, B)); chk(dalloc(h->bufs, &v.cen, B * S * 3));
  std::vector<double> hd(dtr, dtr + nm), hr(drot, drot + nm);
  chk(dput(h->bufs, &v.dtr, hd)); chk(dput(h->bufs, &v.drot, hr));
  if (r) { bd_free(s); return r; }
  v.pos = const_cast<double *>(s->c.bv.pos);
  v.quat = const_cast<double *>(s->c.bv.quat);
  int max_ns = 1;
  for (int i = 0; i < s->nmol; i++) {
    int lo = 0, hi = 0;
    CK(cudaMemcpy(&lo, s->c.bv.mol_off + i, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&hi, s->c.bv.mol_off + i + 1, sizeof(int), cudaMemcpyDeviceToHost));
    max_ns = std::max(max_ns, hi - lo);
  }
  h->move_smem = (size_t)max_ns * 3 * sizeof(double);
  if (h->move_smem > 48 * 1024)
    CK(cudaFuncSetAttribute(pbsam_bd_move_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->move_smem));
  CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming));
  // start after the work already queued on the system's stream (poses set by the caller)
  CK(cudaEventRecord(h->ev_in, s->stream));
  CK(cudaStreamWaitEvent(h->st, h->ev_in, 0));
  pbsam_bd_init_kernel<<<s->B, 32, 0, h->st>>>(s->c, p, v);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->st));
  return PBSAM_OK;
}

// one step: time step and force mask, forces of the systems that need them, move
static cudaError_t bd_enqueue_step(pbsam_system *s, cudaStream_t st)
{
  BDHost *h = s->bd;
  Ctx cb = s->c;
  cb.bv.fmask = h->v.need;
  pbsam_bd_pre_kernel<<<s->B, PBSAM_BD_THREADS, 0, st>>>(s->c, h->p, h->v);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = launch_crews(pbsam_forces_kernel, s->B, s->crew, forces_smem_bytes(s->ctx->prm.poles), st, cb,
                   (const int *)nullptr);
  if (e != cudaSuccess) return e;
  pbsam_bd_move_kernel<<<s->B, PBSAM_BD_THREADS, h->move_smem, st>>>(s->c, h->p, h->v);
  return cudaGetLastError();
}

extern "C" int pbsam_system_bd_run(pbsam_system *s, int n_steps)
{
  if (!s || n_steps < 0) return fail(PBSAM_E_BADARG, "bad argument");
  BDHost *h = s->bd;
  if (!h) return fail(PBSAM_E_STATE, "pbsam_system_bd_init has not been called");
  CK(cudaSetDevice(s->ctx->device));
  if (n_steps == 0) return PBSAM_OK;
  CK(cudaEventRecord(h->ev_in, s->stream));
  CK(cudaStreamWaitEvent(h->st, h->ev_in, 0));
  if (h->use_graph && !h->exec) {
    CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = bd_enqueue_step(s, h->st);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(h->st, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return fail(PBSAM_E_CUDA, std::string("BD step capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    h->graph = g;
    CK(cudaGraphInstantiate(&h->exec, g, 0));
  }
  for (int k = 0; k < n_steps; k++) {
    if (h->use_graph) CK(cudaGraphLaunch(h->exec, h->st));
    else CK(bd_enqueue_step(s, h->st));
  }
  // later work on the system's stream sees the moved poses
  CK(cudaEventRecord(h->ev_out, h->st));
  CK(cudaStreamWaitEvent(s->stream, h->ev_out, 0));
  return PBSAM_OK;
}

extern "C" int pbsam_system_bd_set_contacts(pbsam_system *s, int n_defs, const int *partner, const int *ncontact,
                                            const int *off, const int *k1, const int *k2, const double *dist)
{
  if (!s) return fail(PBSAM_E_BADARG, "null system");
  BDHost *h = s->bd;
  if (!h) return fail(PBSAM_E_STATE, "pbsam_system_bd_init has not been called");
  if (h->p.mode != PBSAM_BD_NAM) return fail(PBSAM_E_BADARG, "docking contacts belong to NAM dynamics");
  if (n_defs < 0 || (n_defs > 0 && (!partner || !ncontact || !off || off[0] != 0)))
    return fail(PBSAM_E_BADARG, "bad contact definitions");
  CK(cudaSetDevice(s->ctx->device));
  int mo[3] = {0, 0, 0};
  CK(cudaMemcpy(mo, s->c.bv.mol_off, 3 * sizeof(int), cudaMemcpyDeviceToHost));
  const int n0 = mo[1] - mo[0], n1 = mo[2] - mo[1];
  for (int d = 0; d < n_defs; d++)
    if (off[d + 1] < off[d]) return fail(PBSAM_E_BADARG, "contact offsets must not decrease");
  const int np = n_defs > 0 ? off[n_defs] : 0;
  if (np > 0 && (!k1 || !k2 || !dist)) return fail(PBSAM_E_BADARG, "null contact pairs");
  for (int e = 0; e < np; e++) {
    if (k1[e] < 0 || k1[e] >= n0 || k2[e] < 0 || k2[e] >= n1)
      return fail(PBSAM_E_BADARG, "a contact names a sphere the molecule does not have");
    if (!std::isfinite(dist[e])) return fail(PBSAM_E_BADARG, "non-finite contact distance");
  }
  CK(cudaStreamSynchronize(h->st));
  BDView &v = h->v;
  v.n_dock = 0;
  if (n_defs > 0) {
    std::vector<int> hp(partner, partner + n_defs), hn(ncontact, ncontact + n_defs), ho(off, off + n_defs + 1);
    std::vector<int> h1(k1, k1 + np), h2(k2, k2 + np);
    std::vector<double> hd(dist, dist + np);
    TRY(dput(h->bufs, &v.dock_partner, hp));
    TRY(dput(h->bufs, &v.dock_ncon, hn));
    TRY(dput(h->bufs, &v.dock_off, ho));
    TRY(dput(h->bufs, &v.dock_k1, h1));
    TRY(dput(h->bufs, &v.dock_k2, h2));
    TRY(dput(h->bufs, &v.dock_dist, hd));
    v.n_dock = n_defs;
  }
  // the step graph holds the view it was captured with: capture again at the next run
  if (h->exec) { cudaGraphExecDestroy(h->exec); h->exec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  return PBSAM_OK;
}

// contactdef reader (CMolContact::readMolContact, src/contact.cpp:53-97, and
// readMolContactWithDist, :105-145): molecule-1 type (0 for NAM), the number of
// definitions, then per definition the partner type, the contacts needed, the number
// of pairs and the pairs (sphere of molecule 1, sphere of molecule 2, and a distance
// when sepdist <= 0).  A file that ends inside a definition is refused.
extern "C" int pbsam_system_bd_set_contacts_file(pbsam_system *s, const char *path, double sepdist)
{
  if (!s || !path) return fail(PBSAM_E_BADARG, "null argument");
  std::ifstream in(path);
  if (!in) return fail(PBSAM_E_IO, std::string("cannot open contact file ") + path);
  int mol1type = -1, ndef = 0;
  if (!(in >> mol1type >> ndef)) return fail(PBSAM_E_IO, std::string("contact file header: ") + path);
  if (mol1type != 0) return fail(PBSAM_E_BADARG, "NAM contact definitions are for molecule type 0");
  std::vector<int> partner, ncon, off(1, 0), k1, k2;
  std::vector<double> dist;
  int mol2type;
  while (in >> mol2type) {
    int nc = 0, npair = 0;
    if (!(in >> nc >> npair) || npair < 0) return fail(PBSAM_E_IO, std::string("contact definition: ") + path);
    for (int n = 0; n < npair; n++) {
      int a, b;
      double dd = sepdist;
      if (!(in >> a >> b) || (sepdist <= 0 && !(in >> dd)))
        return fail(PBSAM_E_IO, std::string("contact file ends inside a definition: ") + path);
      k1.push_back(a);
      k2.push_back(b);
      dist.push_back(dd);
    }
    partner.push_back(mol2type);
    ncon.push_back(nc);
    off.push_back((int)k1.size());
  }
  return pbsam_system_bd_set_contacts(s, (int)partner.size(), partner.data(), ncon.data(), off.data(), k1.data(),
                                      k2.data(), dist.data());
}

extern "C" int pbsam_system_bd_state(pbsam_system *s, double *pos, double *quat, int *status, int *steps,
                                     double *time, int *fevals, int on_device)
{
  if (!s) return fail(PBSAM_E_BADARG, "null system");
  BDHost *h = s->bd;
  if (!h) return fail(PBSAM_E_STATE, "pbsam_system_bd_init has not been called");
  CK(cudaSetDevice(s->ctx->device));
  const cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t B = s->B, nm = s->nmol;
  if (pos) CK(cudaMemcpyAsync(pos, h->v.pos, B * nm * 3 * sizeof(double), k, s->stream));
  if (quat) CK(cudaMemcpyAsync(quat, h->v.quat, B * nm * 4 * sizeof(double), k, s->stream));
  if (status) CK(cudaMemcpyAsync(status, h->v.status, B * sizeof(int), k, s->stream));
  if (steps) CK(cudaMemcpyAsync(steps, h->v.steps, B * sizeof(int), k, s->stream));
  if (time) CK(cudaMemcpyAsync(time, h->v.time, B * sizeof(double), k, s->stream));
  if (fevals) CK(cudaMemcpyAsync(fevals, h->v.fevals, B * sizeof(int), k, s->stream));
  if (!on_device) CK(cudaStreamSynchronize(s->stream));
  return PBSAM_OK;
}
