/* C ABI of the B200 drop-in for PB-SAM's mutual-polarization solve and its
 * force/torque evaluation.
 *
 * The reference exposes this path as a C++ class API called by its drivers
 * (pbsam / bdnam / bdm); each entry point below replaces the reference call
 * named in its comment (paths relative to the PB-SAM source tree).  Plain
 * pointers and sizes only; every call returns an int status (PBSAM_OK = 0,
 * negative = call error).  Per-system outcomes of a force evaluation are
 * reported in a status array (PBSAM_SYS_*), never by exiting the process.
 *
 * Units and layouts follow the reference: lengths in Angstrom, charges in e,
 * expansions in the packed real layout of src/expansion.h:509-553 (p*p doubles
 * per expansion), IMats p^2 x p^2 column-major doubles, quaternions (w,x,y,z).
 * Forces and torques are returned exactly as CMolecule::computeForces returns
 * them (molecule-frame sums rotated by the conjugate orientation,
 * src/moldynamics.cpp:524-550).
 */
#ifndef PBSAM_B200_H
#define PBSAM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define PBSAM_OK 0
#define PBSAM_E_BADARG (-1)
#define PBSAM_E_IO (-2)
#define PBSAM_E_CUDA (-3)
#define PBSAM_E_NOMEM (-4)
#define PBSAM_E_STATE (-5)

/* per-system status of a force evaluation */
#define PBSAM_SYS_OK 0
#define PBSAM_SYS_OVERLAP 1   /* two spheres of different molecules overlap
                                 (computeForces returns false, src/molecule.cpp:1090-1097) */
#define PBSAM_SYS_NOT_CONVERGED 2   /* a polarization or gradient sweep loop stopped at
                                       max_pol_rounds ("Polarization does not converge",
                                       src/molecule.cpp:1963-1967); forces are returned */
#define PBSAM_SYS_NAN 3       /* a non-finite pose (coordinate, or a zero quaternion) was
                                 refused, or the evaluation produced a non-finite force or
                                 torque (CExpan::isBlownup, src/expansion.h:216-221) */

typedef struct pbsam_params {
  int poles;              /* pole order p (the reference's N_POLES, src/expansion.h:5-9) */
  double salt;            /* ionic strength in mol/L; kappa as src/BDnam_main.cpp:53-55 */
  double idiel;           /* interior dielectric (4) */
  double sdiel;           /* solvent dielectric (78) */
  double temperature;     /* K (298.15) */
  double max_polar_dev;   /* MAX_POLAR_DEV, src/molecule.cpp:6 (1e-2) */
  double solve_tol;       /* SOLVE_TOL, src/expcenter.cpp:17 (1e-8) */
  int solve_max_ct;       /* SOLVE_MAX_CT, src/expcenter.cpp:18 (100) */
  int max_pol_rounds;     /* MAX_POL_ROUNDS, src/molecule.cpp:10 (1000) */
  double inter_cutoff;    /* inter-molecular polarization cutoff, src/BDnam.cpp:138 (10) */
  double interact_cutoff; /* interaction cutoff, src/BDnam.cpp:139 (100) */
  double intra_cutoff;    /* intra near-list cutoff, src/BDnam.cpp:82 (30) */
  double min_sep_numeric; /* MINSEPDIST, src/molecule.h:22 (5) */
  int num_points_x;       /* NUM_POINTS_X cap on surface points, src/molecule.cpp:64 (10000) */
  int cluster_size;       /* CTAs (one thread-block cluster) working on each system: 0 = the largest
                             of 16, 8, 4, 2 that keeps a whole batch resident at once; 1..16 forces it;
                             -1 = adaptive: before each evaluation the systems are regrouped by the
                             inner-iteration counts of the previous one, costlier systems getting
                             larger clusters (the rounding of the results may then differ between
                             calls by ~1e-15); the call then waits for the previous evaluation's
                             counters, so consecutive calls of one system do not overlap on the host.
                             No reference counterpart (a B200 launch parameter). */
  int exact;              /* 0 (default): the reference's iteration, reproduced step by step
                             (src/molecule.cpp:1988-2263, src/expcenter.cpp:1079-1135).
                             1: the exact form of the same equations: every sphere's inner F/H
                             fixed point solved directly through an operator prepared once per
                             sphere type at the first system (the reference's iteration of it
                             does not converge on every sphere: its spectral radius can exceed
                             one, and its result then moves with solve_max_ct), every polarized
                             sphere swept until its change is below exact_tol, and forces
                             and torques taken as the exact negative gradient of the lab-frame
                             energy (pbsam_system_compute_energy_lab) by the adjoint of that state,
                             in the lab frame (pbsam_system_backward).  One CTA per system; pole
                             order <= 32.  No reference counterpart. */
  double box_length;      /* 0 (default): no periodic box.  > 0: a cubic periodic box of this
                             edge in A, as CSystem::initConstants(kappa, sdiel, T, true, L)
                             (src/system.h:18-20) sets it for bdm.  Molecule centres are wrapped
                             into the box at each evaluation and BD move (CMolecule::setPos,
                             translate, src/molecule.h:325-327); the pair lists, the
                             polarization and gradient re-expansions, the potential, the minimum
                             separations and the overlap tests take the minimum image of each
                             displacement (CSystem::pbcPos, src/system.cpp:46-55), while the
                             gradient lists of prepareDTA (src/molecule.cpp:1515-1619) and the
                             energy (src/molecule.cpp:1873) take the plain difference of the
                             wrapped centres, as the reference does.  The lab-frame energy and
                             the exact form take the minimum image everywhere. */
  int exact_tables;       /* exact form only.  1 (default): the intra-molecular near-field
                             re-expansions of each molecule type (numeric for overlapping sphere
                             pairs, rotation + translation for the others) are prepared once as
                             full-order p^2 x p^2 operators when they fit in 4 GB (else those of
                             the numeric pairs alone when they fit; p = 10: about 150 MB per
                             35-sphere type) and applied as products in the sweeps and in the
                             backward pass, and the angles of every exposed surface point are
                             tabulated (32 bytes a point) for the surface charges of each
                             solve; 0: transformed and evaluated as the plain drop-in does.
                             The two agree to rounding. */
  double exact_tol;       /* exact form only: the sweeps, and the backward pass's transposed
                             sweeps, stop once the root-mean-square relative change of the
                             polarized spheres' H (their adjoint) is below it.  Default 1e-14;
                             the error of the state, and so of the forces, is of this order. */
  double exact_relax;     /* exact form only: the sweeps' updates (after the first round) and the
                             transposed sweeps' are over-relaxed by this factor in (0, 2),
                             x += w (x_swept - x).  Default 1 (plain Gauss-Seidel); the fixed
                             point does not depend on it, the number of sweeps does. */
} pbsam_params;

typedef struct pbsam_context pbsam_context;
typedef struct pbsam_system pbsam_system;

/* Defaults equal to the reference built with __ACCURATE__ at N_POLES = 10. */
void pbsam_params_default(pbsam_params *prm);

/* Replaces CSystem::initConstants(kappa, sdiel, temp) (src/system.h:19-20,
 * src/system.cpp:15-25) and the constant tables it triggers
 * (CMolecule::initConstants, src/molecule.cpp:41-70).  One context per device. */
int pbsam_context_create(const pbsam_params *prm, int device, pbsam_context **ctx);
int pbsam_context_destroy(pbsam_context *ctx);
/* inverse Debye length used by the context (CSystem::KAPPA) */
int pbsam_context_kappa(const pbsam_context *ctx, double *kappa);

/* Replaces the per-species part of CBDnam::CBDnam (src/BDnam.cpp:59-119):
 * readpqr, readMats (imat.sp<k>.out.bin), readExpansionsP (<name>.<k>.{F,H}.exp),
 * generateMolSPX, generateMolExposedChargesFH, generateMolTypeIntraPolLists and
 * computeMolTypeValues.  All types must be added before the first system. */
int pbsam_moltype_load(pbsam_context *ctx, const char *pqr_path, const char *imat_dir,
                       const char *exp_dir, const char *exp_name, int *type_id);
/* Same from memory: centres[n_sph*3], radii[n_sph], chg_pos[n_chg*3], chg[n_chg],
 * imats[n_sph*p^4], fself/hself[n_sph*p^2], hself_scale[n_sph] (the scale value stored
 * with each H expansion). */
int pbsam_moltype_create(pbsam_context *ctx, int n_sph, const double *centres, const double *radii,
                         int n_chg, const double *chg_pos, const double *chg, const double *imats,
                         const double *fself, const double *hself, const double *hself_scale, int *type_id);
/* number of spheres / exposed surface points of a type */
int pbsam_moltype_info(const pbsam_context *ctx, int type_id, int *n_sph, int *n_points);

/* Replaces constructing the CMolecule objects of a run (src/molecule.h:67-77)
 * followed by CMolecule::initMutualConstants(mols, inter, interact, true)
 * (src/molecule.cpp:77-95), for n_systems independent copies of the same
 * molecule list (mol_types[n_mol], 1 <= n_mol <= 64).  Each system keeps its own
 * solver state between calls, as the reference's molecules do. */
int pbsam_system_create(pbsam_context *ctx, int n_systems, int n_mol, const int *mol_types,
                        pbsam_system **sys);
int pbsam_system_destroy(pbsam_system *sys);
/* Return every system to the freshly constructed state. */
int pbsam_system_reset(pbsam_system *sys);

/* Replaces CMolecule::setPos / setOrient (src/molecule.h:325-326):
 * pos[n_systems*n_mol*3], quat[n_systems*n_mol*4]; on_device != 0 means the
 * pointers are device pointers. */
int pbsam_system_set_poses(pbsam_system *sys, const double *pos, const double *quat, int on_device);

/* Replaces CMolecule::computeForces(mols, force, torque) (src/molecule.h:179,
 * src/moldynamics.cpp:553-587) for every system: force/torque[n_systems*n_mol*3],
 * status[n_systems] (PBSAM_SYS_*).  Any output pointer may be NULL. */
int pbsam_system_compute_forces(pbsam_system *sys, double *force, double *torque, int *status, int on_device);

/* Replaces CMolecule::computeTotalIntEnergy (src/molecule.h:180,
 * src/moldynamics.cpp:358-386) on the state left by the last force evaluation. */
int pbsam_system_compute_energy(pbsam_system *sys, double *energy, int on_device);
/* The same interaction energy with the orientation taken into account: sphere
 * centres at pos + q*cen and every H rotated to the lab frame by its molecule's
 * orientation before the pair re-expansions, so the value is invariant under a
 * rigid motion of the whole system.  Replaces interactCenters_LowMemory
 * (src/molecule.cpp:1850-1890), which uses the unrotated centres and molecule-frame
 * H, in the corrected form; the reference has no such call. */
int pbsam_system_compute_energy_lab(pbsam_system *sys, double *energy, int on_device);

/* Backward pass (exact form only: contexts made with exact = 1).  After
 * pbsam_system_compute_forces, the gradient of each system's lab-frame interaction
 * energy U with respect to every molecule's position and orientation, each scaled by
 * seed[b] = dL/dU of system b (NULL: 1): dpos[n_systems*n_mol*3] = dL/dpos,
 * dquat[n_systems*n_mol*4] = dL/dquat (the derivative along q' = (1, w/2) q,
 * tangent to the unit sphere, w the lab-frame rotation vector), drot[n_systems*n_mol*3]
 * = dL/dw (minus the torque).  Any output may be NULL.  Replaces the reference's
 * per-molecule gradient solves (CMolecule::polarize_mutual phase D,
 * src/molecule.cpp:2081-2228, with prepareDTA / recomputeGrad, src/molecule.cpp:1483-1843)
 * by one transposed solve of the converged state; the reference's own forces are not
 * the gradient of its energy (its energy, src/molecule.cpp:1850-1890, ignores the
 * orientation and its gradient solves differentiate a state its sweeps do not reach). */
int pbsam_system_backward(pbsam_system *sys, const double *seed, double *dpos, double *dquat, double *drot,
                          int on_device);

/* Electrostatic potential at points from the state of the last force evaluation:
 * replaces CMolecule::computePotInSpace (src/moldynamics.cpp:470-506) for molecules that
 * are not aggregated (as in the BD drivers).  points[n_points*3] shared by every system,
 * or [n_systems*n_points*3] with per_system != 0; pot[n_systems*n_points].  lab = 0 uses
 * the reference's convention (unrotated sphere centres and molecule-frame H, as its
 * energy), lab = 1 the rotated centres and lab-frame H. */
int pbsam_system_potential(pbsam_system *sys, int n_points, const double *points, int per_system, int lab,
                           double *pot, int on_device);

/* Counters of the last force evaluation, 8 ints per system: [0] sweeps,
 * [1] inner F/H iterations, [2] inner solves, [3] gradient solves,
 * [4] bit 0: the polarization sweeps hit max_pol_rounds, bit 1: a gradient phase
 * (or the exact form's transposed sweeps) hit it, [5] CTAs that worked on the system. */
int pbsam_system_stats(const pbsam_system *sys, int *stats);

/* CUDA stream the system's work is queued on (cudaStream_t as void*); the
 * calls above synchronise it before returning host results. */
int pbsam_system_set_stream(pbsam_system *sys, void *stream);

/* Device time per phase of the last force evaluation (or self-polarization), 16
 * doubles per system in ms: [0] F/H solves, [1] surface charges, [2] numeric
 * near-field re-expansions, [3] analytic intra re-expansions, [4] inter-molecular
 * LS re-expansions, [5] gradient re-expansions of H (DTA), [6] re-expansions of
 * the gradient solves (inter and intra, before each gradient F/H solve), [7] whole
 * evaluation, [8] gradient surface charges and rotation of the gradient H,
 * [9] set-up (pair lists, molecule rotations), [10] gradient-phase bookkeeping,
 * [11] force and torque sums; sub-phases: [12]-[14] the inter, intra analytic and
 * intra numeric parts of [6], [15] the IMat products within [0].  The phases
 * [0]-[6] and [8]-[11] do not overlap; [7] includes everything.  In the exact form
 * (pbsam_params.exact) [6] is the backward pass and [12]-[14] are its energy
 * adjoint, its transposed sweeps and its first-round and rotation terms. */
int pbsam_system_phase_ms(const pbsam_system *sys, double *ms);

/* Device time in milliseconds of the last force-kernel launch (CUDA events). */
int pbsam_system_last_kernel_ms(const pbsam_system *sys, double *ms);

/* Brownian dynamics on the force path: the Ermak-McCammon step of the reference's
 * drivers, for every system of a batch (each system one trajectory).
 *   PBSAM_BD_NAM   = CBDnam::run / makeMove / compute_dt (src/BDnam.cpp:166-417):
 *                    two molecules, molecule 0 rotates in place, molecule 1
 *                    translates and rotates; forces while the centre distance is
 *                    below force_dist; PBSAM_BD_ESCAPED beyond escape_dist;
 *                    PBSAM_BD_STUCK after max_tries rejected draws.
 *   PBSAM_BD_MULTI = CBDmulti::propagate / makeMove / compute_dt / computeMinSepDist
 *                    (src/BDmulti.cpp:396-566): every molecule moves in turn;
 *                    forces while the minimum separation is below the context's
 *                    interaction cutoff (the periodic box of pbsam_params.box_length
 *                    applies, as bdm's); the minimum separation
 *                    is the smallest sphere gap over all molecule pairs, at least
 *                    dt_ref, as the reference's bdm computes it.
 * Time step dt = min(dt_max, dt_min + max(0, d - dt_ref) / dt_div) ps, d the
 * molecule gap (NAM) or the minimum separation (MULTI); drifts D*dt*fact_tr*F and
 * Dr*dt*ikbt*coul_k*torque; noise N(0, 2*D*dt) per component from Philox4x64-10
 * (key = seed, counter = (draw, system)) where the reference uses drand48.
 * NAM docking (PBSAM_BD_DOCKED) is tested after each move once contact definitions
 * are set (pbsam_system_bd_set_contacts).  A force evaluation that finds overlapping
 * spheres ends the trajectory with PBSAM_BD_FAILED, where the reference exits
 * (src/BDnam.cpp:210-212). */
#define PBSAM_BD_NAM 0
#define PBSAM_BD_MULTI 1
#define PBSAM_BD_RUNNING 0
#define PBSAM_BD_ESCAPED 1
#define PBSAM_BD_STUCK 2
#define PBSAM_BD_DOCKED 3
#define PBSAM_BD_FAILED 4

typedef struct pbsam_bd_params {
  int mode;              /* PBSAM_BD_NAM or PBSAM_BD_MULTI */
  int max_tries;         /* draws per move before giving up (maxc = 500) */
  double force_dist;     /* NAM: forces while centre distance < this (f_DIST = 100) */
  double escape_dist;    /* NAM: escape radius (q_DIST = 500) */
  double dt_min, dt_max, dt_ref, dt_div;   /* time-step schedule (2, none, 5 or 10, 15) */
  double fact_tr;        /* FACT2 = 560.4586 */
  double ikbt;           /* IKbT = 1/(kB*298.15) */
  double coul_k;         /* COUL_K = 2.30708e-18 */
  unsigned long long seed;
  int use_graph;         /* 1: a step is replayed as one CUDA graph */
  int noise;             /* PBSAM_BD_NOISE_PHILOX (default) or PBSAM_BD_NOISE_DRAND48: the
                            reference's own stream (drand48 seeded by srand48(seed + system), the
                            polar Box-Muller of normRand, src/util.h:489-539), drawn sequentially per
                            system, so that system b repeats the reference's bdnam run seeded with
                            seed + b (src/BDnam_main.cpp:39-41 seeds from the clock instead) */
} pbsam_bd_params;
#define PBSAM_BD_NOISE_PHILOX 0
#define PBSAM_BD_NOISE_DRAND48 1

/* Reference values of the chosen driver (src/BDnam.h:10-25, src/BDmulti.cpp:13,
 * src/BDnam.cpp:409-417). */
void pbsam_bd_params_default(int mode, pbsam_bd_params *prm);
/* Start a trajectory in every system from its current poses (set them first with
 * pbsam_system_set_poses): dtr/drot[n_mol] translational (A^2/ps) and rotational
 * (rad^2/ps) diffusion coefficients per molecule (the reference's m_Dtr, m_Dr1,
 * m_Dr2, src/BDnam.cpp:145, src/BDmulti.cpp:204-205). */
int pbsam_system_bd_init(pbsam_system *sys, const pbsam_bd_params *prm, const double *dtr, const double *drot);
/* Queue n_steps steps of every running trajectory on the system's stream (the
 * while loop of CBDnam::run, src/BDnam.cpp:196-243); returns without waiting.
 * Trajectories that stopped (escaped, stuck, failed) are left as they are. */
int pbsam_system_bd_run(pbsam_system *sys, int n_steps);
/* Poses pos[n_systems*n_mol*3], quat[n_systems*n_mol*4], status[n_systems]
 * (PBSAM_BD_*), steps taken, simulated time (ps) and force evaluations per
 * trajectory.  Any pointer may be NULL. */
int pbsam_system_bd_state(pbsam_system *sys, double *pos, double *quat, int *status, int *steps, double *time,
                          int *fevals, int on_device);
/* NAM docking criteria (CBDnam::addMolContact + CBDnam::IsDocked, src/BDnam.cpp:38-41,
 * 379-399): after each move of a running trajectory it is PBSAM_BD_DOCKED when, for
 * some definition d with partner[d] == 1 (the species of molecule 1), at least
 * ncontact[d] >= 1 of its pairs off[d] .. off[d+1]-1 have a surface gap (centre
 * distance minus both radii, CMolecule::getSepDist) of at most dist[e] between sphere
 * k1[e] of molecule 0 and sphere k2[e] of molecule 1 (0-based, PQR order).  n_defs = 0
 * removes them.  After pbsam_system_bd_init; NAM only. */
int pbsam_system_bd_set_contacts(pbsam_system *sys, int n_defs, const int *partner, const int *ncontact,
                                 const int *off, const int *k1, const int *k2, const double *dist);
/* The same from a contactdef file: CMolContact::readMolContact (every pair at distance
 * sepdist, the bdnam command line's docking distance; src/contact.cpp:53-97) when
 * sepdist > 0, readMolContactWithDist (a distance on every pair line, :105-145) when
 * sepdist <= 0.  The molecule-1 type must be 0; a file that ends inside a definition
 * is PBSAM_E_IO. */
int pbsam_system_bd_set_contacts_file(pbsam_system *sys, const char *path, double sepdist);

/* Forces, torques and statuses of the last evaluation of every system, without
 * evaluating again (after a group evaluation, pbsam_group_compute_forces). */
int pbsam_system_get_forces(pbsam_system *sys, double *force, double *torque, int *status, int on_device);

/* Groups of system handles (no reference counterpart: the reference runs one
 * trajectory per process).  The systems of several handles, each with its own
 * molecule list and sphere counts and possibly its own context (pole order), are
 * evaluated in one launch, one CTA per system, longest first: at creation by the
 * square of the sphere count, after pbsam_group_tune by the device time of each
 * system's last evaluation.  Results stay in each handle (pbsam_system_get_forces,
 * pbsam_system_bd_state).  Every handle on the same device; a handle belongs to at
 * most one group at a time and is not used on its own while a group call runs. */
typedef struct pbsam_group pbsam_group;
int pbsam_group_create(int n, pbsam_system *const *systems, pbsam_group **out);
int pbsam_group_destroy(pbsam_group *g);
/* One launch over every system of every handle (CMolecule::computeForces of each). */
int pbsam_group_compute_forces(pbsam_group *g);
/* Reorder the systems by the device time of their last evaluation, longest first. */
int pbsam_group_tune(pbsam_group *g);
/* n_steps BD steps of every trajectory of every handle (each pbsam_system_bd_init'ed,
 * contact lists included): one CUDA graph per step, the same steps as each handle's
 * own pbsam_system_bd_run. */
int pbsam_group_bd_run(pbsam_group *g, int n_steps);

/* bdm restart configurations, host only (no device needed): readConfigWithMolType
 * (src/readutil.cpp:835-886, used by CBDmulti::restartConfig, src/BDmulti.cpp:286-316)
 * and CMolecule::saveConfig (src/molecule.cpp:255-269).  One molecule per line:
 * "x y z qw qx qy qz type".  pbsam_config_read stores up to max_mol molecules (pos
 * [3 each], quat [4 each], moltype; any may be NULL) and sets *n_mol to the number in
 * the file (PBSAM_E_BADARG when it exceeds max_mol; PBSAM_E_IO for a file that ends
 * inside a molecule or has a field that is not a number).  pbsam_config_write writes
 * at full precision (the reference's stream default keeps 6 digits). */
int pbsam_config_read(const char *path, int max_mol, int *n_mol, double *pos, double *quat, int *moltype);
int pbsam_config_write(const char *path, int n_mol, const double *pos, const double *quat, const int *moltype);

/* Molecule-type preparation (the reference's `pbsam mat` and `pbsam spol`).
 *
 * Surface-integral matrices of a molecule's spheres: replaces the CMolecule IMat
 * constructor with build_IMatE (src/molecule.cpp:279-346, src/expcenter.cpp:910-1033);
 * centres are absolute, n_points is NUM_POINTS_I (250000 in the reference);
 * imats receives n_sph * p^4 doubles, the content of imat.sp<k>.out.bin. */
int pbsam_imat_build(pbsam_context *ctx, int n_sph, const double *centres, const double *radii, int n_points,
                     double *imats);
/* No counterpart in the reference.  Same result as pbsam_imat_build, for callers
 * that cannot allocate device memory (their own pool allocator owns the device, or
 * their footprint must stay fixed after load): the work buffers are one fixed
 * device array of about 3.2 MB that the library holds on every device it is used
 * on.  Limits: pole order <= 16, at most 256 spheres overlapping any one sphere;
 * larger cases return PBSAM_E_BADARG.  The first call on a device looks up the
 * array's address; make it before any stream capture.  All calls share the array:
 * calls that overlap on the GPU race, so callers serialise them. */
int pbsam_imat_build_static(pbsam_context *ctx, int n_sph, const double *centres, const double *radii, int n_points,
                            double *imats);
/* Self-polarization of one molecule type: replaces CMolecule::polarize_self
 * (src/molecule.cpp:1898-1979) as run by `pbsam spol` (src/selfp_makemat.cpp:37-118).
 * The type's own F/H inputs are ignored.  Outputs are rounded as the reference
 * writes its .exp files: fself/hself[n_sph*p^2], hself_scale[n_sph]; rounds
 * receives the number of sweeps. */
int pbsam_selfpol(pbsam_context *ctx, int type_id, int max_rounds, double *fself, double *hself,
                  double *hself_scale, int *rounds);

/* No counterpart in the reference.  The FP64 FMA rate (TFLOP/s) and the L2 read
 * bandwidth (GB/s) of a device, timed in place over every SM (best of three launches):
 * the denominators of the force kernel's roofline, whose IMat rows stay in L2 and whose
 * arithmetic is FP64. */
int pbsam_device_peaks(int device, double *fp64_tflops, double *l2_gbs);

/* Single-expansion operations, batched, with the semantics of the reference's
 * rotation, translation and re-expansion classes, for callers that drive expansions
 * one by one (the CRotCoeff / CTransCoeff / CXFormA classes of
 * pb-sam_b200/cpp/pbsam_b200.hpp).  n items; in, out: [n][poles^2] packed real
 * expansions (degrees >= p of in are ignored, those of out are zero); host pointers
 * (on_device = 0) or device pointers of the context's device (1).  One CTA per item. */

/* CRotCoeff::reset(theta, phi, xi, p) (src/rotcoeff.cpp:155-171) then rotate
 * (with_xi = 0, src/rotcoeff.cpp:357-441) or rotateWithXi (with_xi = 1, :250-350), forward
 * (1) or back (0).  rot: [n][3] = theta, phi, xi. */
int pbsam_expan_rotate(pbsam_context *c, int n, const double *rot, int p, int with_xi, int forward,
                       const double *in, double *out, int on_device);

/* CTransCoeff::reset(rho, kappa, p, scalei, scaleo) (src/transcoeff.cpp:172-203) then
 * translate (deriv = 0, :211-286) or dTranslate (deriv = 1, :294-364), with the context's
 * kappa (screened = 1) or 0.  args: [n][3] = rho > 0, scale in, scale out. */
int pbsam_expan_translate(pbsam_context *c, int n, const double *args, int p, int screened, int deriv,
                          const double *in, double *out, int on_device);

/* CXFormA(source, target).reset(P, p) then xformH (screened = 1, src/xforms.cpp:122-132)
 * or xformF (0, :260-270); grad (nullable, screened only): [n][3][poles^2], the x, y, z
 * derivatives w.r.t. the target position (CGradExpan, src/xforms.cpp:85-115).  args:
 * [n][5] = P = target centre - source centre (3), source scale, target scale (the
 * spheres' radii). */
int pbsam_expan_reexpand(pbsam_context *c, int n, const double *args, int p, int screened, const double *in,
                         double *out, double *grad, int on_device);

/* CRotCoeff::reset(const CQuat &, p)'s Euler angles (theta, phi, xi) of a quaternion
 * (w, x, y, z), normalised first (src/rotcoeff.cpp:181-201). */
int pbsam_quat_angles(const double *q, double *angles);

/* Text of the last error on the calling thread. */
const char *pbsam_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
