"""Python host mirror of the B200 PB-SAM drop-in (ctypes over include/pbsam_b200.h).

The reference exposes this path as C++ classes; the names here follow them:

* ``CSystem`` -- ``CSystem::initConstants(kappa, sdiel, temp)`` plus the
  compile-time tolerances of the reference (src/system.h:19-20), i.e. one
  solver context on one GPU.
* ``CSystem.load_moltype`` -- the per-species set-up of ``CBDnam::CBDnam``
  (src/BDnam.cpp:59-119): PQR, ``imat.sp<k>.out.bin``, ``<name>.<k>.{F,H}.exp``.
* ``Molecules`` -- the ``vector<CMolecule*>`` of a run, here for ``n_systems``
  independent copies; ``setPos``/``setOrient`` (src/molecule.h:325-326),
  ``computeForces`` (src/molecule.h:179) and ``computeTotalIntEnergy``
  (src/molecule.h:180).

The CUDA library ``lib/libpbsam_b200.so`` must be built (``__graft_entry__.build``);
there is no CPU fallback: every call runs the sm_100a kernels.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libpbsam_b200.so")

PBSAM_SYS_OK = 0
PBSAM_SYS_OVERLAP = 1
PBSAM_SYS_NOT_CONVERGED = 2
PBSAM_SYS_NAN = 3


class pbsam_params(ctypes.Structure):
    _fields_ = [("poles", ctypes.c_int), ("salt", ctypes.c_double), ("idiel", ctypes.c_double),
                ("sdiel", ctypes.c_double), ("temperature", ctypes.c_double),
                ("max_polar_dev", ctypes.c_double), ("solve_tol", ctypes.c_double),
                ("solve_max_ct", ctypes.c_int), ("max_pol_rounds", ctypes.c_int),
                ("inter_cutoff", ctypes.c_double), ("interact_cutoff", ctypes.c_double),
                ("intra_cutoff", ctypes.c_double), ("min_sep_numeric", ctypes.c_double),
                ("num_points_x", ctypes.c_int), ("cluster_size", ctypes.c_int), ("exact", ctypes.c_int),
                ("box_length", ctypes.c_double), ("exact_tables", ctypes.c_int),
                ("exact_tol", ctypes.c_double), ("exact_relax", ctypes.c_double)]


PBSAM_BD_NAM = 0
PBSAM_BD_MULTI = 1
PBSAM_BD_NOISE_PHILOX = 0
PBSAM_BD_NOISE_DRAND48 = 1
PBSAM_BD_RUNNING = 0
PBSAM_BD_ESCAPED = 1
PBSAM_BD_STUCK = 2
PBSAM_BD_DOCKED = 3
PBSAM_BD_FAILED = 4
BD_STATUS = {0: "RUNNING", 1: "ESCAPED", 2: "STUCK", 3: "DOCKED", 4: "FAILED"}


class pbsam_bd_params(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("max_tries", ctypes.c_int), ("force_dist", ctypes.c_double),
                ("escape_dist", ctypes.c_double), ("dt_min", ctypes.c_double), ("dt_max", ctypes.c_double),
                ("dt_ref", ctypes.c_double), ("dt_div", ctypes.c_double), ("fact_tr", ctypes.c_double),
                ("ikbt", ctypes.c_double), ("coul_k", ctypes.c_double), ("seed", ctypes.c_ulonglong),
                ("use_graph", ctypes.c_int), ("noise", ctypes.c_int)]


# every entry point declared in include/pbsam_b200.h, with ctypes signatures
_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
SIGNATURES = {
    "pbsam_params_default": (None, [ctypes.POINTER(pbsam_params)]),
    "pbsam_context_create": (ctypes.c_int, [ctypes.POINTER(pbsam_params), ctypes.c_int, ctypes.POINTER(_P)]),
    "pbsam_context_destroy": (ctypes.c_int, [_P]),
    "pbsam_context_kappa": (ctypes.c_int, [_P, _DP]),
    "pbsam_moltype_load": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _IP]),
    "pbsam_moltype_create": (ctypes.c_int, [_P, ctypes.c_int, _DP, _DP, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _DP, _IP]),
    "pbsam_moltype_info": (ctypes.c_int, [_P, ctypes.c_int, _IP, _IP]),
    "pbsam_system_create": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _IP, ctypes.POINTER(_P)]),
    "pbsam_system_destroy": (ctypes.c_int, [_P]),
    "pbsam_system_reset": (ctypes.c_int, [_P]),
    "pbsam_system_set_poses": (ctypes.c_int, [_P, _P, _P, ctypes.c_int]),
    "pbsam_system_compute_forces": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int]),
    "pbsam_system_compute_energy": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "pbsam_system_compute_energy_lab": (ctypes.c_int, [_P, _P, ctypes.c_int]),
    "pbsam_system_stats": (ctypes.c_int, [_P, _IP]),
    "pbsam_system_backward": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int]),
    "pbsam_system_potential": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int]),
    "pbsam_system_set_stream": (ctypes.c_int, [_P, _P]),
    "pbsam_system_last_kernel_ms": (ctypes.c_int, [_P, _DP]),
    "pbsam_system_phase_ms": (ctypes.c_int, [_P, _DP]),
    "pbsam_imat_build": (ctypes.c_int, [_P, ctypes.c_int, _DP, _DP, ctypes.c_int, _DP]),
    "pbsam_imat_build_static": (ctypes.c_int, [_P, ctypes.c_int, _DP, _DP, ctypes.c_int, _DP]),
    "pbsam_selfpol": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _DP, _DP, _DP, _IP]),
    "pbsam_bd_params_default": (None, [ctypes.c_int, ctypes.POINTER(pbsam_bd_params)]),
    "pbsam_system_bd_init": (ctypes.c_int, [_P, ctypes.POINTER(pbsam_bd_params), _DP, _DP]),
    "pbsam_system_bd_run": (ctypes.c_int, [_P, ctypes.c_int]),
    "pbsam_system_bd_state": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int]),
    "pbsam_device_peaks": (ctypes.c_int, [ctypes.c_int, _DP, _DP]),
    "pbsam_expan_rotate": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P,
                                          ctypes.c_int]),
    "pbsam_expan_translate": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P,
                                             ctypes.c_int]),
    "pbsam_expan_reexpand": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int, _P, _P, _P,
                                            ctypes.c_int]),
    "pbsam_quat_angles": (ctypes.c_int, [_DP, _DP]),
    "pbsam_system_bd_set_contacts": (ctypes.c_int, [_P, ctypes.c_int, _IP, _IP, _IP, _IP, _IP, _DP]),
    "pbsam_system_bd_set_contacts_file": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_double]),
    "pbsam_config_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _IP, _DP, _DP, _IP]),
    "pbsam_system_get_forces": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int]),
    "pbsam_group_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "pbsam_group_destroy": (ctypes.c_int, [_P]),
    "pbsam_group_compute_forces": (ctypes.c_int, [_P]),
    "pbsam_group_tune": (ctypes.c_int, [_P]),
    "pbsam_group_bd_run": (ctypes.c_int, [_P, ctypes.c_int]),
    "pbsam_config_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _DP, _DP, _IP]),
    "pbsam_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("CUDA library not built: %s (run __graft_entry__.build())" % LIB_PATH)
        _lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


class PbsamError(RuntimeError):
    """A call returned a PBSAM_E_* status; ``code`` holds it."""

    def __init__(self, msg, code=0):
        super().__init__(msg)
        self.code = code


def _check(rc):
    if rc != 0:
        msg = lib().pbsam_last_error()
        raise PbsamError("pbsam error %d: %s" % (rc, msg.decode() if msg else ""), rc)


def default_params(**kw):
    p = pbsam_params()
    lib().pbsam_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def bd_params(mode=PBSAM_BD_NAM, **kw):
    """pbsam_bd_params with the reference driver's values, fields overridden by kw."""
    p = pbsam_bd_params()
    lib().pbsam_bd_params_default(mode, ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _dptr(a):
    return a.ctypes.data_as(_DP)


class Group:
    """Several Molecules handles (different molecule lists, sphere counts, contexts)
    evaluated in one launch, longest systems first (pbsam_group_*)."""

    def __init__(self, handles):
        self.handles = list(handles)
        arr = (_P * len(self.handles))(*[h.handle for h in self.handles])
        g = _P()
        _check(lib().pbsam_group_create(len(self.handles), arr, ctypes.byref(g)))
        self.handle = g

    def compute_forces(self):
        _check(lib().pbsam_group_compute_forces(self.handle))
        return [h.get_forces() for h in self.handles]

    def tune(self):
        _check(lib().pbsam_group_tune(self.handle))

    def bd_run(self, n_steps):
        _check(lib().pbsam_group_bd_run(self.handle, n_steps))

    def close(self):
        if self.handle:
            _check(lib().pbsam_group_destroy(self.handle))
            self.handle = None


def config_read(path):
    """bdm restart configuration: (pos [n][3], quat [n][4], moltype [n])."""
    n = ctypes.c_int()
    rc = lib().pbsam_config_read(path.encode(), 0, ctypes.byref(n), None, None, None)
    if rc != 0 and n.value == 0:
        _check(rc)
    pos, quat, mt = np.zeros((n.value, 3)), np.zeros((n.value, 4)), np.zeros(n.value, dtype=np.int32)
    _check(lib().pbsam_config_read(path.encode(), n.value, ctypes.byref(n), _dptr(pos), _dptr(quat),
                                   mt.ctypes.data_as(_IP)))
    return pos, quat, mt


def config_write(path, pos, quat, moltype):
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    quat = np.ascontiguousarray(quat, dtype=np.float64).reshape(-1, 4)
    mt = np.ascontiguousarray(moltype, dtype=np.int32)
    _check(lib().pbsam_config_write(path.encode(), len(pos), _dptr(pos), _dptr(quat), mt.ctypes.data_as(_IP)))


def quat_angles(q):
    """Euler angles (theta, phi, xi) of a quaternion (w, x, y, z), as CRotCoeff::reset(CQuat)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    a = np.zeros(3)
    _check(lib().pbsam_quat_angles(_dptr(q), _dptr(a)))
    return a


def device_peaks(device=0):
    """(FP64 TFLOP/s, L2 read GB/s) of a device, timed in place."""
    f, l2 = ctypes.c_double(), ctypes.c_double()
    _check(lib().pbsam_device_peaks(device, ctypes.byref(f), ctypes.byref(l2)))
    return f.value, l2.value


class CSystem:
    """Solver context on one GPU (CSystem::initConstants + solver constants)."""

    def __init__(self, poles=10, salt=0.05, device=0, **kw):
        self.params = default_params(poles=poles, salt=salt, **kw)
        h = _P()
        _check(lib().pbsam_context_create(ctypes.byref(self.params), device, ctypes.byref(h)))
        self.handle = h
        self.types = []

    @property
    def kappa(self):
        k = ctypes.c_double()
        _check(lib().pbsam_context_kappa(self.handle, ctypes.byref(k)))
        return k.value

    def load_moltype(self, pqr, imat_dir, exp_dir, exp_name):
        t = ctypes.c_int()
        _check(lib().pbsam_moltype_load(self.handle, pqr.encode(), imat_dir.encode(), exp_dir.encode(),
                                        exp_name.encode(), ctypes.byref(t)))
        self.types.append(t.value)
        return t.value

    def create_moltype(self, centres, radii, chg_pos, chg, imats, fself, hself, hself_scale):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (centres, radii, chg_pos, chg, imats, fself, hself, hself_scale)]
        t = ctypes.c_int()
        _check(lib().pbsam_moltype_create(self.handle, len(arrs[1]), _dptr(arrs[0]), _dptr(arrs[1]), len(arrs[3]),
                                          _dptr(arrs[2]), _dptr(arrs[3]), _dptr(arrs[4]), _dptr(arrs[5]),
                                          _dptr(arrs[6]), _dptr(arrs[7]), ctypes.byref(t)))
        self.types.append(t.value)
        return t.value

    def build_imats(self, centres, radii, n_points=250000):
        """IMats of a molecule's spheres (the reference's `pbsam mat`): [n_sph, p^2, p^2] column-major."""
        centres = np.ascontiguousarray(centres, dtype=np.float64)
        radii = np.ascontiguousarray(radii, dtype=np.float64)
        P2 = self.params.poles ** 2
        out = np.zeros((len(radii), P2 * P2))
        _check(lib().pbsam_imat_build(self.handle, len(radii), _dptr(centres), _dptr(radii), n_points, _dptr(out)))
        return out

    def self_polarize(self, type_id, max_rounds=1700):
        """Self-polarized (F, H, H scale, sweeps) of a type, rounded as the reference's .exp files."""
        ns, _ = self.moltype_info(type_id)
        P2 = self.params.poles ** 2
        F = np.zeros((ns, P2))
        H = np.zeros((ns, P2))
        sc = np.zeros(ns)
        r = ctypes.c_int()
        _check(lib().pbsam_selfpol(self.handle, type_id, max_rounds, _dptr(F), _dptr(H), _dptr(sc), ctypes.byref(r)))
        return F, H, sc, r.value

    def moltype_info(self, t):
        ns, npts = ctypes.c_int(), ctypes.c_int()
        _check(lib().pbsam_moltype_info(self.handle, t, ctypes.byref(ns), ctypes.byref(npts)))
        return ns.value, npts.value

    def molecules(self, mol_types, n_systems=1):
        return Molecules(self, mol_types, n_systems)

    # single-expansion operations (CRotCoeff, CTransCoeff, CXFormA), batched over rows
    def _expan_io(self, x):
        P2 = self.params.poles ** 2
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, P2)
        return x, np.zeros_like(x)

    def expan_rotate(self, rot, p, x, with_xi=False, forward=True):
        """Rotate each row of x (packed expansions) by Euler angles rot[n][3] = theta, phi, xi."""
        x, out = self._expan_io(x)
        rot = np.ascontiguousarray(rot, dtype=np.float64).reshape(-1, 3)
        _check(lib().pbsam_expan_rotate(self.handle, len(x), rot.ctypes.data, p, int(with_xi), int(forward),
                                        x.ctypes.data, out.ctypes.data, 0))
        return out

    def expan_translate(self, args, p, x, screened=True, deriv=False):
        """Coaxial translation of each row of x; args[n][3] = rho, scale in, scale out."""
        x, out = self._expan_io(x)
        args = np.ascontiguousarray(args, dtype=np.float64).reshape(-1, 3)
        _check(lib().pbsam_expan_translate(self.handle, len(x), args.ctypes.data, p, int(screened), int(deriv),
                                           x.ctypes.data, out.ctypes.data, 0))
        return out

    def expan_reexpand(self, args, p, x, screened=True, grad=False):
        """Re-expansion of each row of x from a source to a target sphere; args[n][5] =
        target centre - source centre, source radius, target radius.  grad: also the
        x, y, z derivatives w.r.t. the target position ([n][3][p^2])."""
        x, out = self._expan_io(x)
        args = np.ascontiguousarray(args, dtype=np.float64).reshape(-1, 5)
        g = np.zeros((len(x), 3, x.shape[1])) if grad else None
        _check(lib().pbsam_expan_reexpand(self.handle, len(x), args.ctypes.data, p, int(screened), x.ctypes.data,
                                          out.ctypes.data, g.ctypes.data if grad else None, 0))
        return (out, g) if grad else out

    def close(self):
        if self.handle:
            _check(lib().pbsam_context_destroy(self.handle))
            self.handle = None


class Molecules:
    """n_systems independent copies of a list of molecules (vector<CMolecule*>)."""

    def __init__(self, ctx, mol_types, n_systems=1):
        self.ctx = ctx
        self.n_mol = len(mol_types)
        self.n_systems = n_systems
        mt = (ctypes.c_int * self.n_mol)(*mol_types)
        h = _P()
        _check(lib().pbsam_system_create(ctx.handle, n_systems, self.n_mol, mt, ctypes.byref(h)))
        self.handle = h

    def reset(self):
        _check(lib().pbsam_system_reset(self.handle))

    def set_poses(self, pos, quat):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(self.n_systems, self.n_mol, 3)
        quat = np.ascontiguousarray(quat, dtype=np.float64).reshape(self.n_systems, self.n_mol, 4)
        _check(lib().pbsam_system_set_poses(self.handle, pos.ctypes.data, quat.ctypes.data, 0))

    def set_poses_device(self, pos_ptr, quat_ptr):
        _check(lib().pbsam_system_set_poses(self.handle, pos_ptr, quat_ptr, 1))

    def compute_forces(self):
        """Returns (force[n_systems, n_mol, 3], torque[...], status[n_systems])."""
        f = np.zeros((self.n_systems, self.n_mol, 3))
        t = np.zeros((self.n_systems, self.n_mol, 3))
        st = np.zeros(self.n_systems, dtype=np.int32)
        _check(lib().pbsam_system_compute_forces(self.handle, f.ctypes.data, t.ctypes.data, st.ctypes.data, 0))
        return f, t, st

    def get_forces(self):
        """Forces, torques and statuses of the last evaluation (e.g. by a Group)."""
        f = np.zeros((self.n_systems, self.n_mol, 3))
        t = np.zeros((self.n_systems, self.n_mol, 3))
        st = np.zeros(self.n_systems, dtype=np.int32)
        _check(lib().pbsam_system_get_forces(self.handle, f.ctypes.data, t.ctypes.data, st.ctypes.data, 0))
        return f, t, st

    def compute_forces_device(self, force_ptr, torque_ptr, status_ptr):
        _check(lib().pbsam_system_compute_forces(self.handle, force_ptr, torque_ptr, status_ptr, 1))

    def compute_energy(self, lab=False):
        """Interaction energy per system on the last force evaluation's state: the
        reference's convention (computeTotalIntEnergy: unrotated centres and H), or
        with lab=True the orientation-correct lab-frame form."""
        e = np.zeros(self.n_systems)
        f = lib().pbsam_system_compute_energy_lab if lab else lib().pbsam_system_compute_energy
        _check(f(self.handle, e.ctypes.data, 0))
        return e

    def backward(self, seed=None):
        """Gradient of the lab-frame energy of the last (exact-form) evaluation, times a
        per-system seed dL/dU: (dpos[n_sys, n_mol, 3], dquat[n_sys, n_mol, 4],
        drot[n_sys, n_mol, 3]), drot the derivative for a lab-frame rotation of each
        molecule (minus its torque)."""
        dp = np.zeros((self.n_systems, self.n_mol, 3))
        dq = np.zeros((self.n_systems, self.n_mol, 4))
        dr = np.zeros((self.n_systems, self.n_mol, 3))
        sd = None if seed is None else np.ascontiguousarray(seed, dtype=np.float64).reshape(self.n_systems)
        _check(lib().pbsam_system_backward(self.handle, None if sd is None else sd.ctypes.data, dp.ctypes.data,
                                           dq.ctypes.data, dr.ctypes.data, 0))
        return dp, dq, dr

    def potential(self, points, lab=False):
        """Potential at points ([n, 3] shared, or [n_systems, n, 3]) from the state of the
        last force evaluation (CMolecule::computePotInSpace): [n_systems, n]."""
        pts = np.ascontiguousarray(points, dtype=np.float64)
        per = pts.ndim == 3
        n = pts.shape[-2]
        out = np.zeros((self.n_systems, n))
        _check(lib().pbsam_system_potential(self.handle, n, pts.ctypes.data, int(per), int(bool(lab)),
                                            out.ctypes.data, 0))
        return out

    def stats(self):
        s = np.zeros((self.n_systems, 8), dtype=np.int32)
        _check(lib().pbsam_system_stats(self.handle, s.ctypes.data_as(_IP)))
        return s

    def phase_ms(self):
        """Device ms per phase of the last evaluation (16 per system): solve, surface
        charges, numeric, analytic intra, inter LS, gradient DTA, gradient-solve
        re-expansions, total, gradient surface charges, set-up, gradient bookkeeping,
        forces; sub-phases: gradient inter, intra analytic, intra numeric, IMat products."""
        m = np.zeros((self.n_systems, 16))
        _check(lib().pbsam_system_phase_ms(self.handle, _dptr(m)))
        return m

    def set_stream(self, stream_handle):
        _check(lib().pbsam_system_set_stream(self.handle, ctypes.c_void_p(stream_handle)))

    def last_kernel_ms(self):
        m = ctypes.c_double()
        _check(lib().pbsam_system_last_kernel_ms(self.handle, ctypes.byref(m)))
        return m.value

    # ---- Brownian dynamics (CBDnam::run / CBDmulti::propagate)
    def bd_init(self, dtr, drot, mode=PBSAM_BD_NAM, seed=0, use_graph=True, **kw):
        """Start one trajectory per system from the current poses.  dtr/drot: per-molecule
        translational (A^2/ps) and rotational (rad^2/ps) diffusion coefficients; kw
        overrides fields of pbsam_bd_params (max_tries, force_dist, escape_dist, dt_min,
        dt_max, dt_ref, dt_div, ...)."""
        p = bd_params(mode, seed=seed, use_graph=int(bool(use_graph)), **kw)
        dtr = np.ascontiguousarray(dtr, dtype=np.float64)
        drot = np.ascontiguousarray(drot, dtype=np.float64)
        if dtr.shape != (self.n_mol,) or drot.shape != (self.n_mol,):
            raise ValueError("one diffusion coefficient per molecule")
        _check(lib().pbsam_system_bd_init(self.handle, ctypes.byref(p), _dptr(dtr), _dptr(drot)))
        self.bd_params = p

    def bd_run(self, n_steps):
        """Queue n_steps steps of every running trajectory (asynchronous)."""
        _check(lib().pbsam_system_bd_run(self.handle, int(n_steps)))

    def bd_set_contacts(self, defs):
        """NAM docking criteria: defs = [(partner, ncontact, [(k1, k2, dist), ...]), ...]."""
        partner = np.array([d[0] for d in defs], dtype=np.int32)
        ncon = np.array([d[1] for d in defs], dtype=np.int32)
        off = np.concatenate([[0], np.cumsum([len(d[2]) for d in defs])]).astype(np.int32)
        pairs = [pr for d in defs for pr in d[2]]
        k1 = np.array([pr[0] for pr in pairs], dtype=np.int32)
        k2 = np.array([pr[1] for pr in pairs], dtype=np.int32)
        dist = np.array([pr[2] for pr in pairs], dtype=np.float64)
        ip = lambda a: a.ctypes.data_as(_IP)
        _check(lib().pbsam_system_bd_set_contacts(self.handle, len(defs), ip(partner), ip(ncon), ip(off), ip(k1),
                                                  ip(k2), _dptr(dist)))

    def bd_set_contacts_file(self, path, sepdist):
        """NAM docking criteria from a contactdef file (sepdist <= 0: per-pair distances)."""
        _check(lib().pbsam_system_bd_set_contacts_file(self.handle, path.encode(), sepdist))

    def bd_state(self):
        """dict(pos[n_sys, n_mol, 3], quat[n_sys, n_mol, 4], status, steps, time, fevals)."""
        pos = np.zeros((self.n_systems, self.n_mol, 3))
        quat = np.zeros((self.n_systems, self.n_mol, 4))
        st = np.zeros(self.n_systems, dtype=np.int32)
        steps = np.zeros(self.n_systems, dtype=np.int32)
        tm = np.zeros(self.n_systems)
        fe = np.zeros(self.n_systems, dtype=np.int32)
        _check(lib().pbsam_system_bd_state(self.handle, pos.ctypes.data, quat.ctypes.data, st.ctypes.data,
                                           steps.ctypes.data, tm.ctypes.data, fe.ctypes.data, 0))
        return dict(pos=pos, quat=quat, status=st, steps=steps, time=tm, fevals=fe)

    def close(self):
        if self.handle:
            _check(lib().pbsam_system_destroy(self.handle))
            self.handle = None
