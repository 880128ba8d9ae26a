"""Python access to the CPU oracle (test infrastructure only).

``liboracle()`` loads the restated oracle (oracle/pbsam_oracle.cpp, built into
oracle/libpbsam_oracle.so by ``build()``); ``run_spec`` writes a spec file in
the force-harness format and runs it; ``parse`` reads the harness/oracle output
format (KAPPA / FRAME / FORCE / TORQUE / ENERGY / per-sphere dumps).
Only tests, the smoke check and the bench's CPU-baseline leg use this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libpbsam_oracle.so")
_lib = None

DEFAULT_TOL = (1e-2, 1e-8, 100, 1000)   # MAX_POLAR_DEV, SOLVE_TOL, SOLVE_MAX_CT, MAX_POL_ROUNDS
TIGHT_TOL = (1e-7, 1e-26, 400, 1000)


def build(force=False):
    """Compile the restated oracle (g++, no GPU needed)."""
    src = os.path.join(HERE, "pbsam_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", LIB, src])
    return LIB


PREP_LIB = os.path.join(HERE, "libpbsam_prep.so")
_prep = None


def build_prep(force=False):
    """Compile the multi-threaded preparation library (oracle/pbsam_prep.cpp: the
    oracle plus OpenMP IMat builder and self-polarization; no GPU needed)."""
    srcs = [os.path.join(HERE, f) for f in ("pbsam_prep.cpp", "pbsam_oracle.cpp")]
    if force or not os.path.exists(PREP_LIB) or any(os.path.getmtime(PREP_LIB) < os.path.getmtime(f) for f in srcs):
        subprocess.check_call(["g++", "-std=c++17", "-O3", "-mavx2", "-mfma", "-fopenmp", "-fPIC", "-shared", "-o", PREP_LIB,
                               srcs[0]])
    return PREP_LIB


def libprep():
    global _prep
    if _prep is None:
        build_prep()
        _prep = ctypes.CDLL(PREP_LIB)
        d = ctypes.POINTER(ctypes.c_double)
        _prep.pbsam_prep_imat.argtypes = [ctypes.c_int, ctypes.c_int, d, d, ctypes.c_int, d]
        _prep.pbsam_prep_imat.restype = ctypes.c_int
        _prep.pbsam_prep_selfpol.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, d, d,
                                             ctypes.c_int, d, d, d, ctypes.c_int, d, d, d,
                                             ctypes.POINTER(ctypes.c_int)]
        _prep.pbsam_prep_selfpol.restype = ctypes.c_int
    return _prep


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def prep_imats(poles, centres, radii, n_points=250000):
    """IMats of a molecule's spheres on the host cores ([n_sph, p^4], column-major as
    imat.sp<k>.out.bin holds them): the reference's `pbsam mat`."""
    cen = np.ascontiguousarray(centres, dtype=np.float64)
    rad = np.ascontiguousarray(radii, dtype=np.float64)
    out = np.zeros((len(rad), poles ** 4))
    if libprep().pbsam_prep_imat(poles, len(rad), _dp(cen), _dp(rad), n_points, _dp(out)) != 0:
        raise RuntimeError("pbsam_prep_imat failed")
    return out


def prep_selfpol(poles, centres, radii, chg_pos, chg, imats, salt=0.05, idiel=4.0, max_rounds=1700):
    """Self-polarized (F, H, H scale, sweeps) on the host cores, rounded as the
    reference's .exp files: the reference's `pbsam spol`."""
    cen = np.ascontiguousarray(centres, dtype=np.float64)
    rad = np.ascontiguousarray(radii, dtype=np.float64)
    qp = np.ascontiguousarray(chg_pos, dtype=np.float64).reshape(-1, 3)
    q = np.ascontiguousarray(chg, dtype=np.float64)
    im = np.ascontiguousarray(imats, dtype=np.float64)
    n, P2 = len(rad), poles * poles
    F, H, sc = np.zeros((n, P2)), np.zeros((n, P2)), np.zeros(n)
    r = ctypes.c_int()
    if libprep().pbsam_prep_selfpol(poles, salt, idiel, n, _dp(cen), _dp(rad), len(q), _dp(qp), _dp(q), _dp(im),
                                    max_rounds, _dp(F), _dp(H), _dp(sc), ctypes.byref(r)) != 0:
        raise RuntimeError("pbsam_prep_selfpol failed")
    return F, H, sc, r.value


def liboracle():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        _lib.pbsam_oracle_run.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        _lib.pbsam_oracle_run.restype = ctypes.c_int
    return _lib


def expan_op(np_, kappa, op, args, p, f1, f2, x, grad=False):
    """The oracle's single-expansion operations (pbsam_oracle_expan): op 0 rotate,
    1 translate, 2 re-expand; x [n][np_^2].  Returns out (and the gradient [n][3][np_^2])."""
    lib = liboracle()
    x = np.ascontiguousarray(x, dtype=np.float64)
    a = np.ascontiguousarray(args, dtype=np.float64)
    n = x.shape[0]
    out = np.zeros_like(x)
    g = np.zeros((n, 3, np_ * np_)) if grad else None
    r = lib.pbsam_oracle_expan(ctypes.c_int(np_), ctypes.c_double(kappa), ctypes.c_int(op), ctypes.c_int(n), _dp(a),
                               ctypes.c_int(p), ctypes.c_int(f1), ctypes.c_int(f2), _dp(x), _dp(out),
                               _dp(g) if grad else None)
    if r != 0:
        raise RuntimeError("pbsam_oracle_expan failed")
    return (out, g) if grad else out


def write_spec(path, moltypes, frames, salt=0.05, idiel=4.0, poles=10, tol=DEFAULT_TOL, dump=0, energy=1,
               backward=0, nograd=0, exact=0, potpoints=(), potlab=0):
    """moltypes: list of (pqr, imatdir, expdir, expname); frames: list of lists
    of (type, pos[3], quat[4]).  energy 2 adds the lab-frame energy; backward 1 its
    gradient (DPOS / DROT); nograd 1 leaves out the reference's gradient solves."""
    with open(path, "w") as fh:
        fh.write("salt %r\nidiel %r\npoles %d\ndump %d\nenergy %d\n" % (salt, idiel, poles, dump, energy))
        # options of the oracle alone (the reference harnesses do not read them)
        for key, val in (("backward", backward), ("nograd", nograd), ("exact", exact), ("potlab", potlab)):
            if val:
                fh.write("%s %d\n" % (key, val))
        for pt in potpoints:   # potential at points (both the oracle and the reference harness)
            fh.write("potpoint %.17g %.17g %.17g\n" % tuple(pt))
        fh.write("tol %r %r %d %d\n" % tuple(tol))
        for mt in moltypes:
            fh.write("moltype %s %s %s %s\n" % tuple(mt))
        for fr in frames:
            fh.write("frame\n")
            for (t, pos, q) in fr:
                fh.write("mol %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n" % tuple([t] + list(pos) + list(q)))


BD_DEFAULT = dict(max_tries=500, force_dist=100.0, escape_dist=500.0, dt_min=2.0, dt_max=1e300, dt_ref=5.0,
                  dt_div=15.0)


def write_bd_spec(path, moltypes, frame, mode, n_steps, seed, system, dtr, drot, salt=0.05, idiel=4.0, poles=10,
                  tol=DEFAULT_TOL, noise=None, **bdp):
    """Brownian dynamics from one frame's poses (the oracle's BD mode): n_steps steps of
    trajectory `system` (the noise counter's system word) with the given seed."""
    p = dict(BD_DEFAULT)
    if mode == 1:
        p["dt_ref"] = 10.0
    p.update(bdp)
    write_spec(path, moltypes, [frame], salt=salt, idiel=idiel, poles=poles, tol=tol, energy=0)
    with open(path, "a") as fh:
        fh.write("bd %d %d %d %d\n" % (mode, n_steps, seed, system))
        fh.write("bdp %d %r %r %r %r %r %r\n" % (p["max_tries"], p["force_dist"], p["escape_dist"], p["dt_min"],
                                                  p["dt_max"], p["dt_ref"], p["dt_div"]))
        for a, b in zip(dtr, drot):
            fh.write("bddiff %r %r\n" % (a, b))
        if noise is not None:       # (kind, order): kind 1 = the reference's drand48 stream
            fh.write("bdnoise %d %d\n" % tuple(noise))


def run_bd_spec(spec, out):
    """Returns per step dict(steps, status, fevals, time, pos[n,3], quat[n,4])."""
    rc = liboracle().pbsam_oracle_run(spec.encode(), out.encode())
    if rc != 0:
        raise RuntimeError("oracle failed with status %d" % rc)
    steps = []
    with open(out) as fh:
        for ln in fh:
            t = ln.split()
            if t and t[0] == "BDSTEP":
                steps.append(dict(steps=int(t[1]), status=int(t[2]), fevals=int(t[3]), time=float(t[4]), pos={},
                                  quat={}))
            elif t and t[0] == "POSE":
                v = [float(x) for x in t[2:]]
                steps[-1]["pos"][int(t[1])] = v[:3]
                steps[-1]["quat"][int(t[1])] = v[3:]
    for s in steps:
        n = len(s["pos"])
        s["pos"] = np.array([s["pos"][i] for i in range(n)])
        s["quat"] = np.array([s["quat"][i] for i in range(n)])
    return steps


def ref_bd_harness(poles=6, mode="default"):
    """The reference's own NAM driver with a fixed drand48 seed (oracle/_ref, built by
    build_ref.build_bd_harness), or None when it has not been built."""
    p = os.path.join(HERE, "_ref", "p%d_%s" % (poles, mode), "bd_harness")
    return p if os.path.exists(p) else None


def ref_bdm_harness(poles=6, mode="default"):
    """The reference's own multi-molecule driver (CBDmulti) with a fixed drand48 seed."""
    p = os.path.join(HERE, "_ref", "p%d_%s" % (poles, mode), "bdm_harness")
    return p if os.path.exists(p) else None


def philox(counter, key):
    """One Philox4x64-10 block of the oracle's noise generator."""
    lib = liboracle()
    c = (ctypes.c_ulonglong * 4)(*[int(x) for x in counter])
    lib.pbsam_oracle_philox.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_ulonglong, ctypes.c_ulonglong]
    lib.pbsam_oracle_philox(c, int(key[0]), int(key[1]))
    return [int(x) for x in c]


def run_spec(spec, out):
    rc = liboracle().pbsam_oracle_run(spec.encode(), out.encode())
    if rc != 0:
        raise RuntimeError("oracle failed with status %d" % rc)
    return parse(out)


def parse(path):
    """Returns a list of frames: dict(ok, force[n,3], torque[n,3], energy, dump{tag:{(i,k):array}})."""
    frames = []
    cur = None
    with open(path) as fh:
        for ln in fh:
            t = ln.split()
            if not t:
                continue
            if t[0] == "FRAME":
                cur = dict(ok=int(t[2]) == 1, force={}, torque={}, energy=None, dump={}, info=t[3:])
                frames.append(cur)
            elif t[0] == "FORCE":
                cur["force"][int(t[1])] = [float(x) for x in t[2:5]]
            elif t[0] == "TORQUE":
                cur["torque"][int(t[1])] = [float(x) for x in t[2:5]]
            elif t[0] == "ENERGY":
                cur["energy"] = float(t[1])
            elif t[0] == "ENERGYLAB":
                cur["energy_lab"] = float(t[1])
            elif t[0] == "POT":
                cur.setdefault("pot", {})[int(t[1])] = float(t[2])
            elif t[0] in ("DPOS", "DROT"):
                cur.setdefault(t[0].lower(), {})[int(t[1])] = [float(x) for x in t[2:5]]
            elif t[0] == "KAPPA":
                pass
            elif cur is not None:
                cur["dump"].setdefault(t[0], {})[(int(t[1]), int(t[2]))] = np.array([float(x) for x in t[4:]])
    for fr in frames:
        n = len(fr["force"])
        fr["force"] = np.array([fr["force"][i] for i in range(n)]).reshape(-1, 3)
        fr["torque"] = np.array([fr["torque"][i] for i in range(n)]).reshape(-1, 3)
        if "pot" in fr:
            fr["pot"] = np.array([fr["pot"][i] for i in range(len(fr["pot"]))])
        for key in ("dpos", "drot"):
            if key in fr:
                fr[key] = np.array([fr[key][i] for i in range(len(fr[key]))]).reshape(-1, 3)
    return frames


def golden_moltypes(case_dir):
    return [(os.path.join(case_dir, "mol%s.pqr" % t), os.path.join(case_dir, "im" + t),
             os.path.join(case_dir, "exp" + t), "mol%s.0" % t) for t in ("A", "B")]


def golden_frames(poses_entry):
    return [[(m["type"], m["pos"], m["quat"]) for m in poses_entry]]
