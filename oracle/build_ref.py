#!/usr/bin/env python3
"""Build recipe for the reference PB-SAM binaries used as the pinning oracle.

This is test infrastructure only.  It compiles the reference C++ sources where
they lie (``<reference>/src``) into ``oracle/_ref/`` (git-ignored) so that the
restated oracle and the CUDA drop-in can be checked against the reference's own
output.  Nothing here is shipped or called by the product path.

The reference cannot be compiled verbatim with gcc 13:
  * ``mkl.h`` is absent: a small col-major cblas shim (``oracle/ref_shim/mkl.h``,
    own code) provides ``cblas_dgemm``/``cblas_dgemv`` with plain GEMM semantics;
  * eight non-void functions fall off the end (undefined behaviour that makes
    -O2 builds crash); each gets the ``return`` its callers rely on;
  * ``CRotCoeff::m_zeta`` is declared ``[2N][2N-1]`` but ``initConstants``
    writes column ``2N-1`` (src/rotcoeff.cpp:18-20): the table is padded to 2N.
The patched copies are written under ``oracle/_ref/src_p<P>_<mode>/`` at build
time (git-ignored build output); nothing from the reference is committed.

Variants (``N_POLES`` is a compile-time macro in the reference, src/expansion.h:5-9):
  default : reference tolerances (src/molecule.cpp:6-13, src/expcenter.cpp:16-22), -O2
  tight   : MAX_POLAR_DEV 1e-7, SOLVE_TOL 1e-26, SOLVE_MAX_CT 400, -O2
  fast    : reference tolerances, the reference Makefile flags
            (-O3 -ffast-math -funroll-loops, src/Makefile:5-7) -- the timed CPU baseline

Usage: python oracle/build_ref.py [--poles 10,30] [--modes default,tight,fast]
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference source tree: PBSAM_REFERENCE_SRC, else a checkout named "reference"
# beside the repository
REF_SRC = os.environ.get("PBSAM_REFERENCE_SRC",
                         os.path.normpath(os.path.join(HERE, "..", "..", "reference", "src")))
OUT = os.path.join(HERE, "_ref")

# reference translation units needed by the pbsam driver and by the force harness
LIB_SOURCES = [
    "getmemory.cpp", "expansion.cpp", "triexpan.cpp", "expcenter.cpp",
    "rotcoeff.cpp", "transcoeff.cpp", "xforms.cpp", "lautil.cpp",
    "readutil.cpp", "molecule.cpp", "moldynamics.cpp", "system.cpp",
    "contact.cpp",
]

# (file, old, new): return-only patches and the m_zeta padding
PATCHES = [
    ("expansion.h",
     "static_cast<CExpan &>(*this) = static_cast<const CExpan&>(M);\n\t}",
     "static_cast<CExpan &>(*this) = static_cast<const CExpan&>(M);\n\t\treturn *this;\n\t}"),
    ("expcenter.cpp",
     "  solveSurfaceCharges(m_F, m_H, false);\n}",
     "  return solveSurfaceCharges(m_F, m_H, false);\n}"),
    ("expcenter.cpp",
     "  m_F = M.m_F;\n}",
     "  m_F = M.m_F;\n  return *this;\n}"),
    ("expcenter.h",
     "computeTorqueOn_0(int i) const { /* later, for fixed charge */};",
     "computeTorqueOn_0(int i) const { return CPnt(); };"),
    ("xforms.h",
     "virtual int getOrder() const {};",
     "virtual int getOrder() const { return 0; };"),
    ("contact.h",
     "\t\tm_contactlist = m.getContactList();\n\t}",
     "\t\tm_contactlist = m.getContactList();\n\t\treturn *this;\n\t}"),
    ("contactRigid.h",
     "\t\tm_bDocked = m.getBDocked();\n\t}",
     "\t\tm_bDocked = m.getBDocked();\n\t\treturn *this;\n\t}"),
    ("transform.h",
     "\t\t}\n\t\t//out<<endl;\n\t}\n}",
     "\t\t}\n\t\t//out<<endl;\n\t}\n\treturn out;\n}"),
    ("rotcoeff.h",
     "static REAL m_zeta[N_POLES*2][2*N_POLES-1];",
     "static REAL m_zeta[N_POLES*2][2*N_POLES];"),
    ("rotcoeff.cpp",
     "REAL CRotCoeff::m_zeta[N_POLES*2][2*N_POLES-1];",
     "REAL CRotCoeff::m_zeta[N_POLES*2][2*N_POLES];"),
]

TIGHT = [
    ("molecule.cpp", "#define MAX_POLAR_DEV (1e-2)", "#define MAX_POLAR_DEV (1e-7)"),
    ("expcenter.cpp", "const double SOLVE_TOL = (1e-8);", "const double SOLVE_TOL = (1e-26);"),
    ("expcenter.cpp", "const int SOLVE_MAX_CT = 100;", "const int SOLVE_MAX_CT = 400;"),
]


# self-polarization capped at 25 sweeps (to trace a molecule whose sweeps do not converge)
CAP25 = [
    ("molecule.cpp", "const int MAX_POL_ROUNDS_SELF = 1700;", "const int MAX_POL_ROUNDS_SELF = 25;"),
]


def _replace_once(text, old, new, fname):
    n = text.count(old)
    if n != 1:
        raise RuntimeError("patch site in %s found %d times: %r" % (fname, n, old[:60]))
    return text.replace(old, new)


def stage_sources(poles, mode):
    dst = os.path.join(OUT, "src_p%d_%s" % (poles, mode))
    if os.path.isdir(dst):
        shutil.rmtree(dst)
    os.makedirs(dst)
    for f in os.listdir(REF_SRC):
        if f.endswith(".cpp") or f.endswith(".h"):
            shutil.copy(os.path.join(REF_SRC, f), os.path.join(dst, f))
            os.chmod(os.path.join(dst, f), 0o644)
    patches = list(PATCHES)
    patches.append(("expansion.h", "#define N_POLES 15", "#define N_POLES %d" % poles))
    if mode == "tight":
        patches += TIGHT
    if mode == "cap25":
        patches += CAP25
    for fname, old, new in patches:
        path = os.path.join(dst, fname)
        with open(path) as fh:
            text = fh.read()
        text = _replace_once(text, old, new, fname)
        with open(path, "w") as fh:
            fh.write(text)
    shutil.copy(os.path.join(HERE, "ref_shim", "mkl.h"), os.path.join(dst, "mkl.h"))
    return dst


def build_variant(poles, mode, jobs=8):
    src = stage_sources(poles, mode)
    bindir = os.path.join(OUT, "p%d_%s" % (poles, mode))
    os.makedirs(bindir, exist_ok=True)
    if mode == "fast":
        opt = ["-O3", "-ffast-math", "-funroll-loops", "-m64"]
    else:
        opt = ["-O2"]
    cxx = ["g++", "-std=gnu++11", "-fopenmp", "-fpermissive", "-w",
           "-D__MKL", "-D__OMP", "-D__ACCURATE__"] + opt + ["-I" + src]
    objs = []
    procs = []
    for f in LIB_SOURCES + ["selfp_makemat.cpp"]:
        o = os.path.join(bindir, f.replace(".cpp", ".o"))
        procs.append((subprocess.Popen(cxx + ["-c", os.path.join(src, f), "-o", o]), f))
        if f != "selfp_makemat.cpp":
            objs.append(o)
        if len(procs) >= jobs:
            p, name = procs.pop(0)
            if p.wait() != 0:
                raise RuntimeError("compile failed: " + name)
    h = os.path.join(bindir, "ref_harness.o")
    procs.append((subprocess.Popen(cxx + ["-c", os.path.join(HERE, "ref_harness.cpp"), "-o", h]),
                  "ref_harness.cpp"))
    for p, name in procs:
        if p.wait() != 0:
            raise RuntimeError("compile failed: " + name)
    subprocess.check_call(cxx + objs + [os.path.join(bindir, "selfp_makemat.o"), "-o",
                                        os.path.join(bindir, "pbsam")])
    subprocess.check_call(cxx + objs + [h, "-o", os.path.join(bindir, "harness")])
    build_bd_harness(poles, mode)


def build_bd_harness(poles, mode):
    """The reference's own NAM driver (CBDnam, src/BDnam.cpp) with a fixed drand48
    seed, linked from the staged sources and the objects of build_variant."""
    src = os.path.join(OUT, "src_p%d_%s" % (poles, mode))
    bindir = os.path.join(OUT, "p%d_%s" % (poles, mode))
    if mode == "fast":
        opt = ["-O3", "-ffast-math", "-funroll-loops", "-m64"]
    else:
        opt = ["-O2"]
    cxx = ["g++", "-std=gnu++11", "-fopenmp", "-fpermissive", "-w",
           "-D__MKL", "-D__OMP", "-D__ACCURATE__"] + opt + ["-I" + src]
    objs = [os.path.join(bindir, f.replace(".cpp", ".o")) for f in LIB_SOURCES]
    bdo = os.path.join(bindir, "BDnam.o")
    subprocess.check_call(cxx + ["-c", os.path.join(src, "BDnam.cpp"), "-o", bdo])
    ho = os.path.join(bindir, "ref_bd_harness.o")
    subprocess.check_call(cxx + ["-c", os.path.join(HERE, "ref_bd_harness.cpp"), "-o", ho])
    subprocess.check_call(cxx + objs + [bdo, ho, "-o", os.path.join(bindir, "bd_harness")])
    # the multi-molecule driver (CBDmulti, src/BDmulti.cpp)
    bmo = os.path.join(bindir, "BDmulti.o")
    subprocess.check_call(cxx + ["-c", os.path.join(src, "BDmulti.cpp"), "-o", bmo])
    hmo = os.path.join(bindir, "ref_bdm_harness.o")
    subprocess.check_call(cxx + ["-c", os.path.join(HERE, "ref_bdm_harness.cpp"), "-o", hmo])
    subprocess.check_call(cxx + objs + [bmo, hmo, "-o", os.path.join(bindir, "bdm_harness")])
    return bindir


def available():
    return os.path.isdir(REF_SRC)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--poles", default="10")
    ap.add_argument("--modes", default="default,tight,fast")
    a = ap.parse_args(argv)
    if not available():
        print("reference sources not present; nothing to build")
        return 0
    for p in [int(x) for x in a.poles.split(",") if x]:
        for m in [x for x in a.modes.split(",") if x]:
            d = build_variant(p, m)
            print("built", d)
    return 0


if __name__ == "__main__":
    sys.exit(main())
