#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/<case>/ from the reference.

Runs the reference PB-SAM binaries built by ``oracle/build_ref.py``:
  1. seeded synthetic molecules (pbsam_b200.synth) written as PQR;
  2. ``pbsam mat``  -> imat.sp<k>.out.bin per sphere (src/selfp_makemat.cpp:129-183);
  3. ``pbsam spol`` -> <name>.0.<k>.{F,H}.exp   (src/selfp_makemat.cpp:37-118), 1 thread;
  4. the force harness (oracle/ref_harness.cpp) at seeded poses, once per pose in a
     fresh process (the reference carries state between calls), plus one
     multi-frame run that pins the state carried between consecutive calls.
Both the ``default`` (reference tolerances) and ``tight`` builds are run on the
same inputs.  Needs the reference sources; the committed fixtures do not.

Usage: python tests/golden/make_golden.py [case ...]
"""
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "pb-sam_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
from pbsam_b200 import synth  # noqa: E402

CASES = {
    # config 0: 2 x 8 spheres, r ~ U(3,6), 300 charges q ~ U(-0.6,0.6) net +2/-2, p = 10
    "cfg0": dict(poles=10, salt=0.05, idiel=4.0,
                 mols=[dict(n_sph=8, r=(3, 6), n_q=300, q_amp=0.6, net=2.0, seed=1),
                       dict(n_sph=8, r=(3, 6), n_q=300, q_amp=0.6, net=-2.0, seed=2)],
                 gaps=[1.0, 2.5, 4.0, 7.0, 9.5, 30.0], centre_dist=[40.0], pose_seed=7,
                 seq_frames=3),
    # small, fast case for the CPU test suite: 2 x 4 spheres, p = 6
    "tiny": dict(poles=6, salt=0.1, idiel=4.0,
                 mols=[dict(n_sph=4, r=(3, 5), n_q=60, q_amp=0.6, net=1.0, seed=11),
                       dict(n_sph=4, r=(3, 5), n_q=60, q_amp=0.6, net=-1.0, seed=12)],
                 gaps=[1.5, 5.0, 20.0], centre_dist=[], pose_seed=17, seq_frames=3),
}


def refbin(poles, mode, name):
    return os.path.join(REPO, "oracle", "_ref", "p%d_%s" % (poles, mode), name)


def run(cmd, cwd, threads=1):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    with open(os.path.join(cwd, "log.txt"), "a") as log:
        subprocess.check_call(cmd, cwd=cwd, stdout=log, stderr=subprocess.STDOUT, env=env)


def write_spec(path, case, frames, dump=0):
    with open(path, "w") as fh:
        fh.write("salt %r\nidiel %r\ndump %d\nenergy 1\n" % (case["salt"], case["idiel"], dump))
        for t, name in enumerate(["A", "B"]):
            fh.write("moltype mol%s.pqr im%s exp%s mol%s.0\n" % (name, name, name, name))
        for fr in frames:
            fh.write("frame\n")
            for m in fr:
                fh.write("mol %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n" % tuple(
                    [m["type"]] + list(m["pos"]) + list(m["quat"])))


def make_case(name):
    case = CASES[name]
    p = case["poles"]
    out = os.path.join(HERE, name)
    if os.path.isdir(out):
        shutil.rmtree(out)
    os.makedirs(out)
    for t, (mspec, tag) in enumerate(zip(case["mols"], ["A", "B"])):
        m = synth.make_molecule(mspec["n_sph"], mspec["r"][0], mspec["r"][1], mspec["n_q"],
                                mspec["q_amp"], mspec["net"], seed=mspec["seed"])
        synth.write_pqr(m, os.path.join(out, "mol%s.pqr" % tag))
        im = os.path.join(out, "im" + tag)
        ex = os.path.join(out, "exp" + tag)
        os.makedirs(im)
        os.makedirs(ex)
        run([refbin(p, "default", "pbsam"), "mat", "8", repr(case["salt"]), "../mol%s.pqr" % tag],
            im, threads=8)
        run([refbin(p, "default", "pbsam"), "spol", "1", repr(case["salt"]), "../mol%s.pqr" % tag,
             "../im" + tag, "mol" + tag], ex, threads=1)
        os.remove(os.path.join(im, "log.txt"))
        os.remove(os.path.join(ex, "log.txt"))
    A = synth.read_pqr(os.path.join(out, "molA.pqr"))
    B = synth.read_pqr(os.path.join(out, "molB.pqr"))
    rng = np.random.default_rng(case["pose_seed"])
    poses = []
    for g in case["gaps"]:
        qa, qb, ax = synth.random_quat(rng), synth.random_quat(rng), synth.random_axis(rng)
        d = synth.place_at_gap(A, qa, B, qb, ax, g)
        poses.append(dict(gap=g, frame=[dict(type=0, pos=[0.0, 0.0, 0.0], quat=list(qa)),
                                        dict(type=1, pos=list(d * ax), quat=list(qb))]))
    for d in case["centre_dist"]:
        qa, qb, ax = synth.random_quat(rng), synth.random_quat(rng), synth.random_axis(rng)
        poses.append(dict(centre_dist=d, frame=[dict(type=0, pos=[0.0, 0.0, 0.0], quat=list(qa)),
                                                dict(type=1, pos=list(d * ax), quat=list(qb))]))
    # a short sequence of nearby frames in one process (state carried between calls)
    base = poses[1]["frame"]
    seq = [base]
    for k in range(1, case["seq_frames"]):
        step = rng.normal(scale=0.3, size=3)
        fr = json.loads(json.dumps(seq[-1]))
        fr[1]["pos"] = list(np.array(fr[1]["pos"]) + step)
        seq.append(fr)
    with open(os.path.join(out, "poses.json"), "w") as fh:
        json.dump(dict(poses=poses, sequence=seq, salt=case["salt"], idiel=case["idiel"],
                       poles=p), fh, indent=1)
    for mode in ["default", "tight"]:
        md = os.path.join(out, "ref_" + mode)
        os.makedirs(md)
        for k, ps in enumerate(poses):
            spec = os.path.join(out, "spec.txt")
            write_spec(spec, case, [ps["frame"]], dump=1 if name == "tiny" else 0)
            run([refbin(p, mode, "harness"), "spec.txt", os.path.join(md, "pose%d.txt" % k)], out)
        write_spec(os.path.join(out, "spec.txt"), case, seq)
        run([refbin(p, mode, "harness"), "spec.txt", os.path.join(md, "sequence.txt")], out)
        os.remove(os.path.join(out, "spec.txt"))
    os.remove(os.path.join(out, "log.txt"))
    print("wrote", out)


def main(argv):
    names = argv or list(CASES)
    import build_ref
    for n in names:
        p = CASES[n]["poles"]
        for mode in ["default", "tight"]:
            if not os.path.exists(refbin(p, mode, "harness")):
                build_ref.build_variant(p, mode)
        make_case(n)


if __name__ == "__main__":
    main(sys.argv[1:])
