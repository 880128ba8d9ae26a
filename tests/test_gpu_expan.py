"""Single-expansion operations (pbsam_expan_rotate / _translate / _reexpand) against the
oracle's restatement of CRotCoeff (src/rotcoeff.cpp), CTransCoeff (src/transcoeff.cpp)
and CXFormA (src/xforms.cpp), which the golden tests pin to the reference's own
outputs.  1e-12 relative per expansion, random coefficients, the singular rotations
(theta = 0 and pi) included; and the re-expansion equal to rotation, translation and
rotation back composed through the same entry points.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
NP = 10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def ctx():
    import pbsam_b200 as pb
    return pb.CSystem(poles=NP, salt=0.05)


def rand_expan(rng, n, decay=0.6):
    x = rng.standard_normal((n, NP * NP))
    deg = np.floor(np.sqrt(np.arange(NP * NP)))
    return x * decay ** deg


def test_rotate_vs_oracle():
    rng = np.random.default_rng(11)
    c = ctx()
    try:
        n = 12
        rot = np.column_stack([rng.uniform(0, np.pi, n), rng.uniform(-np.pi, np.pi, n), rng.uniform(-np.pi, np.pi, n)])
        rot[0, 0], rot[1, 0] = 0.0, np.pi          # singular: along +z and -z
        x = rand_expan(rng, n)
        for p in (NP, 6):
            for with_xi in (0, 1):
                for fwd in (1, 0):
                    g = c.expan_rotate(rot, p, x, with_xi=with_xi, forward=fwd)
                    o = oracle.expan_op(NP, c.kappa, 0, rot, p, with_xi, fwd, x)
                    assert rel(g, o) < 1e-12, (p, with_xi, fwd, rel(g, o))
                    assert np.all(g[:, p * p:] == 0.0)
        # forward then back is the identity
        y = c.expan_rotate(rot, NP, c.expan_rotate(rot, NP, x, forward=True), forward=False)
        assert rel(y, x) < 1e-12
    finally:
        c.close()


def test_translate_vs_oracle():
    rng = np.random.default_rng(12)
    c = ctx()
    try:
        n = 10
        args = np.column_stack([rng.uniform(6.0, 40.0, n), rng.uniform(3.0, 6.0, n), rng.uniform(3.0, 6.0, n)])
        x = rand_expan(rng, n)
        for p in (NP, 7):
            for screened in (1, 0):
                for deriv in (0, 1):
                    g = c.expan_translate(args, p, x, screened=screened, deriv=deriv)
                    o = oracle.expan_op(NP, c.kappa, 1, args, p, screened, deriv, x)
                    assert rel(g, o) < 1e-12, (p, screened, deriv, rel(g, o))
    finally:
        c.close()


def test_reexpand_and_gradient_vs_oracle():
    rng = np.random.default_rng(13)
    c = ctx()
    try:
        n = 10
        d = rng.standard_normal((n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        d *= rng.uniform(8.0, 40.0, (n, 1))
        d[0] = [0.0, 0.0, 15.0]                     # singular rotations
        d[1] = [0.0, 0.0, -12.0]
        args = np.column_stack([d, rng.uniform(3.0, 6.0, n), rng.uniform(3.0, 6.0, n)])
        x = rand_expan(rng, n)
        for p in (NP, 5):
            g, gg = c.expan_reexpand(args, p, x, screened=True, grad=True)
            o, og = oracle.expan_op(NP, c.kappa, 2, args, p, 1, 0, x, grad=True)
            assert rel(g, o) < 1e-12 and rel(gg, og) < 1e-11, (p, rel(g, o), rel(gg, og))
            gF = c.expan_reexpand(args, p, x, screened=False)
            oF = oracle.expan_op(NP, c.kappa, 2, args, p, 0, 0, x)
            assert rel(gF, oF) < 1e-12, (p, rel(gF, oF))
    finally:
        c.close()


def test_reexpand_is_rotate_translate_rotate_back():
    """CXFormA::xformH = rotate(theta, phi of P, xi = pi) forward, translate by |P|,
    rotate back (src/xforms.cpp:122-132), through the separate entry points."""
    import pbsam_b200 as pb
    rng = np.random.default_rng(14)
    c = ctx()
    try:
        n = 6
        d = rng.standard_normal((n, 3)) * 15.0
        rs, rt = rng.uniform(3.0, 6.0, n), rng.uniform(3.0, 6.0, n)
        x = rand_expan(rng, n)
        rho = np.linalg.norm(d, axis=1)
        theta = np.arccos(d[:, 2] / rho)
        phi = np.arctan2(d[:, 1], d[:, 0])
        rot = np.column_stack([theta, phi, np.full(n, np.pi)])
        a = c.expan_rotate(rot, NP, x, forward=True)
        b = c.expan_translate(np.column_stack([rho, rs, rt]), NP, a, screened=True)
        y = c.expan_rotate(rot, NP, b, forward=False)
        z = c.expan_reexpand(np.column_stack([d, rs, rt]), NP, x, screened=True)
        assert rel(y, z) < 1e-12, rel(y, z)
        # the Euler angles of a quaternion are those of CRotCoeff::reset(CQuat)
        q = np.array([0.8, 0.2, -0.4, 0.4])
        ang = pb.quat_angles(q)
        assert np.all(np.isfinite(ang)) and 0.0 <= ang[0] <= np.pi
    finally:
        c.close()
