"""The C-ABI library loads and exports every entry point include/pbsam_b200.h declares.

No compute calls here (no GPU needed): on a machine without a usable CUDA driver
the context creation must fail with an error code, not crash.
"""
import ctypes
import os
import re

import pytest

import pbsam_b200 as pb
from conftest import REPO

HEADER = os.path.join(REPO, "include", "pbsam_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pbsam_[a-z_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "pbsam_system_compute_forces" in syms
    assert "pbsam_moltype_load" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    if not os.path.exists(pb.LIB_PATH):
        pytest.skip("CUDA library not built")
    lib = ctypes.CDLL(pb.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    assert set(declared_symbols()) == set(pb.SIGNATURES)


def test_defaults_match_reference_constants():
    if not os.path.exists(pb.LIB_PATH):
        pytest.skip("CUDA library not built")
    p = pb.default_params()
    assert p.poles == 10 and p.solve_max_ct == 100 and p.max_pol_rounds == 1000
    assert p.max_polar_dev == 1e-2 and p.solve_tol == 1e-8
    assert (p.inter_cutoff, p.interact_cutoff, p.intra_cutoff, p.min_sep_numeric) == (10, 100, 30, 5)
    assert p.num_points_x == 10000


def test_context_without_gpu_fails_cleanly():
    if not os.path.exists(pb.LIB_PATH):
        pytest.skip("CUDA library not built")
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(pb.PbsamError):
        pb.CSystem(poles=6)


def test_bd_defaults_match_reference_drivers():
    """pbsam_bd_params_default gives the constants of the reference's drivers
    (src/BDnam.h:10-25, src/BDnam.cpp:409-417, src/BDmulti.cpp:13, 451, 511-517);
    no GPU needed."""
    if not os.path.exists(pb.LIB_PATH):
        pytest.skip("CUDA library not built")
    nam = pb.bd_params(pb.PBSAM_BD_NAM)
    multi = pb.bd_params(pb.PBSAM_BD_MULTI)
    assert nam.max_tries == 500 and nam.force_dist == 100.0 and nam.escape_dist == 500.0
    assert nam.dt_min == 2.0 and nam.dt_ref == 5.0 and nam.dt_div == 15.0 and nam.dt_max >= 1e300
    assert multi.dt_ref == 10.0 and multi.dt_min == 2.0
    assert nam.fact_tr == 5.604586e2 and nam.coul_k == 2.30708e-18
    assert abs(nam.ikbt - 1.0 / (1.3806503e-23 * 298.15)) <= 1e-12 * nam.ikbt
    assert nam.noise == pb.PBSAM_BD_NOISE_PHILOX and nam.use_graph == 1
