"""C-ABI library: loads and exports every symbol of include/pdcs.h (no compute, CPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from pdcs_b200 import build, capi, problems, solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "pdcs.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(pdcs_\w+)\s*\(", text, re.M)))


def test_header_declares_expected_entry_points():
    assert set(capi.EXPORTS) == set(declared_symbols())


def test_library_builds_and_exports_all_symbols():
    build.build()
    lib = ctypes.CDLL(capi.LIB_PATH)
    for sym in declared_symbols():
        assert hasattr(lib, sym), sym


def test_struct_sizes_match_c_layout():
    # 8-byte aligned structs with explicit padding fields
    assert ctypes.sizeof(capi.PdcsProblem) % 8 == 0
    assert ctypes.sizeof(capi.PdcsOptions) % 8 == 0
    assert ctypes.sizeof(capi.PdcsResult) % 8 == 0


def test_default_options_roundtrip():
    lib = capi.load()
    o = capi.PdcsOptions()
    assert lib.pdcs_default_options(ctypes.byref(o)) == 0
    assert o.rescaling_method == 3 and o.max_outer_iter == 10000 and o.max_inner_iter == 500000
    assert o.abs_tol == 1e-6 and o.rel_tol == 1e-6 and o.check_terminate_freq == 2000
    assert o.use_duality_gap_restart == 1 and o.use_kkt_restart == 0
    assert capi.load().pdcs_version().startswith(b"pdcs_b200")


def test_validation_errors_mirror_reference():
    p = problems.mixed_small()
    kw = p.kwargs()
    with pytest.raises(ValueError, match="m does not match the sum"):
        solver.rpdhg_gpu_solve(**{**kw, "mGzero": kw["mGzero"] + 1, "m": kw["m"]})
    with pytest.raises(ValueError, match="greater than 1"):
        solver.rpdhg_gpu_solve(**{**kw, "socG": [1] + list(kw["socG"])[1:],
                                  "m": kw["m"] - kw["socG"][0] + 1,
                                  "G": kw["G"][:kw["m"] - kw["socG"][0] + 1], "h": kw["h"][:kw["m"] - kw["socG"][0] + 1]})
    bl = kw["bl"].copy()
    bl[0] = 100.0
    with pytest.raises(ValueError, match="less than or equal"):
        solver.rpdhg_gpu_solve(**{**kw, "bl": bl})
    with pytest.raises(ValueError, match="does not match the size of G"):
        solver.rpdhg_gpu_solve(**{**kw, "m": kw["m"] + 3, "mGzero": kw["mGzero"] + 3})


def test_build_staleness_check_covers_every_source():
    """Every file under csrc/ and include/ takes part in the library's
    staleness check, so editing any header triggers a rebuild."""
    listed = set(build.deps())
    for d in (os.path.join(ROOT, "pdcs_b200", "csrc"), os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h")):
                assert os.path.join(d, f) in listed, f


def test_portfolio_generator_is_feasible_by_construction():
    """The c2 generator's equal-weight portfolio, with t above its risk, lies
    in the interior of every cone of the program (small instance)."""
    n, f = 2000, 10
    p = problems.portfolio_c2(n=n, factors=f)
    x = np.concatenate([np.full(n, 1.0 / n), [0.0]])
    ng = n // 10
    rs = 1 + ng * 11
    r = p.G @ x - p.h
    x[-1] = 2.0 * float(np.sum(r[rs + 2:] ** 2)) + 1e-12
    r = p.G @ x - p.h
    assert abs(r[0]) < 1e-12                                   # budget
    blocks = r[1:rs].reshape(ng, 11)
    assert np.all(blocks[:, 0] > np.linalg.norm(blocks[:, 1:], axis=1))  # tracking SOC interior
    assert 2 * r[rs] * r[rs + 1] > np.sum(r[rs + 2:] ** 2)      # risk RSOC interior
    assert p.rsocG == [2 + f + n] and p.socG == [11] * ng and p.m == rs + 2 + f + n
