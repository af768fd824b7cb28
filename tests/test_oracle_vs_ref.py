"""Pin the oracle's cone projections to the reference's own projection code.

tests/golden/ref_projections.npz (tests/golden/make_ref_golden.py) holds, for
seeded and adversarial blocks of every cone kind, plain and diagonally scaled:
the output of the reference kernel massive_block_proj
(src/pdcs_gpu/cuda/massive_block_proj.cu:1081, with exp_proj.cu) compiled as
host code (oracle/_ref), the oracle's output, and the projection solved from
its KKT conditions at 60-400 digits.  The oracle must equal the reference to
1e-12 wherever the reference's output is the projection, and the
high-precision projection everywhere (where the reference's search returns a
non-projection or does not return).  With the reference tree present, the
fixture is re-checked against a live build and fresh random blocks are
compared too.
"""
import os
import sys

import numpy as np
import pytest

from oracle import binding as B
from oracle import ref_binding as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_projections.npz")
TAGS = ["soc_u", "soc_s", "rsoc_u", "rsoc_s", "exp_u", "exp_s", "dexp_u", "dexp_s"]
TOL = 1e-12


def blocks(g, tag):
    lens = g[tag + "_len"]
    off = np.concatenate([[0], np.cumsum(lens)])
    for i in range(len(lens)):
        sl = slice(off[i], off[i + 1])
        v = g[tag + "_v"][sl]
        yield i, v, g[tag + "_S"][sl], g[tag + "_ref"][sl], g[tag + "_oracle"][sl], g[tag + "_truth"][sl], \
            max(1.0, float(np.abs(v).max()))


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_equals_high_precision_projection(golden, tag):
    kind, scaled = tag.split("_")[0], tag.endswith("_s")
    for i, v, S, _, po, pt, sc in blocks(golden, tag):
        p = B.project_block(kind, v, S if scaled else None)  # the oracle as built now
        assert np.abs(p - pt).max() <= TOL * sc, (tag, i, v, p, pt)
        assert np.abs(p - po).max() <= TOL * sc, (tag, i)


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_equals_reference_where_reference_is_exact(golden, tag):
    kind, scaled = tag.split("_")[0], tag.endswith("_s")
    exact = 0
    for i, v, S, pr, _, pt, sc in blocks(golden, tag):
        if golden[tag + "_hang"][i] or np.abs(pr - pt).max() > TOL * sc:
            continue
        exact += 1
        p = B.project_block(kind, v, S if scaled else None)
        assert np.abs(p - pr).max() <= 2 * TOL * sc, (tag, i, v, p, pr)
    # the reference is exact on most blocks of every kind (the rest are its
    # known failure branches: see the module docstring of make_ref_golden.py)
    assert exact >= 0.4 * len(golden[tag + "_len"]), (tag, exact)


def test_reference_failures_are_confined(golden):
    """Where the reference's output is not the projection, the oracle's is:
    a non-returning block (unscaled RSOC with x + y ~ 0), or an output off the
    high-precision projection by more than 1e-12 relative."""
    counts = {}
    for tag in TAGS:
        bad = 0
        for i, v, S, pr, po, pt, sc in blocks(golden, tag):
            if golden[tag + "_hang"][i] or np.abs(pr - pt).max() > TOL * sc:
                bad += 1
                assert np.abs(po - pt).max() <= TOL * sc
        counts[tag] = bad
    # plain SOC and the scaled exponential cone match the reference everywhere
    assert counts["soc_u"] == 0 and counts["exp_s"] == 0, counts
    print("reference blocks off the projection:", counts)


have_ref = pytest.mark.skipif(not os.path.isdir(R.REF_CUDA), reason="reference tree not present")


@have_ref
def test_fixture_is_the_reference_output(golden):
    with R.Guarded(timeout=2.0) as g:
        for tag in TAGS:
            kind, scaled = tag.split("_")[0], tag.endswith("_s")
            for i, v, S, pr, _, _, sc in blocks(golden, tag):
                if i % 9 or golden[tag + "_hang"][i]:
                    continue
                out = g.project(kind, v, S if scaled else None)
                assert out is not None
                assert np.abs(out - pr).max() <= 1e-15 * sc, (tag, i)


@have_ref
@pytest.mark.parametrize("kind", ["soc", "rsoc", "exp", "dexp"])
def test_oracle_vs_live_reference_random(kind):
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import mp_cones
    rng = np.random.default_rng({"soc": 1, "rsoc": 2, "exp": 3, "dexp": 4}[kind])
    agree = 0
    with R.Guarded(timeout=2.0) as g:
        for k in range(120):
            d = 3 if kind in ("exp", "dexp") else int(rng.integers(3, 16))
            v = rng.standard_normal(d) * rng.choice([1e-2, 1.0, 1e2])
            S = np.exp(rng.uniform(-2, 2, d)) if k % 2 else None
            po = B.project_block(kind, v, S)
            pr = g.project(kind, v, S)
            sc = max(1.0, float(np.abs(v).max()))
            if pr is not None and np.abs(po - pr).max() <= 2 * TOL * sc:
                agree += 1
                continue
            pt = mp_cones.PROJ[kind](v, np.ones(d) if S is None else S)
            assert np.abs(po - pt).max() <= TOL * sc, (kind, v, S, po, pt, pr)
    assert agree >= 40, agree
