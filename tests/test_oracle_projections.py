"""Pin the oracle's cone projections with invariants and brute force (CPU)."""
import numpy as np
import pytest

from oracle import binding as B
import _proj_reference as R

GOLDEN = "tests/golden/projections.npz"


def _soc_checks(v, p, D):
    """p in {||D y|| <= s}, v - p in its polar, <p, v - p> = 0."""
    scale = max(1.0, np.abs(v).max())
    assert np.linalg.norm(D * p[1:]) <= p[0] + 1e-12 * scale
    r = v - p
    assert np.linalg.norm(r[1:] / D) <= -r[0] + 1e-9 * scale
    assert abs(r @ p) <= 1e-9 * scale ** 2


@pytest.mark.parametrize("seed", range(4))
def test_scaled_soc_invariants(seed):
    rng = np.random.default_rng(seed)
    for _ in range(300):
        d = int(rng.integers(2, 40))
        v = rng.standard_normal(d) * rng.choice([1e-3, 1.0, 1e3])
        S = np.exp(rng.uniform(-3, 3, d))
        p = B.project_block("soc", v, S)
        _soc_checks(v, p, S[0] / S[1:])
        q = B.project_block("soc", p, S)  # idempotence
        assert np.abs(q - p).max() <= 1e-13 * max(1.0, np.abs(v).max())


def test_scaled_soc_matches_bisection():
    rng = np.random.default_rng(11)
    for _ in range(200):
        d = int(rng.integers(2, 12))
        v = rng.standard_normal(d)
        S = np.exp(rng.uniform(-2, 2, d))
        p = B.project_block("soc", v, S)
        ref = R.soc_project_reference(v, S[0] / S[1:])
        assert np.allclose(p, ref, atol=1e-11, rtol=1e-10)


def test_plain_soc_closed_form():
    rng = np.random.default_rng(5)
    for _ in range(200):
        d = int(rng.integers(2, 10))
        v = rng.standard_normal(d)
        p = B.project_block("soc", v)
        t, x = v[0], v[1:]
        nx = np.linalg.norm(x)
        if nx <= t:
            ref = v
        elif nx <= -t:
            ref = np.zeros(d)
        else:
            c = (1 + t / nx) / 2
            ref = np.concatenate([[c * nx], c * x])
        assert np.allclose(p, ref, atol=1e-14)


@pytest.mark.parametrize("seed", range(3))
def test_scaled_rsoc_invariants(seed):
    rng = np.random.default_rng(100 + seed)
    for _ in range(300):
        d = int(rng.integers(3, 30))
        v = rng.standard_normal(d) * rng.choice([1e-2, 1.0, 1e2])
        S = np.exp(rng.uniform(-2, 2, d))
        p = B.project_block("rsoc", v, S)
        Dz = np.sqrt(S[0] * S[1]) / S[2:]
        scale = max(1.0, np.abs(v).max())
        assert p[0] >= -1e-12 * scale and p[1] >= -1e-12 * scale
        assert 2 * p[0] * p[1] >= np.sum((Dz * p[2:]) ** 2) - 1e-9 * scale ** 2
        r = v - p
        a, b = -r[0], -r[1]  # polar: -(dual), dual = {2ab >= ||z/D||^2}
        assert a >= -1e-9 * scale and b >= -1e-9 * scale
        assert 2 * a * b >= np.sum((r[2:] / Dz) ** 2) - 1e-8 * scale ** 2
        assert abs(r @ p) <= 1e-9 * scale ** 2


@pytest.mark.parametrize("scaled", [False, True])
def test_exp_projection_is_global_minimiser(scaled):
    rng = np.random.default_rng(7 if scaled else 8)
    for k in range(60):
        v = rng.standard_normal(3) * rng.choice([0.1, 1.0, 10.0])
        S = np.exp(rng.uniform(-2, 2, 3)) if scaled else np.ones(3)
        p = B.project_block("exp", v, S)
        ok, why = R.check_exp_projection(v, p, S)
        assert ok, (v, S, p, why)


def test_exp_adversarial_cases():
    # roots against a breakpoint, huge |rho|, boundary and polar points
    cases = [
        ([0.05665114, -0.68269979, 0.61457337], [0.21678823, 0.5271339, 5.98022836]),
        ([-2.25655078e+00, 3.82927311e-03, -4.02616473e+00], [0.19308704, 6.76961535, 2.37556143]),
        ([-1.03086414, 0.03952289, -1.3610594], [0.2296303, 0.63566874, 0.52559705]),
        ([1.04310897, -1.02295067, 0.67607805], [0.14794924, 2.95140527, 4.63407111]),
        ([0.0, 1.0, np.e], [1, 1, 1]),            # on the boundary
        ([-1.0, -1.0, -1.0], [1, 1, 1]),          # r, s <= 0
        ([1e-300, 1e-300, 1.0], [1, 1, 1]),
        ([5.0, 1e-8, 1.0], [1, 1, 1]),
    ]
    for v, S in cases:
        v, S = np.array(v, float), np.array(S, float)
        p = B.project_block("exp", v, S)
        ok, why = R.check_exp_projection(v, p, S)
        assert ok, (v, S, p, why)


def test_dual_exp_moreau():
    """P_{S o K*}(v) + P_{(S o K*)polar}(v) = v, (S o K*)polar = -(1/S) o K."""
    rng = np.random.default_rng(3)
    for _ in range(300):
        v = rng.standard_normal(3)
        S = np.exp(rng.uniform(-2, 2, 3))
        p = B.project_block("dexp", v, S)
        q = -B.project_block("exp", -v, 1.0 / S)
        assert np.allclose(p + q, v, atol=1e-13)
        assert abs(p @ q) <= 1e-9


def test_golden_fixtures_reproduce():
    g = np.load(GOLDEN)
    for kind in ("soc", "rsoc"):
        off = 0
        for d in g[kind + "_len"]:
            sl = slice(off, off + d)
            p = B.project_block(kind, g[kind + "_v"][sl], g[kind + "_S"][sl])
            assert np.allclose(p, g[kind + "_p"][sl], atol=1e-12 * max(1, np.abs(g[kind + "_v"][sl]).max()))
            off += d
    for kind in ("exp", "dexp"):
        v = g[kind + "_v"].reshape(-1, 3)
        S = g[kind + "_S"].reshape(-1, 3)
        P = g[kind + "_p"].reshape(-1, 3)
        for i in range(len(v)):
            p = B.project_block(kind, v[i], S[i])
            assert np.allclose(p, P[i], atol=1e-12 * max(1, np.abs(v[i]).max()))
