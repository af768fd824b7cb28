"""Generate the golden projection fixtures from the CPU oracle.

The oracle itself is pinned by invariants (tests/test_oracle_projections.py);
these fixtures freeze its outputs for seeded inputs so that the CUDA
projections can be checked element by element without rebuilding anything.
Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import binding as B  # noqa: E402


def make(seed=20261203):
    rng = np.random.default_rng(seed)
    out = {}
    for kind, dims in (("soc", (2, 3, 5, 11, 33, 70)), ("rsoc", (3, 4, 7, 20, 40))):
        vs, Ss, ps, lens = [], [], [], []
        for d in dims:
            for k in range(40):
                v = rng.standard_normal(d) * rng.choice([1e-3, 1.0, 1e3])
                if k % 5 == 0:
                    v[0] = abs(v[0]) * 10  # interior
                if k % 7 == 0:
                    v[0] = -abs(v[0]) * 10  # polar
                S = np.exp(rng.uniform(-2, 2, d)) if k % 2 else np.ones(d)
                p = B.project_block(kind, v, S)
                vs.append(v); Ss.append(S); ps.append(p); lens.append(d)
        out[kind + "_v"] = np.concatenate(vs)
        out[kind + "_S"] = np.concatenate(Ss)
        out[kind + "_p"] = np.concatenate(ps)
        out[kind + "_len"] = np.array(lens, dtype=np.int64)
    for kind in ("exp", "dexp"):
        v = rng.standard_normal((400, 3)) * rng.choice([0.1, 1.0, 10.0], size=(400, 1))
        S = np.where(np.arange(400)[:, None] % 2 == 0, 1.0, np.exp(rng.uniform(-2, 2, (400, 3))))
        p = np.stack([B.project_block(kind, v[i], S[i]) for i in range(400)])
        out[kind + "_v"], out[kind + "_S"], out[kind + "_p"] = v.ravel(), S.ravel(), p.ravel()
    return out


if __name__ == "__main__":
    data = make()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "projections.npz")
    np.savez_compressed(path, **data)
    print("wrote", path, {k: v.shape for k, v in data.items()})
