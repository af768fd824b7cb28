"""Generate tests/golden/ref_projections.npz from the reference's own cone
projection code (oracle/_ref: src/pdcs_gpu/cuda/massive_block_proj.cu and
exp_proj.cu of the reference, compiled as host code by `make -C oracle ref`).

Each case is one block: input v, scaling S (ones for the unscaled codes), the
reference kernel's output at its tightest projection tolerance (5e-16, the
floor of rpdhg_alg_gpu_gen_scaling.jl:722-723), the oracle's output, and a
60-digit projection from the KKT conditions (mp_cones.py) that decides
between the two where they differ.  The
reference runs in a worker process with a time limit per block; a block on
which it does not return (its search loops never meet their exit test) is
kept with `_hang` = 1 and NaN as the reference output.
Inputs are seeded random blocks plus adversarial ones: interior, polar and
boundary points, |t| near zero, x + y near zero (RSOC), huge and tiny
magnitudes, long blocks.  The fixture lets the CPU and GPU tests compare with
the reference without the reference tree present.
Run:  python tests/golden/make_ref_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import binding as B  # noqa: E402
from oracle import ref_binding as R  # noqa: E402

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import mp_cones  # noqa: E402


def soc_cases(rng, scaled):
    out = []
    for d in (2, 3, 4, 7, 11, 20, 33, 200, 1000):
        for k in range(24 if d < 200 else 4):
            v = rng.standard_normal(d) * rng.choice([1e-6, 1e-2, 1.0, 1e2, 1e6])
            S = np.exp(rng.uniform(-2, 2, d)) if scaled else np.ones(d)
            D = S[0] / S[1:]
            nx = np.linalg.norm(D * v[1:])
            if k % 6 == 1:
                v[0] = 3.0 * nx            # interior
            elif k % 6 == 2:
                v[0] = -3.0 * np.linalg.norm(v[1:] / D)  # polar
            elif k % 6 == 3:
                v[0] = nx                  # boundary
            elif k % 6 == 4:
                v[0] = 1e-13 * nx          # |t| near zero
            out.append((v, S))
    return out


def rsoc_cases(rng, scaled):
    out = []
    for d in (3, 4, 6, 11, 40, 300):
        for k in range(30 if d < 300 else 6):
            v = rng.standard_normal(d) * rng.choice([1e-4, 1.0, 1e3])
            S = np.exp(rng.uniform(-2, 2, d)) if scaled else np.ones(d)
            D = np.sqrt(S[0] * S[1]) / S[2:]
            q = np.sum((D * v[2:]) ** 2)
            if k % 7 == 1:
                v[1] = -v[0] * (1 + 1e-14)  # x + y near zero
            elif k % 7 == 2:
                v[0], v[1] = abs(v[0]), q / (2 * abs(v[0]))  # boundary
            elif k % 7 == 3:
                v[0], v[1] = 2 * abs(v[0]), q / abs(v[0])    # interior
            elif k % 7 == 4:
                v[0] = 0.0
            elif k % 7 == 5:
                v[0], v[1] = -abs(v[0]), -abs(v[1])          # both negative
            out.append((v, S))
    return out


def exp_cases(rng, scaled):
    out = []
    for k in range(270):
        v = rng.standard_normal(3) * rng.choice([1e-3, 0.1, 1.0, 10.0, 1e3])
        S = np.exp(rng.uniform(-2, 2, 3)) if scaled else np.ones(3)
        if k % 9 == 1:
            s = abs(v[1]) + 0.1
            v = np.array([v[0], s, s * np.exp(v[0] / s)]) * S  # boundary
        elif k % 9 == 2:
            v[0], v[1] = -abs(v[0]), -abs(v[1])  # r, s <= 0
        elif k % 9 == 3:
            v[1] = 1e-9 * abs(v[1])              # s near zero
        elif k % 9 == 4:
            v = -np.abs(v) * np.array([-1, 1, 1])  # polar-side points
        out.append((v, S))
    return out


def make(seed=20261204):
    rng = np.random.default_rng(seed)
    data = {}
    g = R.Guarded(timeout=2.0)
    for kind, gen in (("soc", soc_cases), ("rsoc", rsoc_cases), ("exp", exp_cases), ("dexp", exp_cases)):
        for scaled in (False, True):
            tag = f"{kind}_{'s' if scaled else 'u'}"
            vs, Ss, refs, orcs, truth, lens, hang = [], [], [], [], [], [], []
            for v, S in gen(rng, scaled):
                pr = g.project(kind, v, S if scaled else None)
                hang.append(pr is None)
                if pr is None:
                    pr = np.full(v.size, np.nan)
                po = B.project_block(kind, v, S if scaled else None)
                truth.append(mp_cones.PROJ[kind](v, S))
                vs.append(v); Ss.append(S); refs.append(pr); orcs.append(po); lens.append(v.size)
            print(tag, len(lens), "blocks,", sum(hang), "without return", flush=True)
            data[tag + "_hang"] = np.array(hang, dtype=np.int8)
            data[tag + "_v"] = np.concatenate(vs)
            data[tag + "_S"] = np.concatenate(Ss)
            data[tag + "_ref"] = np.concatenate(refs)
            data[tag + "_oracle"] = np.concatenate(orcs)
            data[tag + "_truth"] = np.concatenate(truth)
            data[tag + "_len"] = np.array(lens, dtype=np.int64)
            data[tag + "_code"] = np.array([R.CODE[(kind, scaled)]], dtype=np.int64)
    g.close()
    return data


if __name__ == "__main__":
    d = make()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_projections.npz")
    np.savez_compressed(path, **d)
    print("wrote", path, {k: v.shape for k, v in d.items() if k.endswith("_len")})
