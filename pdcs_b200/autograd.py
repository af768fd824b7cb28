"""Differentiable batched conic layer: torch.autograd.Function over the
batched solver and its solution-map adjoint.

    layer = ConicBatchLayer(problems)                 # structure: sparsity, cones, sizes
    x = layer(c, h, Gval, bl, bu)                      # flat tensors (concatenated over instances)
    loss(x).backward()                                 # gradients of c, h, Gval, bl, bu

Inputs and the output are FP64 tensors concatenated over the instances in
order: c (sum n), h (sum m), Gval (sum nnz, each instance's CSR order with
sorted indices), bl / bu (sum nb); x (sum n) is the primal solution.  The
forward pass solves the batch (pdcs_batch_create + pdcs_batch_solve with
differentiable = 1), the backward pass runs pdcs_batch_grad at that solution.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.sparse as sp
import torch

from . import solver


@dataclasses.dataclass
class _Structure:
    kwargs: list      # per instance: the problem keywords without the data vectors
    pattern: list     # per instance: (indptr, indices) of G with sorted indices
    n: list
    m: list
    nnz: list
    nb: list


def _structure(problems):
    kws, pats = [], []
    for p in problems:
        kw = p.kwargs() if hasattr(p, "kwargs") else dict(p)
        G = sp.csr_matrix(kw["G"])
        G.sort_indices()
        pats.append((G.indptr.copy(), G.indices.copy(), G.shape))
        kws.append({k: v for k, v in kw.items() if k not in ("c", "h", "G", "bl", "bu")})
    return _Structure(kws, pats, [k["n"] for k in kws], [k["m"] for k in kws],
                      [len(p[1]) for p in pats], [k["nb"] for k in kws])


def _split(t, sizes):
    a = t.detach().cpu().numpy().astype(np.float64, copy=False)
    out, o = [], 0
    for s in sizes:
        out.append(a[o:o + s])
        o += s
    return out


class _ConicBatchFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, st, options, c, h, gval, bl, bu):
        cs, hs, gs = _split(c, st.n), _split(h, st.m), _split(gval, st.nnz)
        bls, bus = _split(bl, st.nb), _split(bu, st.nb)
        probs = []
        for i, kw in enumerate(st.kwargs):
            ip, ix, shape = st.pattern[i]
            probs.append(dict(kw, c=cs[i], h=hs[i], G=sp.csr_matrix((gs[i], ix, ip), shape=shape),
                              bl=bls[i], bu=bus[i]))
        handle = solver.BatchHandle(probs, differentiable=True, **options)
        sols, info = handle.solve()
        bad = [i for i, s in enumerate(sols) if s.info.exit_status != "optimal"]
        if bad:
            handle.close()
            raise RuntimeError(f"instances {bad[:8]} not solved to optimality")
        ctx.handle, ctx.st = handle, st
        x = np.concatenate([s.primal for s in sols])
        return torch.as_tensor(x, dtype=torch.float64, device=c.device)

    @staticmethod
    def backward(ctx, gx):
        st, handle = ctx.st, ctx.handle
        grads, _ = handle.grad(_split(gx, st.n))
        handle.close()
        dev = gx.device
        cat = lambda key: torch.as_tensor(np.concatenate([g[key] for g in grads]), dtype=torch.float64, device=dev)
        return None, None, cat("c"), cat("h"), cat("G"), cat("bl"), cat("bu")


class ConicBatchLayer(torch.nn.Module):
    """x*(c, h, Gval, bl, bu) for a fixed batch structure (sparsity patterns, cones, sizes)."""

    def __init__(self, problems, **options):
        super().__init__()
        self.st = _structure(problems)
        self.options = options

    def forward(self, c, h, gval, bl, bu):
        return _ConicBatchFn.apply(self.st, self.options, c, h, gval, bl, bu)

    def flat_params(self, problems):
        """The data of `problems` as the flat FP64 tensors the layer takes."""
        cat = lambda key: torch.as_tensor(np.concatenate([np.asarray(getattr(p, key), dtype=np.float64)
                                                          for p in problems]), dtype=torch.float64)
        gv = []
        for p in problems:
            G = sp.csr_matrix(p.G)
            G.sort_indices()
            gv.append(G.data)
        return cat("c"), cat("h"), torch.as_tensor(np.concatenate(gv)), cat("bl"), cat("bu")
