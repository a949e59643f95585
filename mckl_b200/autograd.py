"""torch.autograd binding of the batched particle filters' adjoint.

``PFLogLikelihood.apply(phi, sx, sy, filters)`` returns the FP64
log-likelihood estimates of the filters (one per filter) as a tensor whose
backward pass multiplies the incoming gradient by the adjoint kernel's
gradient with respect to (phi, sx, sy) -- ancestors and resampling times held
fixed, noise replayed from the counters.  The parameters given are written
into the filters before the run, so the function is a plain map
(phi, sx, sy) -> logL for autograd and finite-difference checks.
"""
from __future__ import annotations

import numpy as np
import torch

from . import BatchedFilters, _check, _bt_shadow_params  # noqa: F401


class PFLogLikelihood(torch.autograd.Function):
    @staticmethod
    def forward(ctx, phi, sx, sy, template: dict, checkpoint_every: int = 32):
        w = dict(template)
        w["phi"] = phi.detach().cpu().double().numpy()
        w["sx"] = sx.detach().cpu().double().numpy()
        w["sy"] = sy.detach().cpu().double().numpy()
        b = BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"],
                           threshold=w.get("threshold", 0.5), fp64=True)
        try:
            # the adjoint kernel is fastest with 1024 threads per filter (twice
            # the resident warps of 512, whatever it spills) unless told otherwise
            b.config(int(w.get("threads", 1024)), int(w.get("ctas_per_sm", 1)))
            ll, g = b.adjoint(checkpoint_every)
        finally:
            b.close()
        grad = torch.from_numpy(g).to(phi.device)
        ctx.save_for_backward(grad)
        return torch.from_numpy(ll).to(phi.device)

    @staticmethod
    def backward(ctx, gout):
        (grad,) = ctx.saved_tensors
        gout = gout.to(grad.dtype)
        return gout * grad[:, 0], gout * grad[:, 1], gout * grad[:, 2], None, None


def loglik(phi, sx, sy, workload: dict, checkpoint_every: int = 32):
    """Differentiable FP64 log-likelihood estimates of the workload's filters."""
    return PFLogLikelihood.apply(phi, sx, sy, workload, checkpoint_every)


def finite_differences(workload: dict, h: float = 1e-5, threads: int | None = None):
    """Central differences of each filter's estimate in (phi, sx, sy) under
    common random numbers with the base run's resampling decisions and
    ancestors: two FP64 runs per parameter whose shadows sit at theta +- h."""
    w = workload
    F = len(w["N"])
    out = np.zeros((F, 3))
    for k, name in enumerate(("phi", "sx", "sy")):
        vals = []
        for sgn in (1.0, -1.0):
            b = BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"],
                               threshold=w.get("threshold", 0.5), fp64=True, shadow=True)
            try:
                if threads is not None:
                    b.config(int(threads), 1)
                p = {n: np.array(w[n], dtype=np.float64, copy=True) for n in ("phi", "sx", "sy")}
                p[name] = p[name] + sgn * h
                b.set_shadow_params(p["phi"], p["sx"], p["sy"])
                b.run()
                vals.append(b.shadow_loglik())
            finally:
                b.close()
        out[:, k] = (vals[0] - vals[1]) / (2 * h)
    return out
