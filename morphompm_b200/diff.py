"""[6] Diff / inverse -- recover a growth parameter from an observed shape with
the trajectory gradient; Gauss-Newton on g with the reference's step clamp and
zero/non-finite gradient nudge, unchanged (python/morphompm/diff.py:9-24).
It reaches the GPU through ``integrate.dloss_dg``.
"""
import numpy as np

from .integrate import dloss_dg, rollout, iso_growth_state, loss_detF  # noqa: F401


def infer_growth(pts, model, cfg, target, n_steps, g_init, advect=False, iters=20,
                 tol=1e-9, return_history=False, **loss_kw):
    g = g_init
    hist = [g_init]
    for it in range(iters):
        loss, dg = dloss_dg(pts, model, cfg, g, n_steps, advect, **loss_kw)
        resid = loss - target
        if abs(resid) < tol:
            break
        if abs(dg) < 1e-12 or not np.isfinite(dg):    # guard: dg crosses 0
            g += 1e-3 * (1.0 if resid < 0 else -1.0)   # nudge off the stationary point
            continue
        step = resid / dg
        g -= max(-0.5, min(0.5, step))                 # damp: cap |dg| for robustness
        hist.append(g)
    return (g, it + 1, hist) if return_history else (g, it + 1)
