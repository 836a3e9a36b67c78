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


# ---------------------------------------------------------------------------
# Batched inverse problems (extensions: the reference solves one scalar g for
# one scene).  Both drive a ``batch.Batch``: every iteration sets the
# per-scene parameters (mpm_plan_update_scenes) and replays the captured
# forward + adjoint graph of the whole batch.
# ---------------------------------------------------------------------------
def infer_growth_batched(batch, targets, g_init, iters=20, tol=1e-9):
    """The Gauss-Newton iteration of ``infer_growth`` (same step clamp and
    stationary-point nudge), run for every scene of the batch at once: scene
    s solves loss_s(g_s) = targets[s] with the growth law g_s = 1 + A_s.
    Returns (g, iterations per scene)."""
    S = len(batch.scenes)
    g = np.full(S, float(g_init)) if np.isscalar(g_init) else np.array(g_init, dtype=np.float64)
    targets = np.asarray(targets, dtype=np.float64)
    done = np.zeros(S, dtype=bool)
    its = np.zeros(S, dtype=np.int64)
    for _ in range(iters):
        batch.set_params(growth_A=g - 1.0)
        batch.replay()
        loss = batch.loss.cpu().numpy()
        dg = batch.dloss_dg.cpu().numpy()
        resid = loss - targets
        done |= np.abs(resid) < tol
        if done.all():
            break
        act = ~done
        its[act] += 1
        stat = act & ((np.abs(dg) < 1e-12) | ~np.isfinite(dg))
        g[stat] += 1e-3 * np.where(resid[stat] < 0, 1.0, -1.0)
        step = act & ~stat
        g[step] -= np.clip(resid[step] / dg[step], -0.5, 0.5)
    return g, its


def fit_batched(batch, params=("g", "E"), iters=50, lr=0.02, g0=None, E0=None, nu0=None):
    """Minimise every scene's loss over its own growth factor g, Young's
    modulus E and/or Poisson ratio nu with Adam (E in log space), using the
    batched trajectory gradients (d/dA for g, mpm_step_bwd_params for E and
    nu).  The batch must be built with material_grads=True when E or nu is
    fitted.  Returns a dict of the final per-scene values and the loss history
    (iters + 1, S)."""
    S = len(batch.scenes)
    g = np.array(g0 if g0 is not None else [1.0 + sc["growth_A"] for sc in batch.scenes], dtype=np.float64)
    E = np.array(E0 if E0 is not None else [sc["E"] for sc in batch.scenes], dtype=np.float64)
    nu = np.array(nu0 if nu0 is not None else [sc["nu"] for sc in batch.scenes], dtype=np.float64)
    names = list(params)
    m = np.zeros((len(names), S))
    v = np.zeros((len(names), S))
    b1, b2, eps = 0.9, 0.999, 1e-12
    hist = []

    def evaluate():
        batch.set_params(growth_A=g - 1.0, E=E, nu=nu)
        batch.replay()
        hist.append(batch.loss.cpu().numpy().copy())
        grads = {"g": batch.dloss_dg.cpu().numpy().copy()}
        if "E" in names or "nu" in names:
            dEn = batch.dloss_dE_nu()
            grads["E"], grads["nu"] = dEn[:, 0] * E, dEn[:, 1]   # d/dlog E, d/dnu
        return grads

    for it in range(1, iters + 1):
        grads = evaluate()
        for k, name in enumerate(names):
            gr = grads[name]
            m[k] = b1 * m[k] + (1 - b1) * gr
            v[k] = b2 * v[k] + (1 - b2) * gr * gr
            upd = lr * (m[k] / (1 - b1 ** it)) / (np.sqrt(v[k] / (1 - b2 ** it)) + eps)
            if name == "g":
                g -= upd
            elif name == "E":
                E *= np.exp(-upd)
            else:
                nu = np.clip(nu - upd, 0.0, 0.49)
    evaluate()
    return {"g": g, "E": E, "nu": nu, "loss": np.array(hist)}
