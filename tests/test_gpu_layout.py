"""Cell-order layout on the device: a batch, dloss_dg and rollout_loss give
the same results for particles in any input order as for the same particles
in cell order, and every accessor returns the caller's order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _scenes(shuffle):
    from morphompm_b200 import scenes
    sc = scenes.config4(seed=9, n_scenes=4, n_lo=400, n_hi=2500)
    sc[0]["model"], sc[1]["model"] = "nh", "hencky"
    sc[2]["phi"] = np.linspace(0.0, 1.0, sc[2]["x"].shape[0])
    if shuffle:
        rng = np.random.default_rng(3)
        out = []
        for s in sc:
            q = rng.permutation(s["x"].shape[0])
            d = dict(s, x=s["x"][q])
            if s.get("phi") is not None:
                d["phi"] = s["phi"][q]
            out.append(d)
        return out
    return sc


def _within_scene_moved(b, scn):
    """Whether the batch's slot order moves particles inside any scene (the
    scene permutation of the model grouping aside)."""
    if b.order is None:
        return False
    off = np.concatenate([[0], np.cumsum([s["x"].shape[0] for s in scn])])
    q = 0
    moved = False
    for u in b.scene_perm:
        k = scn[u]["x"].shape[0]
        moved |= bool(np.any(b.order[q:q + k] != off[u] + np.arange(k)))
        q += k
    return moved


def test_batch_any_order_matches_cell_order():
    from morphompm_b200.batch import Batch, host_slab
    sc = _scenes(False)
    shuf = _scenes(True)
    res = {}
    for tag, scn, reorder in (("sorted", sc, True), ("shuf", shuf, True), ("shuf_raw", shuf, False)):
        b = Batch(scn, 6, dtype=torch.float64, ckpt_every=4, reorder=reorder)
        assert _within_scene_moved(b, scn) == (tag == "shuf")
        b.load(host_slab(scn, np.float64), non_blocking=False)
        b.run()
        torch.cuda.synchronize()
        res[tag] = (b.loss.clone(), b.dloss_dg.clone(), b.final_state().clone(), b.initial_cotangents().clone())
    rel = lambda a, b: float((a - b).abs().max() / b.abs().max())
    # same particles, two layouts: equal to rounding (node sums add in another order)
    for i, tol in ((0, 1e-12), (1, 1e-10)):
        assert rel(res["shuf"][i], res["shuf_raw"][i]) < tol
        assert rel(res["shuf"][i], res["sorted"][i]) < tol
    # per-particle outputs come back in the caller's order
    assert rel(res["shuf"][2], res["shuf_raw"][2]) < 1e-12
    assert rel(res["shuf"][3], res["shuf_raw"][3]) < 1e-9


def test_dloss_dg_and_rollout_loss_any_order():
    from morphompm_b200 import autograd, integrate
    from morphompm_b200.config import Material, SimConfig
    from morphompm_b200.constitutive import NeoHookean
    rng = np.random.default_rng(4)
    pts = rng.uniform(0.35, 0.6, size=(300, 3))            # random order
    cfg = SimConfig(N=12, dx=1 / 12, dt=4e-4, sp=1 / 24, wall=2)
    model = NeoHookean(Material(E=1e4, nu=0.3))
    from morphompm_b200.layout import cell_order_host
    o = cell_order_host(pts, cfg.dx, cfg.grid_shape)
    x_obs = pts + 0.01
    for loss in ("detF", "mse"):
        a = integrate.dloss_dg(pts, model, cfg, 1.15, 5, True, loss=loss, x_obs=x_obs)
        b = integrate.dloss_dg(pts[o], model, cfg, 1.15, 5, True, loss=loss, x_obs=x_obs[o])
        assert abs(a[0] - b[0]) < 1e-12 * abs(b[0]) and abs(a[1] - b[1]) < 1e-10 * abs(b[1])
        dev = dict(dtype=torch.float64, device="cuda")
        x0 = torch.as_tensor(pts, **dev).requires_grad_(True)
        L = autograd.rollout_loss(x0, 1.15, model, cfg, 5, True, loss=loss, x_obs=torch.as_tensor(x_obs, **dev))
        L.backward()
        x1 = torch.as_tensor(pts[o], **dev).requires_grad_(True)
        L1 = autograd.rollout_loss(x1, 1.15, model, cfg, 5, True, loss=loss,
                                   x_obs=torch.as_tensor(x_obs[o], **dev))
        L1.backward()
        g0 = x0.grad.cpu().numpy()
        g1 = x1.grad.cpu().numpy()
        assert np.max(np.abs(g0[o] - g1)) < 1e-9 * np.max(np.abs(g1))
