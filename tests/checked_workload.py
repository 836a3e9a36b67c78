"""Workload run by tests/test_gpu_checked.py under both libraries: the release
build (in the test process) and the bounds-checked build (a child process
with MORPHOMPM_CHECKED=1).  Batches in FP32 and FP64 with an empty and a
one-particle scene, a growth field and checkpoint recompute, and one single
step with its VJP on particles at cell boundaries and grid faces.

    python tests/checked_workload.py OUT.npz     (child: also writes the violation count)
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def run() -> dict:
    import torch
    from morphompm_b200 import scenes, transfer
    from morphompm_b200.batch import Batch, host_slab
    from morphompm_b200.config import Material, SimConfig
    from morphompm_b200.constitutive import Hencky
    from morphompm_b200.state import ParticleState
    out = {}
    sc = scenes.config4(seed=13, n_scenes=4, n_lo=300, n_hi=2500)
    sc[0]["model"], sc[1]["model"] = "nh", "hencky"
    sc[2] = dict(sc[2], model="hb", hb=dict(kappa=1e4, K=1.0, n=0.5, tau_y=10.0, m=100.0, eps=1e-4),
                 phi=np.linspace(0.0, 1.0, sc[2]["x"].shape[0]))
    batch = [sc[0], dict(sc[1], x=sc[1]["x"][:0]), dict(sc[3], x=sc[3]["x"][:1]), sc[1], sc[2], sc[3]]
    for dt, npd in ((torch.float32, np.float32), (torch.float64, np.float64)):
        b = Batch(batch, 7, dtype=dt, ckpt_every=3)
        b.load(host_slab(batch, npd), non_blocking=False)
        b.run()
        tag = str(dt).split(".")[-1]
        out[f"{tag}_loss"] = b.loss.cpu().numpy()
        out[f"{tag}_dg"] = b.dloss_dg.cpu().numpy()
        out[f"{tag}_final"] = b.final_state().cpu().numpy()
        out[f"{tag}_bar0"] = b.initial_cotangents().cpu().numpy()
        out[f"{tag}_status"] = np.array([b.plan.status()])
    rng = np.random.default_rng(5)
    N, dx = 16, 1.0 / 16
    x = np.concatenate([(rng.integers(2, 13, size=(30, 3)) + 0.5) * dx, rng.uniform(0.0, 1.0, size=(60, 3))])
    n = x.shape[0]
    st = ParticleState(x, 0.1 * rng.standard_normal((n, 3)), 0.3 * rng.standard_normal((n, 3, 3)),
                       np.eye(3) + 0.02 * rng.standard_normal((n, 3, 3)),
                       1.1 * np.eye(3) + 0.01 * rng.standard_normal((n, 3, 3)))
    cfg = SimConfig(N=N, dx=dx, dt=5e-4, sp=dx / 2, material=Material(E=1e4, nu=0.3))
    ns, cache = transfer.step(st, Hencky(cfg.material), cfg, advect=True)
    bars = [rng.standard_normal(s) for s in ((n, 3), (n, 3), (n, 3, 3), (n, 3, 3), (n, 3, 3))]
    g = transfer.step_vjp(cache, *bars, advect=True)
    out["step_F"] = ns.F
    out["step_x"] = ns.x
    for i, a in enumerate(g):
        out[f"step_g{i}"] = a
    torch.cuda.synchronize()
    return out


def violations():
    import ctypes as C
    import torch
    from morphompm_b200 import _lib as L
    lib = L.load()
    cnt, site, idx = C.c_int64(0), C.c_int32(0), C.c_int64(0)
    rc = lib.mpm_check_violations(C.byref(cnt), C.byref(site), C.byref(idx),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, cnt.value, site.value, idx.value


if __name__ == "__main__":
    res = run()
    rc, cnt, site, idx = violations()
    res["violations"] = np.array([rc, cnt, site, idx])
    np.savez(sys.argv[1], **res)
