"""[8] I/O at the device boundary: particle states and configs to and from the
reference's formats (python/morphompm/io.py:1-117), same file layouts.

    .npz   lossless (x, v, C, F, Fg)                         load + save
    .csv   header x,y,z,vx,vy,vz,C00..C22,F00..F22,Fg00..Fg22,
           9 significant digits                              load + save
    .json  config (N, dx, dt, damping, sp, material)         load + save
    .vtk   legacy ASCII POLYDATA: points, det F, det Fg      save

States may hold numpy arrays or device tensors: each field crosses to the
host once, whole, and the text formats are written vectorised, so a
2M-particle state saves in seconds rather than through a per-particle loop.
``save_batch`` writes every scene of a batch from its (24, n) slab.
Loaded states are numpy arrays, as the reference returns them; ``to_device``
(``devarray``) moves them to the GPU.
"""
from __future__ import annotations

import csv
import json
import os

import numpy as np

from .config import Material, SimConfig
from .state import ParticleState

_CCOLS = [f"C{i}{j}" for i in range(3) for j in range(3)]
_FCOLS = [f"F{i}{j}" for i in range(3) for j in range(3)]
_GCOLS = [f"Fg{i}{j}" for i in range(3) for j in range(3)]
_CSV_HEADER = ["x", "y", "z", "vx", "vy", "vz"] + _CCOLS + _FCOLS + _GCOLS


def _host(a) -> np.ndarray:
    """One whole-array copy to the host (numpy passes through)."""
    if isinstance(a, np.ndarray):
        return a
    try:
        import torch
        if isinstance(a, torch.Tensor):
            return a.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    return np.asarray(a)


def host_state(state) -> ParticleState:
    """The state with every field as a host numpy array (io.py's canonical form)."""
    return ParticleState(*(_host(getattr(state, k)) for k in ("x", "v", "C", "F", "Fg")))


# -- ParticleState <-> file (dispatch on extension; io.py:29-49) -------------------
def save_state(state, path):
    ext = os.path.splitext(path)[1].lower()
    if ext not in (".npz", ".csv", ".vtk"):
        raise ValueError(f"unsupported save format '{ext}' (use .npz/.csv/.vtk)")
    st = host_state(state)
    if ext == ".npz":
        np.savez(path, x=st.x, v=st.v, C=st.C, F=st.F, Fg=st.Fg)
    elif ext == ".csv":
        _save_csv(st, path)
    else:
        _save_vtk(st, path)


def load_state(path) -> ParticleState:
    ext = os.path.splitext(path)[1].lower()
    if ext == ".npz":
        d = np.load(path)
        return ParticleState(d["x"], d["v"], d["C"], d["F"], d["Fg"])
    if ext == ".csv":
        return _load_csv(path)
    raise ValueError(f"unsupported load format '{ext}' (use .npz/.csv)")


def _rows(st) -> np.ndarray:
    n = st.n
    return np.concatenate([st.x.reshape(n, 3), st.v.reshape(n, 3), st.C.reshape(n, 9), st.F.reshape(n, 9),
                           st.Fg.reshape(n, 9)], axis=1).astype(np.float64)


def _save_csv(st, path):
    # io.py:52-58: one row per particle, every value formatted '%.9g'
    with open(path, "w", newline="") as f:
        f.write(",".join(_CSV_HEADER) + "\r\n")
        if st.n:
            np.savetxt(f, _rows(st), fmt="%.9g", delimiter=",", newline="\r\n")


def _load_csv(path) -> ParticleState:
    with open(path) as f:
        header = next(csv.reader(f))
    col = {c: i for i, c in enumerate(header)}
    data = np.loadtxt(path, delimiter=",", skiprows=1, ndmin=2)
    n = data.shape[0]
    take = lambda cols: data[:, [col[c] for c in cols]]
    return ParticleState(take(("x", "y", "z")), take(("vx", "vy", "vz")), take(_CCOLS).reshape(n, 3, 3),
                         take(_FCOLS).reshape(n, 3, 3), take(_GCOLS).reshape(n, 3, 3))


def _save_vtk(st, path):
    """Legacy-ASCII VTK POLYDATA with det F and det Fg point scalars (io.py:76-94)."""
    n = st.n
    detF = np.linalg.det(st.F.astype(np.float64)) if n else np.zeros(0)
    detFg = np.linalg.det(st.Fg.astype(np.float64)) if n else np.zeros(0)
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\nmorphompm particles\nASCII\n")
        f.write("DATASET POLYDATA\n")
        f.write(f"POINTS {n} float\n")
        if n:
            np.savetxt(f, st.x.astype(np.float64), fmt="%.6g", delimiter=" ")
        f.write(f"VERTICES {n} {2 * n}\n")
        if n:
            np.savetxt(f, np.stack([np.ones(n, np.int64), np.arange(n)], 1), fmt="%d", delimiter=" ")
        f.write(f"POINT_DATA {n}\n")
        for name, arr in (("detF", detF), ("detFg", detFg)):
            f.write(f"SCALARS {name} float 1\nLOOKUP_TABLE default\n")
            if n:
                np.savetxt(f, arr, fmt="%.6g")


# -- batches ------------------------------------------------------------------
def save_batch(batch, path_pattern, slab=None):
    """Write each scene of a ``batch.Batch`` to path_pattern.format(s=index),
    from a (24, n) slab in the scenes' particle order (default: the final
    state of the last trajectory).
    The growth tensor is the scene's growth law at the end of the trajectory,
    g I with g = 1 + A ramp(n_steps - 1) phi."""
    from .runtime import ROW_C, ROW_F, ROW_V, ROW_X
    from .batch import host_phi
    s_all = _host(batch.final_state() if slab is None else slab).astype(np.float64)
    phi = host_phi(batch.scenes, np.float64)
    paths = []
    for s, (p0, p1) in enumerate(zip(batch.plan.offsets[:-1], batch.plan.offsets[1:])):
        sc = batch.scenes[s]
        k = p1 - p0
        ramp = 1.0 if sc.get("ramp_steps", 0) <= 0 else min(1.0, batch.n_steps / sc["ramp_steps"])
        g = 1.0 + sc.get("growth_A", 0.0) * ramp * (phi[p0:p1] if phi is not None else np.ones(k))
        st = ParticleState(s_all[ROW_X:ROW_X + 3, p0:p1].T, s_all[ROW_V:ROW_V + 3, p0:p1].T,
                           s_all[ROW_C:ROW_C + 9, p0:p1].T.reshape(k, 3, 3),
                           s_all[ROW_F:ROW_F + 9, p0:p1].T.reshape(k, 3, 3),
                           g[:, None, None] * np.eye(3)[None])
        path = path_pattern.format(s=s)
        save_state(st, path)
        paths.append(path)
    return paths


# -- SimConfig <-> json (io.py:98-111) ------------------------------------------
def save_config(cfg, path):
    with open(path, "w") as f:
        json.dump({"N": cfg.N, "dx": cfg.dx, "dt": cfg.dt, "damping": cfg.damping,
                   "sp": cfg.sp, "material": {"E": cfg.material.E, "nu": cfg.material.nu,
                                              "density": cfg.material.density}}, f, indent=2)


def load_config(path):
    with open(path) as f:
        d = json.load(f)
    m = d.get("material", {})
    return SimConfig(N=d["N"], dx=d["dx"], dt=d["dt"], damping=d["damping"], sp=d["sp"],
                     material=Material(E=m.get("E", 1e4), nu=m.get("nu", 0.3), density=m.get("density", 1000.0)))


# -- measured curves (io.py:114-125) -------------------------------------------
def load_curve(path, xcol=0, ycol=1):
    """Two-column numeric CSV (digitised rheometry, measured wavelength);
    header and malformed rows are skipped."""
    rows = []
    with open(path) as f:
        for r in csv.reader(f):
            try:
                rows.append((float(r[xcol]), float(r[ycol])))
            except (ValueError, IndexError):
                continue
    a = np.array(rows)
    return a[:, 0], a[:, 1]
