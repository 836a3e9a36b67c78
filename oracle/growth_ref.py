"""ctypes wrapper of oracle/_ref/libgrowth_ref.so: the reference's C++ FP32
forward solver (include/morphompm/growth_solver.h) built by build_ref.py.
Test and measurement infrastructure only."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libgrowth_ref.so")
_lib = None


def available() -> bool:
    return os.path.isfile(LIB)


def _load():
    global _lib
    if _lib is None:
        lib = C.CDLL(LIB)
        f, i, ll, vp = C.c_float, C.c_int, C.c_longlong, C.c_void_p
        fp = C.POINTER(C.c_float)
        lib.ref_create.restype = vp
        lib.ref_create.argtypes = [i, f, f, f, f, f, f, f]
        lib.ref_destroy.argtypes = [vp]
        lib.ref_add.argtypes = [vp, ll, fp, f, f]
        lib.ref_add_each.argtypes = [vp, ll, fp, fp, fp]
        lib.ref_set_growth.argtypes = [vp, f]
        lib.ref_set_growth_tensors.argtypes = [vp, fp]
        lib.ref_step.argtypes = [vp, f, i]
        lib.ref_get.argtypes = [vp, fp, fp, fp, fp]
        _lib = lib
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class RefSolver:
    """GrowthSolver(N, dx) with E, nu, damping and gravity set (growth_solver.h:44-55)."""

    def __init__(self, N, dx, E=1e4, nu=0.3, damping=0.0, gravity=(0.0, 0.0, 0.0)):
        self.lib = _load()
        self.h = self.lib.ref_create(int(N), float(dx), float(E), float(nu), float(damping), *map(float, gravity))
        self.n = 0

    def add(self, x, mass, density):
        x = np.ascontiguousarray(x, dtype=np.float32)
        self.lib.ref_add(self.h, x.shape[0], _fp(x), float(mass), float(density))
        self.n += x.shape[0]

    def add_each(self, x, mass, density):
        x = np.ascontiguousarray(x, dtype=np.float32)
        m = np.ascontiguousarray(mass, dtype=np.float32)
        d = np.ascontiguousarray(density, dtype=np.float32)
        self.lib.ref_add_each(self.h, x.shape[0], _fp(x), _fp(m), _fp(d))
        self.n += x.shape[0]

    def set_growth(self, g):
        self.lib.ref_set_growth(self.h, float(g))

    def set_growth_tensors(self, Fg):
        Fg = np.ascontiguousarray(Fg, dtype=np.float32).reshape(self.n, 3, 3)
        self.lib.ref_set_growth_tensors(self.h, _fp(Fg))

    def step(self, dt, steps=1):
        self.lib.ref_step(self.h, float(dt), int(steps))

    def get(self):
        x = np.zeros((self.n, 3), np.float32)
        v = np.zeros((self.n, 3), np.float32)
        F = np.zeros((self.n, 3, 3), np.float32)
        Cm = np.zeros((self.n, 3, 3), np.float32)
        self.lib.ref_get(self.h, _fp(x), _fp(v), _fp(F), _fp(Cm))
        return x, v, F, Cm

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None


def blob(center, half, sp):
    """Particles on the lattice of the reference's C++ tests: for each axis
    c - h, c - h + sp, ... <= c + h + 1e-6, accumulated in single precision
    as its loops do (test_growth.cpp:44-52, 123-127, 341-344)."""
    c = np.broadcast_to(np.asarray(center, dtype=np.float64), 3)
    h = np.broadcast_to(np.asarray(half, dtype=np.float64), 3)
    axes = []
    for d in range(3):
        vals = []
        lo, hi = np.float32(np.float32(c[d]) - np.float32(h[d])), np.float32(np.float32(c[d]) + np.float32(h[d]))
        x = lo
        while x <= np.float32(hi + np.float32(1e-6)):
            vals.append(x)
            x = np.float32(x + np.float32(sp))
        axes.append(vals)
    return np.array([(a, b, e) for a in axes[0] for b in axes[1] for e in axes[2]], dtype=np.float32)


def parity_cube(sp=0.03, lo=0.27, hi=0.33):
    """The 27-particle cube of the reference's parity scene (test_growth.cpp:341-344)."""
    pts = []
    x = np.float32(lo)
    while x <= np.float32(hi) + np.float32(1e-6):
        y = np.float32(lo)
        while y <= np.float32(hi) + np.float32(1e-6):
            z = np.float32(lo)
            while z <= np.float32(hi) + np.float32(1e-6):
                pts.append((x, y, z))
                z = np.float32(z + np.float32(sp))
            y = np.float32(y + np.float32(sp))
        x = np.float32(x + np.float32(sp))
    return np.array(pts, dtype=np.float32)
