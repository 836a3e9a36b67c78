"""ctypes binding of the C ABI in ``include/morphompm_b200.h``.

The shared library is built in-tree (``python -m morphompm_b200.build``).  There
is no CPU fallback: if the library is missing or no CUDA device is present, the
first call raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB, LIB_CHECKED, build, up_to_date

# MORPHOMPM_CHECKED=1: the bounds-checked build of the same sources
CHECKED = os.environ.get("MORPHOMPM_CHECKED", "0") == "1"

MPM_OK = 0
MPM_ERR_ARG = 1
MPM_ERR_CUDA = 2
MPM_ERR_NONFINITE = 4
MPM_WARN_OUTSIDE = 8
MPM_ERR_TAPE = 16
MPM_ERR_UNSUPPORTED = 32
MPM_ERR_TOO_LARGE = 64
MPM_FWD_CHAINED = 1
MPM_FWD_EMIT = 2

KERNELS = ["bin", "sort", "mark", "compact", "prepass", "p2g", "g2p", "bwd_payload", "bwd_p2g",
           "bwd_particle", "reduce"]

MODEL_NEOHOOKEAN = 0
MODEL_HENCKY = 1
MODEL_EXTERNAL = 3
MODEL_HERSCHEL_BULKLEY = 2

i32, i64, f32, f64, vp = C.c_int32, C.c_int64, C.c_float, C.c_double, C.c_void_p


class MpmScene(C.Structure):
    _fields_ = [
        ("shape", i32 * 3), ("model", i32),
        ("p_begin", i64), ("p_end", i64),
        ("wall", i32), ("clamp_lo", i32 * 3), ("clamp_hi", i32 * 3), ("growth_mode", i32),
        ("dx", f64), ("dt", f64), ("damping", f64), ("pmass", f64), ("vol0", f64),
        ("mass_eps", f64), ("gravity", f64 * 3),
        ("mu", f64), ("lam", f64),
        ("kappa", f64), ("K", f64), ("n_exp", f64), ("tau_y", f64), ("m_pap", f64), ("eps", f64),
        ("growth_A", f64), ("ramp_steps", f64),
    ]


class MpmParticles(C.Structure):
    _fields_ = [("x", vp), ("v", vp), ("C", vp), ("F", vp), ("Fg", vp),
                ("sp3", i64), ("sc3", i64), ("sp9", i64), ("sc9", i64)]


class MpmCotangents(C.Structure):
    _fields_ = [("x", vp), ("v", vp), ("C", vp), ("F", vp), ("Fg", vp),
                ("sp3", i64), ("sc3", i64), ("sp9", i64), ("sc9", i64)]


class MpmTuning(C.Structure):
    _fields_ = [("tile_xy", i32), ("scatter_ctas_per_sm", i32), ("scatter_oxb", i32),
                ("particle_block", i32), ("active_tile_cap", i32), ("fp64_gap_thresh", f32),
                ("tile_z", i32)]


EXPORTS = {
    "mpm_version": (i32, []),
    "mpm_plan_create": (i32, [C.POINTER(MpmScene), i32, i32, C.POINTER(MpmTuning), C.POINTER(vp)]),
    "mpm_plan_destroy": (None, [vp]),
    "mpm_plan_workspace_bytes": (i32, [vp, C.POINTER(C.c_size_t)]),
    "mpm_plan_tape_bytes": (i32, [vp, C.POINTER(C.c_size_t)]),
    "mpm_plan_num_particles": (i64, [vp]),
    "mpm_plan_bind": (i32, [vp, vp, vp]),
    "mpm_plan_read_status": (i32, [vp, C.POINTER(i32), vp]),
    "mpm_plan_read_fp64_fallbacks": (i32, [vp, C.POINTER(i64), vp]),
    "mpm_plan_set_growth_field": (i32, [vp, vp]),
    "mpm_plan_set_particle_mass": (i32, [vp, vp, vp]),
    "mpm_plan_set_external_stress": (i32, [vp, vp, vp]),
    "mpm_plan_profile_begin": (i32, [vp, C.c_uint32, i32]),
    "mpm_plan_profile_end": (i32, [vp, C.POINTER(f64), C.POINTER(i32)]),
    "mpm_plan_launch_count": (i64, [vp]),
    "mpm_plan_active_tiles": (i32, [vp, vp, C.POINTER(i32), vp]),
    "mpm_plan_update_scenes": (i32, [vp, C.POINTER(MpmScene), i32, vp]),
    "mpm_step_fwd": (i32, [vp, C.POINTER(MpmParticles), C.POINTER(MpmParticles), i32, i32, vp, vp]),
    "mpm_step_fwd_chain": (i32, [vp, C.POINTER(MpmParticles), C.POINTER(MpmParticles), i32, i32, vp, i32, vp]),
    "mpm_step_bwd": (i32, [vp, C.POINTER(MpmParticles), vp, C.POINTER(MpmCotangents),
                           C.POINTER(MpmCotangents), vp, i32, i32, vp, vp]),
    "mpm_step_bwd_params": (i32, [vp, C.POINTER(MpmParticles), vp, C.POINTER(MpmCotangents),
                                  C.POINTER(MpmCotangents), vp, vp, i32, i32, vp, vp]),
    "mpm_stress": (i32, [C.POINTER(MpmScene), i32, i64, vp, vp, vp, vp, vp]),
    "mpm_stress_vjp": (i32, [C.POINTER(MpmScene), i32, i64, vp, vp, vp, vp, vp, vp, vp, vp]),
    "mpm_bin_keys": (i32, [C.POINTER(MpmScene), i32, i64, vp, vp, vp]),
    "mpm_rollout_workspace_bytes": (i32, [vp, i32, i32, C.POINTER(C.c_size_t)]),
    "mpm_rollout_fwd": (i32, [vp, vp, vp, i32, i32, i32, vp, vp, vp]),
    "mpm_rollout_bwd": (i32, [vp, vp, vp, i32, i32, i32, vp, vp, vp, vp, vp, vp]),
    "mpm_loss_detF": (i32, [vp, vp, i64, i64, vp, vp, vp]),
    "mpm_loss_mse": (i32, [vp, vp, i64, i64, vp, vp, vp, vp]),
    "mpm_step_fwd_noalloc": (i32, [C.POINTER(MpmScene), i32, C.POINTER(MpmParticles), C.POINTER(MpmParticles),
                                   i32, i32, C.POINTER(i32), vp]),
    "mpm_check_violations": (i32, [C.POINTER(i64), C.POINTER(i32), C.POINTER(i64), vp]),
}

_lib = None


def lib_path() -> str:
    return LIB_CHECKED if CHECKED else LIB


def load(build_if_missing: bool = True):
    """Load the shared library (building it first if sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path) or (build_if_missing and not up_to_date(CHECKED)):
        if not build_if_missing:
            raise RuntimeError(f"morphompm_b200 CUDA library not built: {path}")
        build(checked=CHECKED)
    lib = C.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MpmError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        names = [n for n, b in (("ARG", 1), ("CUDA", 2), ("NONFINITE", 4), ("OUTSIDE", 8),
                                ("TAPE", 16), ("UNSUPPORTED", 32)) if code & b]
        super().__init__(f"morphompm_b200 {where} failed: status {code} ({'|'.join(names)})")


def check(code, where=""):
    if code != MPM_OK:
        raise MpmError(code, where)
