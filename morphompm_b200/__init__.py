"""morphompm_b200 -- B200-native (sm_100a) differentiable MLS-MPM growth step.

Modules mirror the reference package (2nugu/morphompm, python/morphompm):
config, state, constitutive, transfer, integrate, diff.  The kernels live in
``csrc/`` behind the C ABI declared in ``include/morphompm_b200.h``; ``batch``
adds batched, graph-captured trajectories of many uneven scenes.
"""
from importlib import import_module

__all__ = ["config", "state", "constitutive", "transfer", "integrate", "diff", "batch", "scenes"]


def __getattr__(name):
    if name in __all__:
        return import_module(f".{name}", __name__)
    raise AttributeError(name)
