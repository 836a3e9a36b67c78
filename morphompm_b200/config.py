"""[0] Config -- material and discretisation, field-for-field the reference's
``Material`` / ``SimConfig`` (python/morphompm/config.py:7-40).

Optional fields extend it for the B200 path without changing any default:
a non-cubic ``shape`` (defaults to (N, N, N)), sticky ``wall`` nodes, a sticky
``clamp`` box, ``gravity`` and the grid-mass threshold ``mass_eps``
(transfer.py:56 uses 1e-12); the arithmetic type ``dtype`` ("float32" or
"float64"; default: that of the inputs, numpy arrays run in float64), the
CUDA ``device`` (default: the inputs' or the current one) and
``checkpoint_every`` (default: keep every step) of the trajectory gradients.
The JSON config files keep the reference's fields only (io.py:98-111).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple


@dataclass
class Material:
    E: float = 1.0e4          # Young's modulus [Pa]
    nu: float = 0.3           # Poisson ratio
    density: float = 1000.0   # [kg/m^3]

    @property
    def mu(self) -> float:
        return self.E / (2.0 * (1.0 + self.nu))

    @property
    def lam(self) -> float:
        return self.E * self.nu / ((1.0 + self.nu) * (1.0 - 2.0 * self.nu))


@dataclass
class SimConfig:
    N: int = 8                 # dense grid resolution per axis
    dx: float = 0.1
    dt: float = 1.0e-3
    damping: float = 0.05      # quasi-static relaxation per step
    sp: float = 0.02           # particle spacing (sets mass/volume)
    material: Material = field(default_factory=Material)
    # -- extensions (defaults = reference behaviour) --
    shape: Optional[Tuple[int, int, int]] = None
    wall: int = 0
    clamp_lo: Sequence[int] = (0, 0, 0)
    clamp_hi: Sequence[int] = (0, 0, 0)
    gravity: Sequence[float] = (0.0, 0.0, 0.0)
    mass_eps: float = 1.0e-12
    dtype: Optional[str] = None
    device: Optional[str] = None
    checkpoint_every: Optional[int] = None

    @property
    def inv_dx(self) -> float:
        return 1.0 / self.dx

    @property
    def pmass(self) -> float:
        return self.material.density * self.sp ** 3

    @property
    def vol0(self) -> float:
        return self.sp ** 3    # = pmass / density

    @property
    def grid_shape(self) -> Tuple[int, int, int]:
        return tuple(self.shape) if self.shape is not None else (self.N, self.N, self.N)


_DTYPES = ("float32", "float64")


def compute_target(cfg):
    """(torch dtype or None, device or None) that ``cfg`` asks the device path
    to compute in; None leaves the choice to the inputs.  Configs without the
    extension fields (the reference's own SimConfig) ask for nothing."""
    dt = getattr(cfg, "dtype", None)
    if dt is not None and dt not in _DTYPES:
        raise ValueError(f"SimConfig.dtype must be one of {_DTYPES} or None, not {dt!r}")
    if dt is not None:
        import torch
        dt = getattr(torch, dt)
    return dt, getattr(cfg, "device", None)
