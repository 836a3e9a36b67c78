"""[1] State -- the particle container of the reference
(python/morphompm/state.py:11-31): arrays x (n,3), v (n,3), C (n,3,3),
F (n,3,3), Fg (n,3,3).  The arrays may be numpy arrays (the reference's type;
they are moved to the GPU for every call and results come back as numpy) or
torch CUDA tensors (float64 selects the FP64 path, float32 the FP32 path; they
stay on the device).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np


@dataclass
class ParticleState:
    x: Any    # (n, 3) position
    v: Any    # (n, 3) velocity
    C: Any    # (n, 3, 3) APIC affine
    F: Any    # (n, 3, 3) total deformation gradient
    Fg: Any   # (n, 3, 3) growth tensor

    @property
    def n(self) -> int:
        return self.x.shape[0]

    @staticmethod
    def rest(x0) -> "ParticleState":
        """Particles at rest: v=C=0, F=Fg=I (state.py:23-31)."""
        try:
            import torch
            if isinstance(x0, torch.Tensor):
                n = x0.shape[0]
                I = torch.eye(3, dtype=x0.dtype, device=x0.device).expand(n, 3, 3)
                return ParticleState(x=x0.clone(), v=torch.zeros_like(x0),
                                     C=torch.zeros(n, 3, 3, dtype=x0.dtype, device=x0.device),
                                     F=I.clone(), Fg=I.clone())
        except ImportError:  # pragma: no cover
            pass
        n = x0.shape[0]
        I = np.tile(np.eye(3), (n, 1, 1))
        return ParticleState(x=x0.copy(), v=np.zeros((n, 3)), C=np.zeros((n, 3, 3)), F=I.copy(), Fg=I.copy())
