"""qj: B200 (sm_100a) kick-drift-kick Schroedinger-Poisson step of
quantum-jax, behind the C ABI of libqj.so (include/qj.h)."""

from ._lib import QjError, lib  # noqa: F401
from .core import (FUSED_F32, PLAIN_F64, Ensemble, Grid, HostPipeline, Phys, Plan,  # noqa: F401
                   StarsStep)
