"""B200-native (sm_100a) implementation of the PCOM v2.2 baroclinic time step.

Public pieces:
  pcom_b200.model.Model   -- the time-stepping driver (mirrors main.f90)
  pcom_b200.synth         -- seeded synthetic input cases
  include/pcom_gpu.h      -- the C ABI a Fortran driver binds
"""
from . import synth  # noqa: F401

__all__ = ["synth", "model", "build"]
