"""pictor_b200 -- the particle-in-cell time step of PICTOR on NVIDIA B200.

Hand-written CUDA for sm_100a behind a C ABI (``include/pictor_b200.h``);
this package holds the kernels (``csrc/``), their in-tree build and a thin
host-side mirror of the reference's GPU entry points.
"""
from ._capi import PicError, lib, library_path  # noqa: F401
from .simulation import Fields, Particles, PicConfig, Simulation, init_scale, step_many  # noqa: F401

__all__ = ["PicError", "lib", "library_path", "Fields", "Particles", "PicConfig", "Simulation", "init_scale",
           "step_many"]
