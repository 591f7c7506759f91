"""B200-native CaMa-Flood v4 physics time step (CMF_PHYSICS_ADVANCE) behind the reference's
driver boundary.  See include/cmf_gpu.h for the C ABI; this package is its Python host side."""
from .model import HostModel, PhysicsBatch, PhysicsGPU  # noqa: F401
from . import synth  # noqa: F401

__all__ = ["HostModel", "PhysicsGPU", "synth"]
