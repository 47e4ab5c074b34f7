"""remd_b200 -- a B200-native engine for the replica-exchange MD hot path of
rigid water (TIP3P/TIP4P/TIP5P): switched LJ + Coulomb forces, the nanotube /
slit wall, the Nose-Poincare / Andersen quaternion integrator and the
Metropolis T/P exchange, behind the reference's REMDGPU call surface.

The compute path is the CUDA library remd_b200/_lib/libremd_b200.so, reached
through the C-ABI declared in include/remd_b200.h; remd_b200.engine loads it
and raises if it is missing.  Importing this package loads nothing.
"""
__all__ = ["inputs", "systems", "engine"]
