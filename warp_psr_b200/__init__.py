"""B200-native screened-Poisson surface reconstruction with warp-psr's API.

``reconstruct(positions, normals, **options)`` runs the whole degree-1 PSR/SPSR path —
sample grouping, density and normal splats, tree, cascadic solve, field and isovalue —
as hand-written sm_100a CUDA kernels in ``libpsr_b200.so`` behind a C ABI.
"""
from .reconstruction import (reconstruct, reconstruct_differentiable, Reconstruction, DifferentiableReconstruction,
                             LevelField, DeviceField)
from . import ops

__all__ = ["reconstruct", "reconstruct_differentiable", "Reconstruction", "DifferentiableReconstruction",
           "LevelField", "DeviceField", "ops"]
