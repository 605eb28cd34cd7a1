"""B200-native exterior Burton-Miller BEM solve (HornSculpt's CudaBemSolver path).

The compute path is libhs_bem.so (C ABI in include/hs_bem.h, sm_100a
kernels); this package is its Python host mirror plus synthetic meshes.
"""
from .bem import (AcousticMedium, BemBoundaryData, BemCancelled, BemError, BemExcitation, BemExcitationResult,
                  BemFrequencyResult, BemNumerics, BemRequest, BemResult, BemUnsupported, CudaBemSolver,
                  CudaStorageOptions, FaceImpedance, FaceVelocity, FarFieldObservation, FastMultipoleSettings,
                  StopToken, host_plan)
from .meshes import DRIVEN, WALL, SurfaceMesh, icosphere, octahedral_sphere, scalene_tetrahedron

__all__ = [
    "AcousticMedium", "BemBoundaryData", "BemCancelled", "BemError", "BemExcitation", "BemExcitationResult",
    "BemFrequencyResult", "BemNumerics", "BemRequest", "BemResult", "BemUnsupported", "CudaBemSolver",
    "CudaStorageOptions", "FaceImpedance", "FaceVelocity", "FarFieldObservation", "FastMultipoleSettings",
    "StopToken", "host_plan", "DRIVEN", "WALL", "SurfaceMesh", "icosphere", "octahedral_sphere",
    "scalene_tetrahedron",
]
