"""B200-native exterior Burton-Miller BEM solve (HornSculpt's CudaBemSolver path).

The compute path is libhs_bem.so (C ABI in include/hs_bem.h, sm_100a
kernels); this package is its Python host mirror plus synthetic meshes.
"""
from .bem import (AcousticMedium, BemBoundaryData, BemCancelled, BemError, BemExcitation, BemExcitationResult,
                  BemFrequencyResult, BemNumerics, BemRequest, BemResult, BemServer, BemUnsupported, CudaBemSolver,
                  CudaStorageOptions, FaceImpedance, FaceVelocity, FarFieldObservation, FastMultipoleSettings,
                  FieldPointStatus, PressureFieldSample, PressureFieldSettings, ServeOptions, ServeTiming, StopToken,
                  autotune_clear, autotune_enable, autotune_report, debug_lu_factor, device_plan, host_plan)
from .coupling import BemPort, CouplingBasis, PortSolution, coupled_solve, make_coupling_basis, port_impedance
from .fixtures import read_fixture, write_fixture
from .study import StudyRequest, complex_result_document, describe_study_capabilities, parse_study_request
from .meshes import (DRIVEN, WALL, SurfaceMesh, exponential_horn, icosphere, octahedral_sphere, revolved_sphere,
                     scalene_tetrahedron)

__all__ = [
    "AcousticMedium", "BemBoundaryData", "BemCancelled", "BemError", "BemExcitation", "BemExcitationResult",
    "BemFrequencyResult", "BemNumerics", "BemRequest", "BemResult", "BemServer", "BemUnsupported", "CudaBemSolver",
    "CudaStorageOptions", "FaceImpedance", "FaceVelocity", "FarFieldObservation", "FastMultipoleSettings",
    "FieldPointStatus", "PressureFieldSample", "PressureFieldSettings",
    "ServeOptions", "ServeTiming", "StopToken", "autotune_clear", "autotune_enable", "autotune_report", "debug_lu_factor", "device_plan", "host_plan", "DRIVEN", "WALL", "SurfaceMesh", "exponential_horn",
    "icosphere", "octahedral_sphere", "revolved_sphere", "scalene_tetrahedron", "read_fixture", "write_fixture", "StudyRequest", "parse_study_request",
    "describe_study_capabilities", "complex_result_document", "BemPort", "CouplingBasis", "PortSolution",
    "coupled_solve", "make_coupling_basis", "port_impedance",
]
