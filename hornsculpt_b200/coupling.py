"""The BEM side of lumped-element (LEM) coupling: unit-port basis, port radiation
impedance, coupled superposition and the pressure-closure check.

In the reference, a coupled request solves the Burton–Miller system once per port,
for a unit volume velocity Q = 1 entering the air domain through that port's faces
(``makeCouplingBasis``, ``modules/bem/lem_coupling.cpp:9-87``). From those solves it
builds the port impedance matrix Z_ij. This is the power-dual mean pressure at port
i per unit flow at port j (``cuda_solver.cu:1584-1606``). The lumped network
(``lem::solve``) then yields the port flows Q_j. The coupled field is the
superposition sum_j p_j Q_j (``:1608-1630``). Its port pressures must close with
the network's to a relative 1e-3 (``validateCouplingClosure``,
``lem_coupling.cpp:97-120``).

Here the unit-port solves are one multi-excitation request of this solver. The
network solver is the caller's (the reference's ``modules/lem`` is not part of this
library): a callable that maps (frequency, Z) to the port flows and pressures.
The coupled result comes from superposing the basis solutions, which the
linearity of the discrete system makes exact. The reference refines the combined
equation once more with its retained factors. The dense forms here already solve
each basis system to the request's residual tolerance.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Dict, List, Sequence, Tuple

import numpy as np

from .bem import BemExcitation, BemRequest, FaceVelocity
from .meshes import DRIVEN, SurfaceMesh

# lem_coupling.cpp / bem.hpp: relativePortPressureClosureTolerance
PORT_PRESSURE_CLOSURE_TOLERANCE = 1e-3


@dataclasses.dataclass
class BemPort:
    """A driven-surface port of the network (lem.hpp BemPort): its faces, and a
    positive velocity shape per face (missing faces weigh 1)."""
    name: str
    face_ids: Sequence[int]
    velocity_weights: Dict[int, float] = dataclasses.field(default_factory=dict)


@dataclasses.dataclass
class CouplingBasis:
    """Unit-flow excitations per port, modal areas S_w = sum w_f A_f, the port of each
    panel (-1 outside the ports) and its normal velocity for Q = 1, w_f / S_w."""
    excitations: List[BemExcitation]
    areas: List[float]
    panel_ports: np.ndarray
    panel_velocities: np.ndarray


@dataclasses.dataclass
class PortSolution:
    """The network's answer at one frequency: volume velocity and pressure per port."""
    volume_velocity: complex
    pressure: complex


def _panel_areas(mesh: SurfaceMesh) -> np.ndarray:
    v = mesh.vertices[mesh.triangles]
    return 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)


def make_coupling_basis(ports: Sequence[BemPort], mesh: SurfaceMesh) -> CouplingBasis:
    """makeCouplingBasis for the exterior-solid domain (lem_coupling.cpp:9-87): every
    port face must be an existing Driven face of exactly one port, and every Driven
    face must belong to a port."""
    if not ports or len(ports) > 1024:
        raise ValueError("Coupling needs between one and 1024 BEM ports.")
    areas = _panel_areas(mesh)
    faces: Dict[int, Tuple[float, int]] = {}
    for face, kind, area in zip(mesh.face_ids.tolist(), mesh.boundary.tolist(), areas.tolist()):
        a, k = faces.get(face, (0.0, kind))
        if k != kind:
            raise ValueError("Conflicting boundary conditions on one face.")
        faces[face] = (a + area, kind)
    face_port: Dict[int, int] = {}
    face_velocity: Dict[int, float] = {}
    basis = CouplingBasis([], [], np.full(mesh.triangle_count, -1, np.int32), np.zeros(mesh.triangle_count))
    for j, port in enumerate(ports):
        area = 0.0
        for fid in port.face_ids:
            found = faces.get(fid)
            if found is None or found[1] != DRIVEN or fid in face_port:
                raise ValueError("Coupled faces must exist, match their port type (Driven surface or Wall "
                                 "interface), and belong to exactly one port.")
            face_port[fid] = j
            area += port.velocity_weights.get(fid, 1.0) * found[0]
        if not (area > 0) or not np.isfinite(area):
            raise ValueError("Invalid BEM coupling port area.")
        basis.areas.append(area)
        excitation = BemExcitation(port.name, [])
        for fid in port.face_ids:
            velocity = port.velocity_weights.get(fid, 1.0) / area
            if not (velocity > 0) or not np.isfinite(velocity) or velocity > np.finfo(np.float32).max:
                raise ValueError("BEM port modal velocity exceeds storage.")
            excitation.faces.append(FaceVelocity(fid, complex(velocity)))
            face_velocity[fid] = velocity
        basis.excitations.append(excitation)
    for fid, (_, kind) in faces.items():
        if kind == DRIVEN and fid not in face_port:
            raise ValueError("Every Driven face needs a BEM port in a coupled request.")
    for t, fid in enumerate(mesh.face_ids.tolist()):
        if fid in face_port:
            basis.panel_ports[t] = face_port[fid]
            basis.panel_velocities[t] = face_velocity[fid]
    return basis


def port_impedance(basis: CouplingBasis, mesh: SurfaceMesh, surface_pressures: Sequence[np.ndarray]) -> np.ndarray:
    """Z[i, j] = sum over the panels of port i of the DP0 mean pressure of basis solve
    j times area times the panel's unit-flow velocity (cuda_solver.cu:1588-1600)."""
    areas = _panel_areas(mesh)
    P = len(basis.excitations)
    Z = np.zeros((P, P), complex)
    inside = basis.panel_ports >= 0
    weight = areas * basis.panel_velocities
    for j in range(P):
        np.add.at(Z[:, j], basis.panel_ports[inside], (surface_pressures[j] * weight)[inside])
    return Z


def coupled_velocities(basis: CouplingBasis, flows: Sequence[complex]) -> List[FaceVelocity]:
    """coupledVelocities (lem_coupling.cpp:89-96): each port's unit-flow face
    velocities scaled by its network flow."""
    if len(flows) != len(basis.excitations):
        raise ValueError("LEM result port count does not match its BEM basis.")
    return [FaceVelocity(f.face_id, f.normal_velocity * q) for e, q in zip(basis.excitations, flows) for f in e.faces]


def validate_closure(basis: CouplingBasis, mesh: SurfaceMesh, ports: Sequence[PortSolution],
                     surface_pressure: np.ndarray) -> None:
    """validateCouplingClosure (lem_coupling.cpp:97-120): the power-dual mean pressure
    of the coupled surface pressure at each port against the network's port pressure."""
    if len(ports) != len(basis.areas) or len(surface_pressure) != mesh.triangle_count:
        raise ValueError("BEM pressure-closure dimensions are inconsistent.")
    areas = _panel_areas(mesh)
    means = np.zeros(len(ports), complex)
    mags = np.zeros(len(ports))
    for t in np.nonzero(basis.panel_ports >= 0)[0]:
        w = areas[t] * basis.panel_velocities[t]
        means[basis.panel_ports[t]] += w * surface_pressure[t]
        mags[basis.panel_ports[t]] += w * abs(surface_pressure[t])
    for i, port in enumerate(ports):
        scale = max(mags[i], abs(port.pressure))
        diff = abs(means[i] - port.pressure)
        if not np.isfinite(scale) or not np.isfinite(diff) or diff > PORT_PRESSURE_CLOSURE_TOLERANCE * scale:
            raise RuntimeError("BEM and LEM port pressures fail the feedback consistency check.")


@dataclasses.dataclass
class CoupledFrequency:
    frequency: float
    impedance: np.ndarray            # Z, ports x ports, Pa s / m^3
    ports: List[PortSolution]
    face_velocities: List[FaceVelocity]
    pressure_trace: np.ndarray       # coupled P1 pressure
    surface_pressure: np.ndarray     # coupled DP0 mean pressure
    observer_pressure: np.ndarray


def coupled_solve(solver, mesh: SurfaceMesh, ports: Sequence[BemPort], request: BemRequest,
                  network: Callable[[float, np.ndarray], Sequence[PortSolution]]) -> List[CoupledFrequency]:
    """Unit-port basis solves (one request, one excitation per port), port impedance,
    the caller's network, coupled superposition and the closure check per frequency.
    `request` supplies frequencies, observers, medium and numerics; its excitations
    are replaced by the basis."""
    basis = make_coupling_basis(ports, mesh)
    basis_request = dataclasses.replace(request, excitations=basis.excitations)
    result = solver.solve(basis_request)
    out = []
    for frame in result.frequencies:
        surfaces = [e.boundary.surface_pressure for e in frame.excitations]
        Z = port_impedance(basis, mesh, surfaces)
        solution = list(network(frame.frequency, Z))
        flows = np.array([s.volume_velocity for s in solution], complex)
        trace = sum(e.boundary.pressure_trace * q for e, q in zip(frame.excitations, flows))
        surface = sum(s * q for s, q in zip(surfaces, flows))
        observer = sum(e.observer_pressure * q for e, q in zip(frame.excitations, flows))
        validate_closure(basis, mesh, solution, surface)
        out.append(CoupledFrequency(frame.frequency, Z, solution, coupled_velocities(basis, flows), trace, surface,
                                    observer))
    return out
