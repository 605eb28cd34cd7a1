"""Python mirror of HornSculpt's BEM solver interface
(``modules/bem/include/hornsculpt/bem.hpp:27-388``) over the C ABI of
libhs_bem.so. Names, defaults, units and error classes follow the reference:
invalid meshes and requests raise ValueError (std::invalid_argument), device,
numerical and convergence failures raise BemError (std::runtime_error).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import functools
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import BemCancelled, BemError, BemUnsupported  # noqa: F401  (re-exported)
from .meshes import SurfaceMesh


@dataclasses.dataclass
class AcousticMedium:
    density: float = 1.21
    sound_speed: float = 343.0


@dataclasses.dataclass
class FaceVelocity:
    face_id: int
    normal_velocity: complex = 1.0 + 0.0j  # RMS m/s, out of the solid


@dataclasses.dataclass
class BemExcitation:
    name: str
    faces: list


@dataclasses.dataclass
class FastMultipoleSettings:
    leaf_support_capacity: int = 16
    separation_ratio: float = 1.5
    maximum_iterations: int = 300
    restart_length: int = 40
    preconditioner_block_width: int = 32


@dataclasses.dataclass
class BemNumerics:
    quadrature_order: int = 4
    singular_order: int = 4
    near_distance_ratio: float = 1.0
    near_relative_tolerance: float = 1e-4
    near_maximum_depth: int = 6
    relative_residual_tolerance: float = 5e-5
    maximum_refinement_steps: int = 3
    acceleration: str = "dense"  # "dense" | "fast_multipole"
    precision: str = "fp64"      # "fp64" (plain form) | "mixed" (FP32 samples and LU, FP64 refinement)
    fast_multipole: FastMultipoleSettings = dataclasses.field(default_factory=FastMultipoleSettings)

    def to_c(self) -> _lib.hs_numerics:
        n = _lib.hs_numerics()
        n.quadrature_order = self.quadrature_order
        n.singular_order = self.singular_order
        n.near_distance_ratio = self.near_distance_ratio
        n.near_relative_tolerance = self.near_relative_tolerance
        n.near_maximum_depth = self.near_maximum_depth
        n.relative_residual_tolerance = self.relative_residual_tolerance
        n.maximum_refinement_steps = self.maximum_refinement_steps
        n.acceleration = {"dense": 0, "fast_multipole": 1}.get(self.acceleration, 99)
        n.precision = {"fp64": 0, "mixed": 1}.get(self.precision, 99)
        f = self.fast_multipole
        n.fmm_leaf_support_capacity = f.leaf_support_capacity
        n.fmm_separation_ratio = f.separation_ratio
        n.fmm_maximum_iterations = f.maximum_iterations
        n.fmm_restart_length = f.restart_length
        n.fmm_preconditioner_block_width = f.preconditioner_block_width
        return n


@dataclasses.dataclass
class FarFieldObservation:
    origin: tuple = (0.0, 0.0, 0.0)
    reference_distance: float = 1.0


@dataclasses.dataclass
class BemRequest:
    frequencies: Sequence[float]
    excitations: Sequence[BemExcitation]
    observers: Sequence[Sequence[float]] = ()
    medium: AcousticMedium = dataclasses.field(default_factory=AcousticMedium)
    numerics: BemNumerics = dataclasses.field(default_factory=BemNumerics)
    far_field: Optional[FarFieldObservation] = None
    interaction_plan_frequencies: Sequence[float] = ()


@dataclasses.dataclass
class FaceImpedance:
    face_id: int
    area: float
    mean_pressure: complex
    volume_velocity: complex
    volume_impedance: complex


@dataclasses.dataclass
class BemBoundaryData:
    surface_pressure: np.ndarray   # DP0 mean pressure per triangle
    pressure_trace: np.ndarray     # P1 pressure per vertex
    normal_derivative: np.ndarray  # DP0 q = -i rho omega v per triangle


@dataclasses.dataclass
class BemExcitationResult:
    name: str
    observer_pressure: np.ndarray
    impedances: list
    refinement_steps: int
    boundary_residual: float
    field_quadrature_comparison_degree: int
    field_quadrature_verification_degree: int
    field_quadrature_discrepancy: float
    boundary: BemBoundaryData
    iterations: int = 0


@dataclasses.dataclass
class BemFrequencyResult:
    frequency: float
    excitations: list
    assembly_milliseconds: float
    solve_milliseconds: float
    factorization_milliseconds: float
    triangular_solve_milliseconds: float
    field_milliseconds: float
    residual_check_milliseconds: float
    interaction_plan_milliseconds: float
    interaction_plan_reused: bool


@dataclasses.dataclass
class BemResult:
    device: str
    triangle_count: int
    pressure_dof_count: int
    peak_device_bytes: int
    frequencies: list
    acceleration: str = "dense"


class FieldPointStatus(enum.IntEnum):
    """Status of a pressure field sample (field_evaluation.hpp:8)."""
    AIR = 0
    BOUNDARY = 1
    EXCLUDED = 2
    QUADRATURE_NOT_CONVERGED = 3


@dataclasses.dataclass
class PressureFieldSettings:
    """Sampling settings of evaluatePressureField (field_evaluation.hpp:14-20)."""
    minimum_boundary_distance: float = 1e-4  # m; a sampling exclusion distance
    relative_quadrature_tolerance: float = 1e-4
    maximum_quadrature_depth: int = 8


@dataclasses.dataclass
class PressureFieldSample:
    position: tuple
    pressure: complex
    status: FieldPointStatus


class StopToken:
    """Cooperative cancellation flag polled by the solver between device batches."""

    def __init__(self):
        self._flag = C.c_int32(0)

    def request_stop(self):
        self._flag.value = 1

    @property
    def stop_requested(self) -> bool:
        return bool(self._flag.value)


@dataclasses.dataclass
class CudaStorageOptions:
    quadrature_patches: str = "automatic"  # "automatic" | "device" | "mapped_host"


def _cplx(buf: np.ndarray) -> np.ndarray:
    return buf[0::2] + 1j * buf[1::2]


class CudaBemSolver:
    """One closed exterior surface mesh resident on the current CUDA device."""

    def __init__(self, mesh: SurfaceMesh, storage: CudaStorageOptions = CudaStorageOptions()):
        lib = _lib.load()
        residency = {"automatic": 0, "device": 1, "mapped_host": 2}.get(storage.quadrature_patches, 99)
        self._mesh = mesh
        handle = C.c_void_p()
        _lib.check(lib.hs_bem_session_create(mesh.vertices.ctypes.data, mesh.vertex_count, mesh.triangles.ctypes.data,
                                             mesh.face_ids.ctypes.data, mesh.boundary.ctypes.data,
                                             mesh.triangle_count, residency, C.byref(handle)))
        self._handle = handle
        self._lib = lib

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.hs_bem_session_destroy(self._handle)
            self._handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    @functools.lru_cache(maxsize=None)
    def device_description() -> str:
        buf = C.create_string_buffer(256)
        _lib.check(_lib.load().hs_device_description(buf, 256))
        return buf.value.decode()

    def set_stream(self, cuda_stream: int | None) -> None:
        _lib.check(self._lib.hs_bem_session_set_stream(self._handle, C.c_void_p(cuda_stream or 0)))

    def set_profiling(self, enabled: bool) -> None:
        _lib.check(self._lib.hs_bem_session_set_profiling(self._handle, int(enabled)))

    def profile(self) -> dict:
        """{kernel family: (milliseconds, launches)} of the CUDA events recorded so far."""
        cap = 64
        names = C.create_string_buffer(4096)
        ms = (C.c_double * cap)()
        launches = (C.c_uint64 * cap)()
        count = C.c_size_t()
        _lib.check(self._lib.hs_bem_session_profile(self._handle, names, 4096, ms, launches, cap, C.byref(count)))
        keys = names.value.decode().split(",") if count.value else []
        return {k: (ms[i], launches[i]) for i, k in enumerate(keys)}

    WORK_KEYS = ("pairs_q6", "pairs_q12", "pairs_q16", "pairs_q64", "regular_samples", "singular_samples",
                 "near_samples", "frequencies")

    def set_plane_wave_threshold(self, threshold: float) -> None:
        """k x shortest M2L distance from which a fast-multipole level translates in the plane-wave form."""
        _lib.check(self._lib.hs_bem_session_set_plane_wave_threshold(self._handle, threshold))

    def set_planner(self, planner: str) -> None:
        """Interaction planner: "device" (default; the pair refinement on the GPU) or "host" (host threads,
        like the reference). Both give the same plan bit for bit."""
        _lib.check(self._lib.hs_bem_session_set_planner(self._handle, {"device": 0, "host": 1}[planner]))

    def plan_stats(self) -> dict:
        """Statistics of the session's last device plan (see device_plan)."""
        stats = (C.c_double * 20)()
        _lib.check(self._lib.hs_bem_session_plan_stats(self._handle, stats))
        return dict(zip(PLAN_STATS, list(stats)))

    def set_fmm_grouped_m2l(self, enabled: bool) -> None:
        """Rotational M2L grouped by translation class (default) or one CTA per target node."""
        _lib.check(self._lib.hs_bem_session_set_fmm_grouped_m2l(self._handle, 1 if enabled else 0))

    def set_fmm_audit(self, mode: str) -> None:
        """Fast-multipole acceptance audit: "automatic" (the reference's policy), "expansion" (finer
        expansions and panel-rule promotion) or "direct" (the exact dense system's residual)."""
        code = {"automatic": 0, "expansion": 1, "direct": 2}[mode]
        _lib.check(self._lib.hs_bem_session_set_fmm_audit(self._handle, code))

    def fmm_audit_counts(self) -> tuple:
        """(direct audits, far-field panel-rule promotions) of this session so far."""
        d, q = C.c_uint64(), C.c_uint64()
        _lib.check(self._lib.hs_bem_session_fmm_audit_counts(self._handle, C.byref(d), C.byref(q)))
        return d.value, q.value

    def set_graphs(self, enabled: bool) -> None:
        """Replay of the dense batch chain and the fast-multipole far-field apply as captured CUDA graphs."""
        _lib.check(self._lib.hs_bem_session_set_graphs(self._handle, int(enabled)))

    def graph_launches(self) -> int:
        """Dense-chain graph replays of this session so far."""
        n = C.c_uint64()
        _lib.check(self._lib.hs_bem_session_graph_launches(self._handle, C.byref(n)))
        return n.value

    def work(self) -> dict:
        """Work counters (pairs per regular rule, samples per pair class) since profiling was enabled."""
        buf = (C.c_uint64 * 8)()
        count = C.c_size_t()
        _lib.check(self._lib.hs_bem_session_work(self._handle, buf, 8, C.byref(count)))
        return {k: int(buf[i]) for i, k in enumerate(self.WORK_KEYS[: count.value])}

    def solve(self, request: BemRequest, stop: StopToken | None = None,
              progress: Callable | None = None) -> BemResult:
        req, keep = self._c_request(request)
        out = C.c_void_p()
        cb = _lib.PROGRESS_FN(lambda p, _u: progress(p.contents) if progress else None) if progress else \
            _lib.PROGRESS_FN()
        flag = C.byref(stop._flag) if stop is not None else None
        _lib.check(self._lib.hs_bem_solve(self._handle, C.byref(req), flag, cb, None, C.byref(out)))
        try:
            return self._read(out, request)
        finally:
            self._lib.hs_result_free(out)
            del keep

    def solve_coupled(self, request: BemRequest, network: Callable, stop: StopToken | None = None):
        """LEM-coupled solve in the library (hs_bem_solve_coupled; CudaBemSolver::solve
        with a coupling, cuda_solver.cu:1584-1667). request.excitations are the unit-flow
        port basis (coupling.make_coupling_basis); network(frequency, Z) returns the
        port flows and pressures (two sequences of complex, one per port). Returns the
        BemResult (one excitation per frequency: the coupled field, named "LEM") and per
        frequency (Z, flows, pressures)."""
        req, keep = self._c_request(request)
        out = C.c_void_p()
        failure = []

        def bridge(frequency, ports, z, q, p, _user):
            try:
                Z = np.ctypeslib.as_array(z, (2 * ports * ports,)).view(np.complex128).reshape(ports, ports)
                flows, pressures = network(frequency, Z.copy())
                flows, pressures = np.asarray(flows, np.complex128), np.asarray(pressures, np.complex128)
                if flows.shape != (ports,) or pressures.shape != (ports,):
                    raise ValueError("LEM result port count does not match its BEM basis.")
                np.ctypeslib.as_array(q, (2 * ports,))[:] = flows.view(np.float64)
                np.ctypeslib.as_array(p, (2 * ports,))[:] = pressures.view(np.float64)
                return _lib.HS_OK
            except Exception as e:  # reported after the call
                failure.append(e)
                return _lib.HS_E_INVALID
        cb = _lib.NETWORK_FN(bridge)
        flag = C.byref(stop._flag) if stop is not None else None
        status = self._lib.hs_bem_solve_coupled(self._handle, C.byref(req), cb, None, flag, C.byref(out))
        if failure:
            raise failure[0]
        _lib.check(status)
        try:
            coupled = dataclasses.replace(request, excitations=[BemExcitation("LEM", [])])
            result = self._read(out, coupled)
            ports = C.c_size_t()
            extra = []
            for f in range(len(result.frequencies)):
                _lib.check(self._lib.hs_result_coupling(out, f, None, None, None, C.byref(ports)))
                n = ports.value
                Z, q, pr = np.zeros(2 * n * n), np.zeros(2 * n), np.zeros(2 * n)
                _lib.check(self._lib.hs_result_coupling(out, f, Z.ctypes.data, q.ctypes.data, pr.ctypes.data,
                                                        C.byref(ports)))
                extra.append((_cplx(Z).reshape(n, n), _cplx(q), _cplx(pr)))
            return result, extra
        finally:
            self._lib.hs_result_free(out)
            del keep

    def pressure_field(self, frequency: float, solution: BemExcitationResult, points,
                       settings: PressureFieldSettings = PressureFieldSettings(),
                       medium: AcousticMedium = AcousticMedium()) -> list:
        """Pressure samples at world points from a solution's boundary traces:
        HornSculpt's evaluatePressureField (field_evaluation.hpp:29-33) for the
        exterior closed-surface form, on the GPU with this session's mesh. Points
        within minimum_boundary_distance of the surface are BOUNDARY, points
        inside the closed surface EXCLUDED, points whose adaptive quadrature does
        not converge within the depth QUADRATURE_NOT_CONVERGED (pressure 0)."""
        b = solution.boundary
        trace = np.ascontiguousarray(np.asarray(b.pressure_trace, np.complex128)).view(np.float64)
        deriv = np.ascontiguousarray(np.asarray(b.normal_derivative, np.complex128)).view(np.float64)
        pts = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 3))
        n = len(pts)
        out = np.zeros(2 * max(n, 1))
        status = np.zeros(max(n, 1), np.int32)
        st = _lib.hs_field_settings(settings.minimum_boundary_distance, settings.relative_quadrature_tolerance,
                                    settings.maximum_quadrature_depth)
        _lib.check(self._lib.hs_bem_pressure_field(self._handle, frequency, medium.sound_speed, trace.ctypes.data,
                                                   deriv.ctypes.data, pts.ctypes.data, n, C.byref(st),
                                                   out.ctypes.data, status.ctypes.data))
        return [PressureFieldSample(tuple(pts[i]), complex(out[2 * i], out[2 * i + 1]), FieldPointStatus(status[i]))
                for i in range(n)]

    # -- marshalling --------------------------------------------------------
    def _c_request(self, r: BemRequest):
        freqs = np.ascontiguousarray(r.frequencies, np.float64)
        plan = np.ascontiguousarray(r.interaction_plan_frequencies, np.float64)
        offsets = [0]
        face_ids, vel = [], []
        for ex in r.excitations:
            for fv in ex.faces:
                face_ids.append(fv.face_id)
                v = complex(fv.normal_velocity)
                vel += [v.real, v.imag]
            offsets.append(len(face_ids))
        offsets = np.asarray(offsets, np.uintp)
        face_ids = np.asarray(face_ids or [0], np.uint32)
        vel = np.asarray(vel or [0.0, 0.0], np.float64)
        obs = np.ascontiguousarray(np.asarray(r.observers, np.float64).reshape(-1, 3))
        c = _lib.hs_request()
        c.density = r.medium.density
        c.sound_speed = r.medium.sound_speed
        dp = C.POINTER(C.c_double)
        c.frequencies = freqs.ctypes.data_as(dp)
        c.frequency_count = len(freqs)
        c.plan_frequencies = plan.ctypes.data_as(dp) if len(plan) else None
        c.plan_frequency_count = len(plan)
        c.excitation_count = len(r.excitations)
        c.excitation_face_offsets = offsets.ctypes.data_as(C.POINTER(C.c_size_t))
        c.excitation_face_ids = face_ids.ctypes.data_as(C.POINTER(C.c_uint32))
        c.excitation_velocities = vel.ctypes.data_as(dp)
        c.observers = obs.ctypes.data_as(dp) if len(obs) else None
        c.observer_count = len(obs)
        if r.far_field is not None:
            c.far_field = 1
            for i in range(3):
                c.far_origin[i] = float(r.far_field.origin[i])
            c.far_reference_distance = r.far_field.reference_distance
        c.numerics = r.numerics.to_c()
        return c, (freqs, plan, offsets, face_ids, vel, obs)

    def _read(self, out, request: BemRequest) -> BemResult:
        lib = self._lib
        F = lib.hs_result_frequency_count(out)
        E = lib.hs_result_excitation_count(out)
        T = lib.hs_result_triangle_count(out)
        N = lib.hs_result_pressure_dof_count(out)
        O = lib.hs_result_observer_count(out)
        # one copy of the whole result; the per-frequency arrays are views of it
        traces = np.empty((F, E, N), np.complex128)
        surface = np.empty((F, E, T), np.complex128)
        normal = np.empty((F, E, T), np.complex128)
        observers = np.empty((F, E, O), np.complex128)
        xinfo = (_lib.hs_excitation_info * max(F * E, 1))()
        finfo = (_lib.hs_frequency_info * max(F, 1))()
        _lib.check(lib.hs_result_copy_all(out, traces.ctypes.data, surface.ctypes.data, normal.ctypes.data,
                                          observers.ctypes.data if O else None, xinfo, finfo))
        frames = []
        for f in range(F):
            fi = finfo[f]
            excs = []
            for e in range(E):
                info = xinfo[f * E + e]
                impedances = []
                if info.impedance_count:
                    imp = (_lib.hs_face_impedance * info.impedance_count)()
                    _lib.check(lib.hs_result_impedances(out, f, e, imp))
                    impedances = [FaceImpedance(x.face_id, x.area, complex(*x.mean_pressure),
                                                complex(*x.volume_velocity), complex(*x.volume_impedance)) for x in imp]
                excs.append(BemExcitationResult(
                    name=request.excitations[e].name, observer_pressure=observers[f, e], impedances=impedances,
                    refinement_steps=info.refinement_steps, iterations=info.iterations,
                    boundary_residual=info.boundary_residual,
                    field_quadrature_comparison_degree=info.field_comparison_degree,
                    field_quadrature_verification_degree=info.field_verification_degree,
                    field_quadrature_discrepancy=info.field_discrepancy,
                    boundary=BemBoundaryData(surface[f, e], traces[f, e], normal[f, e])))
            frames.append(BemFrequencyResult(fi.frequency, excs, fi.assembly_ms, fi.solve_ms, fi.factorization_ms,
                                             fi.triangular_solve_ms, fi.field_ms, fi.residual_check_ms,
                                             fi.interaction_plan_ms, bool(fi.interaction_plan_reused)))
        return BemResult(self.device_description(), T, N, lib.hs_result_peak_device_bytes(out), frames)

    # -- test hooks ---------------------------------------------------------
    def debug_assemble(self, numerics: BemNumerics, plan_k: float, k: float, flux: np.ndarray):
        """Row-equilibrated matrix (N x N, complex) and right-hand side for per-triangle flux."""
        N, T = self._mesh.vertex_count, self._mesh.triangle_count
        q = np.zeros(2 * T)
        q[0::2], q[1::2] = np.real(flux), np.imag(flux)
        A = np.zeros(2 * N * N)
        b = np.zeros(2 * N)
        n = numerics.to_c()
        _lib.check(self._lib.hs_bem_debug_assemble(self._handle, C.byref(n), plan_k, k, q.ctypes.data, A.ctypes.data,
                                                   b.ctypes.data))
        return _cplx(A).reshape(N, N).T, _cplx(b)  # column-major -> [row, col]

    def debug_fmm_far(self, numerics: BemNumerics, k: float, tolerance: float, pressure: np.ndarray):
        """Far part of the fast-multipole operator applied to a P1 vector (row-equilibrated
        like debug_assemble), the near support-pair pattern as CSR (row_start, cols) and
        the far-field levels as rows (level, order, nodes, M2L links, plane wave)."""
        N = self._mesh.vertex_count
        p = np.zeros(2 * N)
        p[0::2], p[1::2] = np.real(pressure), np.imag(pressure)
        far = np.zeros(2 * N)
        row = np.zeros(N + 1, np.uint32)
        count, levels = C.c_size_t(), C.c_size_t()
        n = numerics.to_c()
        _lib.check(self._lib.hs_bem_debug_fmm_far(self._handle, C.byref(n), k, tolerance, p.ctypes.data, far.ctypes.data,
                                                  row.ctypes.data, None, 0, C.byref(count), None, 0, C.byref(levels)))
        cols = np.zeros(max(count.value, 1), np.uint32)
        info = np.zeros((max(levels.value, 1), 5), np.uint32)
        _lib.check(self._lib.hs_bem_debug_fmm_far(self._handle, C.byref(n), k, tolerance, p.ctypes.data, far.ctypes.data,
                                                  row.ctypes.data, cols.ctypes.data, count.value, C.byref(count),
                                                  info.ctypes.data, levels.value, C.byref(levels)))
        return _cplx(far), row, cols[: count.value], info[: levels.value]


@dataclasses.dataclass
class ServeOptions:
    """hs_serve_options: the serving form's request loop."""
    workers: int = 4
    memory_fraction: float = 0.6
    resident_meshes: int = 8
    planning_frequency: float = 0.0   # Hz; > 0: every request plans at this frequency
    max_batch_frequencies: int = 32


@dataclasses.dataclass
class ServeTiming:
    queue_ms: float
    run_ms: float
    latency_ms: float
    footprint_bytes: int
    batched_requests: int


class BemServer:
    """Serving form: a persistent request loop on the current CUDA device.

    submit() copies a mesh and request and returns a ticket at once; the
    library admits requests in arrival order as device memory allows, runs up
    to `workers` at once on separate streams (requests on different meshes
    overlap on the GPU), keeps meshes resident for reuse and batches queued
    requests on the same mesh. wait(ticket) returns (BemResult, ServeTiming)."""

    _c_request = CudaBemSolver._c_request
    _read = CudaBemSolver._read
    device_description = staticmethod(CudaBemSolver.device_description)

    def __init__(self, options: ServeOptions = ServeOptions()):
        lib = _lib.load()
        o = _lib.hs_serve_options()
        lib.hs_serve_options_default(C.byref(o))
        for f in dataclasses.fields(options):
            setattr(o, f.name, getattr(options, f.name))
        handle = C.c_void_p()
        _lib.check(lib.hs_serve_create(C.byref(o), C.byref(handle)))
        self._handle, self._lib = handle, lib
        self._requests = {}

    def submit(self, mesh: SurfaceMesh, request: BemRequest) -> int:
        req, keep = self._c_request(request)
        ticket = C.c_uint64()
        _lib.check(self._lib.hs_serve_submit(self._handle, mesh.vertices.ctypes.data, mesh.vertex_count,
                                             mesh.triangles.ctypes.data, mesh.face_ids.ctypes.data,
                                             mesh.boundary.ctypes.data, mesh.triangle_count, C.byref(req),
                                             C.byref(ticket)))
        del keep
        self._requests[ticket.value] = request
        return ticket.value

    def wait(self, ticket: int):
        request = self._requests.pop(ticket, None)
        if request is None:
            raise ValueError("Unknown or already collected serving ticket.")
        out = C.c_void_p()
        t = _lib.hs_serve_timing()
        status = self._lib.hs_serve_wait(self._handle, ticket, C.byref(out), C.byref(t))
        _lib.check(status)
        try:
            result = self._read(out, request)
        finally:
            self._lib.hs_result_free(out)
        return result, ServeTiming(t.queue_ms, t.run_ms, t.latency_ms, t.footprint_bytes, t.batched_requests)

    def close(self):
        if getattr(self, "_handle", None):
            self._lib.hs_serve_destroy(self._handle)
            self._handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _plan_arrays(mesh: SurfaceMesh, sizes) -> dict:
    nt, nn, npch, nw, ntr, depth = list(sizes)
    return dict(touching=np.zeros((nt, 9), np.uint32), near=np.zeros((nn, 5), np.uint32),
                patches=np.zeros((npch, 22)), whole=np.zeros(nw, np.uint8),
                offsets=np.zeros(mesh.triangle_count + 1, np.uint32), trials=np.zeros(ntr, np.uint32), depth=depth)


def _plan_pointers(out: dict):
    return (out["touching"].ctypes.data, out["near"].ctypes.data, out["patches"].ctypes.data,
            out["whole"].ctypes.data, out["offsets"].ctypes.data, out["trials"].ctypes.data)


def host_plan(mesh: SurfaceMesh, numerics: BemNumerics, max_k: float) -> dict:
    """The library's host interaction plan of a mesh (no device needed)."""
    lib = _lib.load()
    n = numerics.to_c()
    sizes = (C.c_size_t * 6)()
    args = (mesh.vertices.ctypes.data, mesh.vertex_count, mesh.triangles.ctypes.data, mesh.triangle_count, C.byref(n),
            max_k, sizes)
    _lib.check(lib.hs_bem_debug_plan(*args, None, None, None, None, None, None))
    out = _plan_arrays(mesh, sizes)
    _lib.check(lib.hs_bem_debug_plan(*args, *_plan_pointers(out)))
    return out


PLAN_STATS = ("device_pairs", "projected_pairs", "flagged_pairs", "whole_panel_pairs", "device_ms", "host_ms",
              "resolved_pairs", "frame_ms", "classify_ms", "refine_ms", "readback_ms", "host_part_ms",
              "host_runs_ms", "host_pairs_ms", "host_flatten_ms", "host_fill_ms", "host_csr_ms", "samples",
              "refine_kernel_ms", "root_settled_pairs")


def device_plan(mesh: SurfaceMesh, numerics: BemNumerics, max_k: float, emulate: bool = False) -> dict:
    """The interaction plan from the device planner (on the current CUDA
    device, or with emulate=True its algorithm run on the host), with its
    statistics under "stats". The plan is computed once and read out once;
    it equals host_plan's bit for bit."""
    lib = _lib.load()
    n = numerics.to_c()
    sizes = (C.c_size_t * 6)()
    stats = (C.c_double * 20)()
    args = (mesh.vertices.ctypes.data, mesh.vertex_count, mesh.triangles.ctypes.data, mesh.triangle_count, C.byref(n),
            max_k, 1 if emulate else 0, stats, sizes)
    _lib.check(lib.hs_bem_debug_plan_device(*args, None, None, None, None, None, None))
    out = _plan_arrays(mesh, sizes)
    _lib.check(lib.hs_bem_debug_plan_device(*args, *_plan_pointers(out)))
    out["stats"] = dict(zip(PLAN_STATS, list(stats)))
    return out


def debug_lu_factor(matrices: np.ndarray, fp32: bool = False):
    """The solver's batched LU of complex matrices (batch x n x n, [row, col]).

    Returns (factors, pivots, info): factors batch x n x n complex holding unit
    L below the diagonal and U on and above it (LAPACK zgetrf layout), pivots
    batch x n 0-based row interchanges, info the batch's breakdown word.
    fp32 selects the mixed form's FP32 factorisation (input rounded to FP32,
    tensor-core trailing updates)."""
    lib = _lib.load()
    a = np.asarray(matrices, np.complex128)
    if a.ndim == 2:
        a = a[None]
    batch, n, m = a.shape
    if n != m:
        raise ValueError("debug_lu_factor needs square matrices")
    cm = np.ascontiguousarray(np.transpose(a, (0, 2, 1)))  # column-major per matrix
    src = np.ascontiguousarray(np.stack([cm.real, cm.imag], -1))
    out = np.zeros_like(src)
    piv = np.zeros((batch, n), np.int32)
    info = C.c_int32()
    _lib.check(lib.hs_bem_debug_lu(1 if fp32 else 0, n, batch, src.ctypes.data, out.ctypes.data, piv.ctypes.data,
                                   C.byref(info)))
    factors = np.transpose(out[..., 0] + 1j * out[..., 1], (0, 2, 1))
    return factors, piv, info.value


def autotune_report() -> dict:
    """{size class: (chosen candidate, [ms per candidate])} of the launch-shape autotuner."""
    lib = _lib.load()
    need = C.c_size_t()
    _lib.check(lib.hs_autotune_report(None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    _lib.check(lib.hs_autotune_report(buf, need.value, C.byref(need)))
    out = {}
    for item in buf.value.decode().split(";"):
        if item:
            key, rest = item.split("=")
            choice, ms = rest.split(":")
            out[key] = (int(choice), [float(x) for x in ms.split("/") if x])
    return out


def autotune_enable(enabled: bool = True) -> None:
    _lib.check(_lib.load().hs_autotune_set_enabled(int(enabled)))


def autotune_clear() -> None:
    _lib.check(_lib.load().hs_autotune_clear())
