"""Test infrastructure only: ctypes access to the FP64 CPU oracle
(``oracle/liboracle.so``) and to HornSculpt's own galerkin CPU code compiled
into ``oracle/_ref/libhsref.so``. Imported by tests/, the smoke check and
bench.py's CPU-baseline leg; never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
_P = C.c_void_p
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
_szp = np.ctypeslib.ndpointer(np.uintp, flags="C")


class Numerics(C.Structure):
    """Mirrors ``BemNumerics`` (``modules/bem/include/hornsculpt/bem.hpp:113-123``)."""

    _fields_ = [("quadrature_order", C.c_uint), ("singular_order", C.c_uint), ("near_ratio", C.c_double),
                ("near_tol", C.c_double), ("near_depth", C.c_uint), ("residual_tol", C.c_double),
                ("max_refine", C.c_uint)]

    @classmethod
    def default(cls, **kw):
        n = cls(4, 4, 1.0, 1e-4, 6, 5e-5, 3)
        for k, v in kw.items():
            setattr(n, k, v)
        return n


def build(reference: str | None = None) -> None:
    env = dict(os.environ)
    cmd = ["make", "-s", "-C", str(HERE)]
    if reference:
        cmd.append(f"REFERENCE={reference}")
    subprocess.run(cmd, check=True, env=env)


_oracle = None
_ref = None


def _load_oracle():
    global _oracle
    if _oracle is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        lib = C.CDLL(str(path))
        lib.oracle_last_error.restype = C.c_char_p
        lib.oracle_plan_build.argtypes = [_f64p, C.c_size_t, _u32p, C.c_size_t, C.POINTER(Numerics), C.c_double,
                                          C.POINTER(_P)]
        lib.oracle_assemble.argtypes = [_f64p, C.c_size_t, _u32p, C.c_size_t, C.POINTER(Numerics), C.c_double,
                                        C.c_double, _f64p, _f64p, _f64p]
        lib.oracle_solve.argtypes = [_f64p, C.c_size_t, _u32p, _u32p, _u8p, C.c_size_t, C.c_double, C.c_double,
                                     _f64p, C.c_size_t, C.c_double, C.c_size_t, _szp, _u32p, _f64p, _f64p,
                                     C.c_size_t, C.c_int, _f64p, C.c_double, C.POINTER(Numerics), _f64p, _f64p,
                                     _f64p, _f64p, _u32p, _f64p, _u32p]
        lib.oracle_laplace_pair.argtypes = [_f64p, _u32p, _f64p, _u32p, C.c_uint, C.POINTER(C.c_double)]
        lib.oracle_estimate_patch.argtypes = [_f64p, _f64p, _u32p, _u32p, _f64p, C.c_double, _f64p, _f64p]
        _oracle = lib
    return _oracle


def use_lapack(enabled: bool = True) -> str:
    """Makes ``solve`` factor with LAPACK zgetrf / zgetrs (scipy's OpenBLAS,
    through the function pointers scipy.linalg.cython_lapack exports) instead
    of the built-in textbook LU; returns the provider's description."""
    lib = _load_oracle()
    lib.oracle_set_lapack.argtypes = [_P, _P]
    if not enabled:
        lib.oracle_set_lapack(None, None)
        return "textbook LU"
    import scipy
    import scipy.linalg.cython_lapack as cl
    get = C.pythonapi.PyCapsule_GetPointer
    get.restype = _P
    get.argtypes = [C.py_object, C.c_char_p]
    name = C.pythonapi.PyCapsule_GetName
    name.restype = C.c_char_p
    name.argtypes = [C.py_object]
    fns = [get(cl.__pyx_capi__[f], name(cl.__pyx_capi__[f])) for f in ("zgetrf", "zgetrs")]
    lib.oracle_set_lapack(*fns)
    return f"LAPACK zgetrf/zgetrs from scipy {scipy.__version__} (OpenBLAS)"


def reference_available() -> bool:
    return (HERE / "_ref" / "libhsref.so").exists()


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(str(HERE / "_ref" / "libhsref.so"))
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_plan_build.argtypes = [_f64p, C.c_size_t, _u32p, C.c_size_t, C.POINTER(Numerics), C.c_double,
                                       C.c_uint, C.POINTER(_P)]
        lib.ref_estimate_patch.argtypes = [_f64p, _f64p, _u32p, _u32p, _f64p, C.c_double, _f64p, _f64p]
        lib.ref_triangle_rule.argtypes = [C.c_uint, _P, C.POINTER(C.c_size_t)]
        lib.ref_gauss.argtypes = [C.c_uint, _f64p]
        lib.ref_pressure_field.argtypes = [_f64p, C.c_size_t, _u32p, C.c_size_t, _f64p, _f64p, C.c_double,
                                           C.c_double, _f64p, C.c_size_t, C.c_double, C.c_double, C.c_uint, _f64p,
                                           np.ctypeslib.ndpointer(np.int32, flags="C")]
        _ref = lib
    return _ref


class OracleError(RuntimeError):
    pass


def _check(lib, prefix, code):
    if code:
        msg = getattr(lib, f"{prefix}_last_error")().decode()
        raise (ValueError if code == 1 else OracleError)(msg)


def _plan_arrays(lib, prefix, handle):
    sizes = (C.c_size_t * 6)()
    getattr(lib, f"{prefix}_plan_sizes")(handle, sizes)
    nt, nn, npch, nw, ntr, depth = list(sizes)
    touching = np.zeros((nt, 9), np.uint32)
    near = np.zeros((nn, 5), np.uint32)
    patches = np.zeros((npch, 22), np.float64)
    whole = np.zeros(nw, np.uint8)
    trials = np.zeros(ntr, np.uint32)
    getattr(lib, f"{prefix}_plan_touching")(handle, touching.ctypes.data_as(_P))
    getattr(lib, f"{prefix}_plan_near")(handle, near.ctypes.data_as(_P))
    getattr(lib, f"{prefix}_plan_patches")(handle, patches.ctypes.data_as(_P))
    getattr(lib, f"{prefix}_plan_whole")(handle, whole.ctypes.data_as(_P))
    return dict(touching=touching, near=near, patches=patches, whole=whole, trials=trials, depth=depth)


def _finish_plan(lib, prefix, handle, T):
    out = _plan_arrays(lib, prefix, handle)
    offsets = np.zeros(T + 1, np.uint32)
    getattr(lib, f"{prefix}_plan_offsets")(handle, offsets.ctypes.data_as(_P), out["trials"].ctypes.data_as(_P))
    out["offsets"] = offsets
    getattr(lib, f"{prefix}_plan_free")(handle)
    return out


def oracle_plan(mesh, numerics: Numerics, max_k: float) -> dict:
    lib = _load_oracle()
    h = _P()
    _check(lib, "oracle", lib.oracle_plan_build(mesh.vertices.ravel(), mesh.vertex_count, mesh.triangles.ravel(),
                                                 mesh.triangle_count, C.byref(numerics), max_k, C.byref(h)))
    return _finish_plan(lib, "oracle", h, mesh.triangle_count)


def reference_plan(mesh, numerics: Numerics, max_k: float, threads: int = 0) -> dict:
    lib = _load_ref()
    h = _P()
    _check(lib, "ref", lib.ref_plan_build(mesh.vertices.ravel(), mesh.vertex_count, mesh.triangles.ravel(),
                                           mesh.triangle_count, C.byref(numerics), max_k, threads, C.byref(h)))
    return _finish_plan(lib, "ref", h, mesh.triangle_count)


def reference_triangle_rule(degree: int) -> np.ndarray:
    lib = _load_ref()
    n = C.c_size_t()
    _check(lib, "ref", lib.ref_triangle_rule(degree, None, C.byref(n)))
    out = np.zeros((n.value, 4))
    _check(lib, "ref", lib.ref_triangle_rule(degree, out.ctypes.data_as(_P), C.byref(n)))
    return out


def reference_gauss(order: int) -> np.ndarray:
    lib = _load_ref()
    out = np.zeros((order, 2))
    _check(lib, "ref", lib.ref_gauss(order, out.ravel()))
    return out


def reference_pressure_field(mesh, frequency: float, sound_speed: float, pressure_trace, normal_derivative, points,
                             minimum_boundary_distance: float = 1e-4, tolerance: float = 1e-4, depth: int = 8):
    """HornSculpt's own evaluatePressureField (field_evaluation.cpp:330-463) on
    the exterior mesh: (pressures complex [P], statuses int [P])."""
    lib = _load_ref()
    verts = np.ascontiguousarray(mesh.vertices, np.float64).ravel()
    tris = np.ascontiguousarray(mesh.triangles, np.uint32).ravel()
    trace = np.ascontiguousarray(np.asarray(pressure_trace, np.complex128)).view(np.float64)
    deriv = np.ascontiguousarray(np.asarray(normal_derivative, np.complex128)).view(np.float64)
    pts = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 3))
    out = np.zeros(2 * len(pts))
    status = np.zeros(len(pts), np.int32)
    _check(lib, "ref", lib.ref_pressure_field(verts, mesh.vertex_count, tris, mesh.triangle_count, trace, deriv,
                                              frequency, sound_speed, pts.ravel(), len(pts),
                                              minimum_boundary_distance, tolerance, depth, out, status))
    return out.view(np.complex128), status


def reference_support_tree(mesh, leaf_capacity=32, separation_ratio=1.5, near_distance_ratio=2.0):
    """The reference's makeSupportTree (fmm/support_tree.cpp:407) on the mesh centred
    on vertex 0: (sizes[6], links (M, 2)) with sizes = nodes, levels, pp near, pp far,
    pf near, pf far and links the four lists' (target, source) pairs in that order."""
    lib = _load_ref()
    sizes = np.zeros(6, np.uintp)
    verts = np.ascontiguousarray(mesh.vertices, np.float64)
    tris = np.ascontiguousarray(mesh.triangles, np.uint32)
    lib.ref_support_tree.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_uint, C.c_double, C.c_double,
                                     C.c_void_p, C.c_void_p, C.c_size_t]
    _check(lib, "ref", lib.ref_support_tree(verts.ctypes.data, mesh.vertex_count, tris.ctypes.data,
                                            mesh.triangle_count, leaf_capacity, separation_ratio, near_distance_ratio,
                                            sizes.ctypes.data, None, 0))
    total = int(sizes[2:].sum())
    links = np.zeros((max(total, 1), 2), np.uint32)
    _check(lib, "ref", lib.ref_support_tree(verts.ctypes.data, mesh.vertex_count, tris.ctypes.data,
                                            mesh.triangle_count, leaf_capacity, separation_ratio, near_distance_ratio,
                                            sizes.ctypes.data, links.ctypes.data, total))
    return sizes.astype(np.int64), links[:total]


def estimate_patch(which: str, tri_a, tri_b, nodes_a, nodes_b, patch22, k):
    lib = _load_oracle() if which == "oracle" else _load_ref()
    prefix = "oracle" if which == "oracle" else "ref"
    mom = np.zeros(72)
    err = np.zeros(3)
    fn = getattr(lib, f"{prefix}_estimate_patch")
    _check(lib, prefix, fn(np.ascontiguousarray(tri_a, np.float64).ravel(), np.ascontiguousarray(tri_b, np.float64).ravel(),
                           np.ascontiguousarray(nodes_a, np.uint32), np.ascontiguousarray(nodes_b, np.uint32),
                           np.ascontiguousarray(patch22, np.float64), k, mom, err))
    return mom[0::2] + 1j * mom[1::2], err


def laplace_pair(tri_a, nodes_a, tri_b, nodes_b, order: int) -> float:
    lib = _load_oracle()
    v = C.c_double()
    _check(lib, "oracle", lib.oracle_laplace_pair(np.ascontiguousarray(tri_a, np.float64).ravel(),
                                                  np.ascontiguousarray(nodes_a, np.uint32),
                                                  np.ascontiguousarray(tri_b, np.float64).ravel(),
                                                  np.ascontiguousarray(nodes_b, np.uint32), order, C.byref(v)))
    return v.value


def assemble(mesh, numerics: Numerics, plan_k: float, k: float, q: np.ndarray):
    """Row-equilibrated dense system (A row-major, rhs) for one excitation."""
    lib = _load_oracle()
    N, T = mesh.vertex_count, mesh.triangle_count
    A = np.zeros(2 * N * N)
    rhs = np.zeros(2 * N)
    qq = np.zeros(2 * T)
    qq[0::2] = np.real(q)
    qq[1::2] = np.imag(q)
    _check(lib, "oracle", lib.oracle_assemble(mesh.vertices.ravel(), N, mesh.triangles.ravel(), T, C.byref(numerics),
                                              plan_k, k, qq, A, rhs))
    return (A[0::2] + 1j * A[1::2]).reshape(N, N), rhs[0::2] + 1j * rhs[1::2]


def solve(mesh, frequencies, excitations, observers=(), *, density=1.21, sound_speed=343.0, numerics=None,
          plan_frequencies=(), far_field=None):
    """Full dense FP64 solve. excitations: list of lists of (face_id, complex velocity).
    far_field: None or (origin xyz, reference distance). Returns a dict of arrays."""
    lib = _load_oracle()
    numerics = numerics or Numerics.default()
    N, T = mesh.vertex_count, mesh.triangle_count
    F, E = len(frequencies), len(excitations)
    obs = np.ascontiguousarray(np.asarray(observers, np.float64).reshape(-1, 3))
    O = len(obs)
    offsets = np.zeros(E + 1, np.uintp)
    faces, vel = [], []
    for e, ex in enumerate(excitations):
        for fid, v in ex:
            faces.append(fid)
            vel += [complex(v).real, complex(v).imag]
        offsets[e + 1] = len(faces)
    faces = np.array(faces or [0], np.uint32)
    vel = np.array(vel or [0.0, 0.0])
    plan_f = max(plan_frequencies) if len(plan_frequencies) else 0.0
    trace = np.zeros(2 * F * E * N)
    surface = np.zeros(2 * F * E * T)
    observed = np.zeros(max(1, 2 * F * E * O))
    residual = np.zeros(F * E)
    degrees = np.zeros(max(1, 2 * F * E), np.uint32)
    disc = np.zeros(max(1, F * E))
    refine = np.zeros(F, np.uint32)
    fo = np.zeros(3)
    fd = 1.0
    if far_field is not None:
        fo = np.asarray(far_field[0], np.float64)
        fd = float(far_field[1])
    _check(lib, "oracle", lib.oracle_solve(mesh.vertices.ravel(), N, mesh.triangles.ravel(), mesh.face_ids,
                                           mesh.boundary, T, density, sound_speed,
                                           np.ascontiguousarray(frequencies, np.float64), F, plan_f, E, offsets, faces,
                                           vel, obs.ravel() if O else np.zeros(3), O, int(far_field is not None), fo,
                                           fd, C.byref(numerics), trace, surface, observed, residual, degrees, disc,
                                           refine))
    c = lambda a, *shape: (a[0::2] + 1j * a[1::2]).reshape(*shape)
    return dict(trace=c(trace, F, E, N), surface=c(surface, F, E, T),
                observer=c(observed[: 2 * F * E * O], F, E, O), residual=residual.reshape(F, E),
                field_degrees=degrees[: 2 * F * E].reshape(F, E, 2), field_discrepancy=disc[: F * E].reshape(F, E),
                refinements=refine)
