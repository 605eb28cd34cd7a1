"""Captured CUDA graphs: a session replays the dense batch chain (assembly,
LU, initial solves) and the fast-multipole far-field apply as graphs. A
replayed solve must equal the same solve run as plain launches, bit for bit,
and the replays must actually happen."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

pytestmark = pytest.mark.gpu


def _request(numerics, freqs=(300.0, 900.0, 2100.0)):
    return hs.BemRequest(frequencies=list(freqs), observers=[(0, 0, 0.4), (0.5, 0.1, 0.0)],
                         excitations=[hs.BemExcitation("unit", [hs.FaceVelocity(1, 1.0)])], numerics=numerics)


def _same(a, b):
    for fa, fb in zip(a.frequencies, b.frequencies):
        ea, eb = fa.excitations[0], fb.excitations[0]
        assert np.array_equal(ea.boundary.pressure_trace, eb.boundary.pressure_trace)
        assert np.array_equal(ea.observer_pressure, eb.observer_pressure)
        assert ea.boundary_residual == eb.boundary_residual


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_chain_graph_replay_equals_launches(precision):
    mesh = meshes.octahedral_sphere(3)
    numerics = hs.BemNumerics(precision=precision)
    with hs.CudaBemSolver(mesh) as solver:
        solver.set_graphs(False)
        plain = solver.solve(_request(numerics))
    with hs.CudaBemSolver(mesh) as solver:
        first = solver.solve(_request(numerics))     # plain launches (first use of the batch shape)
        second = solver.solve(_request(numerics))    # captured, then replayed
        third = solver.solve(_request(numerics))     # replayed
        assert solver.graph_launches() == 2
        # a different batch shape gets its own graph; the first use runs as launches
        other = solver.solve(_request(numerics, (500.0,)))
        assert solver.graph_launches() == 2
    for r in (first, second, third):
        _same(plain, r)
    assert other.frequencies[0].excitations[0].boundary_residual < 1e-9


def test_fast_multipole_graph_replay_equals_launches():
    mesh = meshes.icosphere(3)
    numerics = hs.BemNumerics(precision="fp64", acceleration="fast_multipole", relative_residual_tolerance=1e-7)
    with hs.CudaBemSolver(mesh) as solver:
        solver.set_graphs(False)
        plain = solver.solve(_request(numerics, (1500.0,)))
    with hs.CudaBemSolver(mesh) as solver:
        replayed = solver.solve(_request(numerics, (1500.0,)))
    _same(plain, replayed)


def test_autotuned_launch_shapes_keep_results():
    """The regular-pair kernels' grid shape is tuned on first use per size class;
    a tuned solve equals an untuned one bit for bit, and the tuned classes are
    reported with one time per candidate."""
    mesh = meshes.icosphere(3)
    for precision in ("fp64", "mixed"):
        numerics = hs.BemNumerics(precision=precision)
        hs.autotune_clear()
        hs.autotune_enable(False)
        with hs.CudaBemSolver(mesh) as solver:
            untuned = solver.solve(_request(numerics))
        hs.autotune_enable(True)
        with hs.CudaBemSolver(mesh) as solver:
            tuned = solver.solve(_request(numerics))   # tunes while it solves
            again = solver.solve(_request(numerics))   # uses the choices
        _same(untuned, tuned)
        _same(untuned, again)
        report = hs.autotune_report()
        prefix = "regular_mixed" if precision == "mixed" else "regular_fp64"
        classes = [k for k in report if k.startswith(prefix)]
        assert classes, report
        for k in classes:
            choice, ms = report[k]
            assert 0 <= choice < len(ms) and all(t > 0 for t in ms)


def test_autotuned_fast_multipole_leaf_size():
    """Leaf capacity 0 asks the autotuner: the solve meets its tolerance against
    the dense solve and the chosen leaf class is reported."""
    mesh = meshes.icosphere(3)
    auto = hs.BemNumerics(precision="fp64", acceleration="fast_multipole", relative_residual_tolerance=1e-7,
                          fast_multipole=hs.FastMultipoleSettings(leaf_support_capacity=0))
    dense = hs.BemNumerics(precision="fp64", relative_residual_tolerance=1e-7)
    with hs.CudaBemSolver(mesh) as solver:
        a = solver.solve(_request(auto, (1500.0,)))
        d = solver.solve(_request(dense, (1500.0,)))
    ta, td = a.frequencies[0].excitations[0], d.frequencies[0].excitations[0]
    assert ta.boundary_residual <= 1e-7
    assert np.linalg.norm(ta.boundary.pressure_trace - td.boundary.pressure_trace) < 1e-5 * np.linalg.norm(
        td.boundary.pressure_trace)
    leaf = [k for k in hs.autotune_report() if k.startswith("fmm_leaf")]
    assert leaf
