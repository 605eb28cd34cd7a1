"""Serving form (hs_serve_*): persistent request loop with admission by
device footprint, concurrent requests on separate streams, resident meshes
and same-mesh batching. The contract tested here: a result is the same
alone and in the mix (bit for bit, since every request on a mesh plans at the
server's planning frequency and every per-frequency computation is
independent of its batch), queued compatible requests on one mesh are solved
together, and bad requests fail at submit."""
import numpy as np
import pytest

import hornsculpt_b200 as hs
from hornsculpt_b200 import meshes

pytestmark = pytest.mark.gpu

PLAN_HZ = 2000.0


def _request(freqs, precision="mixed", face=1, obs=((0, 0, 0.4), (0.3, 0.2, 0.1))):
    return hs.BemRequest(frequencies=list(freqs), observers=list(obs),
                         excitations=[hs.BemExcitation("drive", [hs.FaceVelocity(face, 1.0)])],
                         numerics=hs.BemNumerics(precision=precision))


def _same(a, b):
    assert [f.frequency for f in a.frequencies] == [f.frequency for f in b.frequencies]
    for fa, fb in zip(a.frequencies, b.frequencies):
        for ea, eb in zip(fa.excitations, fb.excitations):
            assert np.array_equal(ea.boundary.pressure_trace, eb.boundary.pressure_trace)
            assert np.array_equal(ea.observer_pressure, eb.observer_pressure)
            assert ea.boundary_residual == eb.boundary_residual


def test_result_is_the_same_alone_and_in_the_mix():
    sphere = meshes.octahedral_sphere(3)
    horn = meshes.exponential_horn(h=0.0128, seed=5)
    small = meshes.icosphere(2)
    target = (sphere, _request([300.0, 900.0]))
    others = [(horn, _request([400.0, 1500.0], face=meshes.HORN_THROAT, obs=((0, 0, 0.6),))),
              (small, _request([700.0], precision="fp64")),
              (sphere, _request([600.0, 1100.0], precision="fp64")),
              (horn, _request([250.0], face=meshes.HORN_THROAT, obs=((0, 0, 0.6),)))]
    options = hs.ServeOptions(workers=1, planning_frequency=PLAN_HZ)
    with hs.BemServer(options) as server:
        alone, t_alone = server.wait(server.submit(*target))
    options = hs.ServeOptions(workers=4, planning_frequency=PLAN_HZ)
    with hs.BemServer(options) as server:
        tickets = [server.submit(*others[0]), server.submit(*target)] + [server.submit(*o) for o in others[1:]]
        results = [server.wait(t) for t in tickets]
    _same(alone, results[1][0])
    assert t_alone.latency_ms >= t_alone.run_ms > 0
    # a direct session solve with the same planning raster gives the same result
    req = target[1]
    req.interaction_plan_frequencies = sorted(set(req.frequencies) | {PLAN_HZ})
    with hs.CudaBemSolver(sphere) as solver:
        _same(alone, solver.solve(req))
    for (mesh, request), (result, timing) in zip([others[0], target] + others[1:], results):
        assert len(result.frequencies) == len(request.frequencies)
        assert all(e.boundary_residual <= (1e-10 if request.numerics.precision == "mixed" else 5e-5)
                   for f in result.frequencies for e in f.excitations)
        assert timing.footprint_bytes > 0 and timing.latency_ms >= timing.run_ms


def test_queued_requests_on_one_mesh_are_batched():
    """With one worker busy on another mesh, two compatible requests on the
    same mesh queue up and are solved in one session call; their results equal
    the ones they get alone."""
    sphere = meshes.octahedral_sphere(3)
    blocker = (meshes.icosphere(3), _request([500.0 + 100.0 * i for i in range(12)], precision="fp64"))
    a, b = _request([300.0, 900.0]), _request([600.0, 900.0])
    options = hs.ServeOptions(workers=1, planning_frequency=PLAN_HZ)
    with hs.BemServer(options) as server:
        tb = server.submit(*blocker)
        ta, tb2 = server.submit(sphere, a), server.submit(sphere, b)
        server.wait(tb)
        (ra, ia), (rb, ib) = server.wait(ta), server.wait(tb2)
        assert ia.batched_requests == 2 and ib.batched_requests == 2
        alone_a, _ = server.wait(server.submit(sphere, a))
    _same(ra, alone_a)
    assert [f.frequency for f in rb.frequencies] == [600.0, 900.0]
    # the shared frequency comes from the same solve
    assert np.array_equal(ra.frequencies[1].excitations[0].boundary.pressure_trace,
                          rb.frequencies[1].excitations[0].boundary.pressure_trace)


def test_bad_requests_fail_at_submit():
    sphere = meshes.octahedral_sphere(2)
    with hs.BemServer(hs.ServeOptions(workers=2, planning_frequency=PLAN_HZ)) as server:
        with pytest.raises(ValueError, match="planning frequency"):
            server.submit(sphere, _request([2500.0]))
        flipped = meshes.SurfaceMesh(sphere.vertices, sphere.triangles[:, ::-1], sphere.face_ids, sphere.boundary)
        with pytest.raises(ValueError, match="outward winding"):
            server.submit(flipped, _request([500.0]))
        with pytest.raises(ValueError, match="ticket"):
            server.wait(12345)
    with pytest.raises(ValueError, match="serving options"):
        hs.BemServer(hs.ServeOptions(workers=0))


def test_reference_fixture_request_is_served():
    """A request in the reference's fixture JSON (hornsculpt-solver-input-1) read back
    and served gives the result of the request it was written from, bit for bit."""
    import json
    sphere = meshes.octahedral_sphere(3)
    request = _request([500.0, 1200.0])
    mesh2, request2, _ = hs.read_fixture(json.dumps(hs.write_fixture(sphere, request, "sphere")).encode())
    request2.numerics = hs.BemNumerics(precision="mixed")
    with hs.BemServer(hs.ServeOptions(workers=2, planning_frequency=PLAN_HZ)) as server:
        direct = server.wait(server.submit(sphere, request))[0]
        replayed = server.wait(server.submit(mesh2, request2))[0]
    _same(direct, replayed)


def test_fast_multipole_request_is_served():
    """A fast-multipole (FP64) request through the serving loop: admitted by its sparse
    footprint and equal to the direct session solve within the solver tolerance."""
    horn = meshes.exponential_horn(h=0.0128, seed=5)
    request = hs.BemRequest(frequencies=[900.0], observers=[(0, 0, 0.6)],
                            excitations=[hs.BemExcitation("drive", [hs.FaceVelocity(meshes.HORN_THROAT, 1.0)])],
                            numerics=hs.BemNumerics(precision="fp64", acceleration="fast_multipole",
                                                    relative_residual_tolerance=1e-6))
    with hs.BemServer(hs.ServeOptions(workers=1, planning_frequency=PLAN_HZ)) as server:
        served, timing = server.wait(server.submit(horn, request))
    request.interaction_plan_frequencies = sorted(set(request.frequencies) | {PLAN_HZ})
    with hs.CudaBemSolver(horn) as solver:
        direct = solver.solve(request)
    a = served.frequencies[0].excitations[0].boundary.pressure_trace
    b = direct.frequencies[0].excitations[0].boundary.pressure_trace
    assert np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(b)
    assert served.frequencies[0].excitations[0].iterations > 0 and timing.footprint_bytes > 0


def test_continuous_batching_joins_a_running_call():
    """A request that arrives while another request on the same mesh is being
    solved joins the running call at its next frequency batch (ahead of the
    call's remaining frequencies) and is completed as soon as its own
    frequencies are solved, well before the long call ends. Its result equals
    its solve alone, bit for bit."""
    import time
    sphere = meshes.octahedral_sphere(4)
    long_freqs = [float(f) for f in np.geomspace(150.0, 1900.0, 24)]
    late = _request([333.0, 1234.0])
    with hs.BemServer(hs.ServeOptions(workers=1, planning_frequency=PLAN_HZ)) as server:
        alone, _ = server.wait(server.submit(sphere, late))
    # one frequency per batch: the long call is 24 batches, the late request joins the next one
    options = hs.ServeOptions(workers=1, planning_frequency=PLAN_HZ, max_batch_frequencies=1)
    with hs.BemServer(options) as server:
        server.wait(server.submit(sphere, _request([500.0])))  # mesh resident and planned
        t_long = time.perf_counter()
        long_ticket = server.submit(sphere, _request(long_freqs))
        time.sleep(0.02)
        t_late = time.perf_counter()
        late_ticket = server.submit(sphere, late)
        late_result, late_timing = server.wait(late_ticket)
        long_result, long_timing = server.wait(long_ticket)
    _same(alone, late_result)
    assert late_timing.batched_requests >= 2 and long_timing.batched_requests >= 2
    late_finish = t_late + late_timing.latency_ms / 1e3
    long_finish = t_long + long_timing.latency_ms / 1e3
    assert late_finish < long_finish - 0.25 * long_timing.run_ms / 1e3
    assert [f.frequency for f in long_result.frequencies] == long_freqs
