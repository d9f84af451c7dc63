"""The serving loop on the device with a mixed stream: static elastic solves (BatchEngine slots)
and J2 load paths (J2Lane cohorts) at once. Each J2 result is bit for bit the load path alone
(serving.solve_j2_alone: plain Newton with Jacobi-PCG on an InternalForce of that mesh), and
each static solution bit for bit the same request served alone."""
import numpy as np
import pytest
import torch

import femorax_b200 as fx
from femorax_b200 import serving

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
RTOL = 1e-8


def engine():
    return fx.BatchEngine(1 << 22, 8, options=fx.SolveOptions(relative_tolerance=RTOL))


STREAM = [serving.Request(0, 6, 5, 9, E=70e6, nu=0.3),
          serving.J2Request(1, 1, 1, 24, E=60e6, sigma_y=80e3, total=0.0, steps_per_cycle=4),
          serving.Request(2, 4, 4, 12, E=120e6, nu=0.35),
          serving.J2Request(3, 2, 2, 30, E=90e6, sigma_y=150e3, total=0.0, steps_per_cycle=4),
          serving.J2Request(4, 1, 1, 21, E=45e6, sigma_y=60e3, total=0.0, steps_per_cycle=4),
          serving.Request(5, 7, 3, 5, E=50e6, nu=0.25)]


def with_loads(stream):
    """J2 loads at 1.2 times the force that first yields the base in elastic bending."""
    out = []
    for r in stream:
        if isinstance(r, serving.J2Request):
            b, L = r.nx * r.h, r.nz * r.h
            r = serving.J2Request(r.id, r.nx, r.ny, r.nz, r.E, r.sigma_y, 1.2 * r.sigma_y * b ** 3 / (6.0 * L), r.h,
                                  r.cycles, r.steps_per_cycle, arrival=0.001 * r.id)
        else:
            r = serving.Request(r.id, r.nx, r.ny, r.nz, r.E, r.nu, r.q, r.h, arrival=0.001 * r.id)
        out.append(r)
    return out


def test_mixed_stream_same_alone_and_in_the_mix():
    stream = with_loads(STREAM)
    srv = serving.Server(engine(), hbm_budget=1 << 34, max_cohort=2)
    served, wall = srv.run(stream, realtime=False)
    assert sorted(s.id for s in served) == [r.id for r in stream]
    by_id = {s.id: s for s in served}
    for r in stream:
        s = by_id[r.id]
        assert s.result.converged, r.id
        if isinstance(r, serving.J2Request):
            mesh, f, mon, n = serving.prepare_j2(r)
            force = fx.InternalForce(mesh)
            u, res = serving.solve_j2_alone(r, force, torch.as_tensor(f, device=DEV), mon)
            assert np.array_equal(s.x, u), r.id
            assert np.array_equal(s.result.monitor, res.monitor), r.id
            assert np.array_equal(s.result.newton, res.newton), r.id
        else:
            alone, _ = serving.Server(engine(), hbm_budget=1 << 34).run([r], realtime=False)
            assert np.array_equal(s.x, alone[0].x), r.id
    assert srv.resident == 0
    summ = serving.summary(served, wall)
    assert summ["converged"] == len(stream)


def test_admission_budget_from_free_device_memory():
    """Without a given budget the loop sizes admissions against the device's free memory
    (fx_device_memory, cudaMemGetInfo) less its reserve."""
    free0, total = fx.device_memory(0)
    assert 0 < free0 <= total
    srv = serving.Server(engine(), reserve=1 << 30)
    assert 0 < srv.budget <= total - (1 << 30)
    assert abs(srv.budget - (free0 - (1 << 30))) <= total // 10


def test_native_server_same_alone_and_in_the_mix():
    """The loop in C++ (fx_server_*, serving.NativeServer) on the same mixed stream: every J2 result
    bit for bit the load path alone, every static solution bit for bit the Python loop's (the same
    engine arithmetic), two requests on one shared InternalForce included."""
    stream = with_loads(STREAM)
    prep = {r.id: serving.prepare_any(r) for r in stream}
    twin = serving.Request(99, 6, 5, 9, E=70e6, nu=0.3, q=-60e3)
    force0, b0, n0 = prep[0]
    prep[99] = (force0, b0 * 0.6, n0)  # the same mesh and force as request 0, its own load
    stream = stream + [twin]
    srv = serving.NativeServer(engine(), hbm_budget=1 << 34, prepare_fn=lambda r, d: prep[r.id], max_cohort=2)
    served, wall = srv.run(stream, realtime=False)
    assert sorted(s.id for s in served) == sorted(r.id for r in stream) and wall > 0
    by_id = {s.id: s for s in served}
    py, _ = serving.Server(engine(), hbm_budget=1 << 34, prepare_fn=lambda r, d: prep[r.id]).run(
        [r for r in stream if not isinstance(r, serving.J2Request)], realtime=False)
    py = {s.id: s for s in py}
    for r in stream:
        s = by_id[r.id]
        assert s.result.converged, r.id
        assert 0.0 <= s.admitted <= s.done
        if isinstance(r, serving.J2Request):
            mesh, f, mon, n = prep[r.id]
            force = fx.InternalForce(mesh)
            u, res = serving.solve_j2_alone(r, force, torch.as_tensor(f, device=DEV), mon)
            assert np.array_equal(s.x, u), r.id
            assert np.array_equal(s.result.monitor, res.monitor), r.id
            assert np.array_equal(s.result.newton, res.newton), r.id
        else:
            assert np.array_equal(s.x, py[r.id].x), r.id
    op = fx.MatrixFreeOperator(force0, fx.OperatorCoefficients())
    for rid, b in ((0, b0), (99, b0 * 0.6)):
        y = torch.zeros(n0, dtype=torch.float64, device=DEV)
        op.apply(torch.as_tensor(by_id[rid].x, device=DEV), y)
        assert np.linalg.norm(b - y.cpu().numpy()) <= RTOL * np.linalg.norm(b)


def test_native_server_real_time():
    """Arrivals in real time: no request is admitted before it arrives, every one is served, and the
    latencies come from the library's clock."""
    stream = [serving.Request(i, 4 + i % 3, 4, 6 + i, arrival=0.02 * i) for i in range(8)]
    served, wall = serving.NativeServer(engine(), hbm_budget=1 << 34).run(stream, realtime=True)
    assert len(served) == 8 and all(s.result.converged for s in served)
    for s in served:
        assert s.admitted >= s.arrival - 1e-9 and s.done >= s.admitted, s
    assert wall >= 0.14


def test_native_server_second_cohort_starts_while_first_runs():
    """A J2 request that arrives while a cohort runs starts another cohort on a free lane (it does not
    wait for the first path to end), and both results are bit for bit their paths alone."""
    a0 = with_loads([serving.J2Request(0, 2, 2, 30, E=90e6, sigma_y=150e3, total=0.0, steps_per_cycle=8)])[0]
    a = serving.J2Request(0, a0.nx, a0.ny, a0.nz, a0.E, a0.sigma_y, a0.total, a0.h, cycles=3, steps_per_cycle=8,
                          arrival=0.0)
    b0 = with_loads([serving.J2Request(1, 1, 1, 24, E=60e6, sigma_y=80e3, total=0.0, steps_per_cycle=4)])[0]
    b = serving.J2Request(1, b0.nx, b0.ny, b0.nz, b0.E, b0.sigma_y, b0.total, b0.h, cycles=1, steps_per_cycle=4,
                          arrival=0.02)
    prep = {r.id: serving.prepare_j2(r) for r in (a, b)}
    srv = serving.NativeServer(engine(), hbm_budget=1 << 34, prepare_fn=lambda r, d: prep[r.id], max_lanes=2)
    served, _ = srv.run([a, b], realtime=True)
    s = {x.id: x for x in served}
    assert s[1].admitted < s[0].done, (s[1].admitted, s[0].done)
    for r in (a, b):
        mesh, f, mon, n = prep[r.id]
        u, res = serving.solve_j2_alone(r, fx.InternalForce(mesh), torch.as_tensor(f, device=DEV), mon)
        assert s[r.id].result.converged
        assert np.array_equal(s[r.id].x, u) and np.array_equal(s[r.id].result.monitor, res.monitor), r.id
