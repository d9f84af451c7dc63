"""Batched and served solves (fx_engine_*) on a B200, through the C ABI.

- each slot's solution is bit for bit the single-mesh mixed-precision solve (FX_SOLVER_IR: FP32
  PCG inside FP64 refinement) of the same mesh, with the same inner iteration and round counts;
- a request's solution is bit for bit the same alone and in a mix, also when others join between
  its rounds (continuous batching);
- every solution meets the 1e-8 relative FP64 residual, checked here with the FP64 operator, and
  agrees with the plain FP64 CG solution to 1e-6 relative;
- admission refuses when no slot or no range of chunks is free, and a retire makes room again;
- the block-per-chunk and warp-per-chunk forms of the CG vector kernels give the same bits.
"""
import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import serving

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

DEV = torch.device("cuda:0")
RTOL = 1e-8
REQS = [
    serving.Request(0, 6, 5, 9),
    serving.Request(1, 10, 10, 12, E=120e6, nu=0.35),
    serving.Request(2, 3, 4, 40, E=60e6, nu=0.28),
    serving.Request(3, 14, 12, 7, E=150e6, nu=0.32, q=-50e3),
]


@pytest.fixture(scope="module")
def prepared():
    return {r.id: serving.prepare(r) for r in REQS}


def engine(capacity=1 << 20, slots=8):
    return fx.BatchEngine(capacity, slots, options=fx.SolveOptions(relative_tolerance=RTOL))


def run_to_end(e, slots, ticks=200):
    out = {}
    for _ in range(ticks):
        e.round()
        for s in list(slots):
            if e.finished(s):
                out[slots.pop(s)] = e.retire(s)
        if not slots:
            return out
    raise AssertionError("the engine did not finish")


@pytest.fixture(scope="module")
def alone(prepared):
    res = {}
    for rid, (force, b, n) in prepared.items():
        e = engine()
        s = e.admit(force, b)
        res[rid] = run_to_end(e, {s: rid})[rid]
    return res


def test_slot_equals_single_mixed_solve(prepared, alone):
    for rid, (force, b, n) in prepared.items():
        op = fx.MatrixFreeOperator(force, fx.OperatorCoefficients())
        ir = fx.MixedPrecisionSolver(fx.SolveOptions(relative_tolerance=RTOL), inner_tolerance=1e-4)
        ir.setup(op)
        x = torch.zeros(n, dtype=torch.float64, device=DEV)
        r = ir.solve(torch.as_tensor(b, device=DEV), x)
        xe, re = alone[rid]
        assert r.converged and re.converged
        assert np.array_equal(xe, x.cpu().numpy()), rid
        assert (re.iterations, re.refinements) == (r.iterations, r.refinements)
        assert re.final_residual == r.final_residual


def single_ir(force, b, n):
    op = fx.MatrixFreeOperator(force, fx.OperatorCoefficients())
    ir = fx.MixedPrecisionSolver(fx.SolveOptions(relative_tolerance=RTOL), inner_tolerance=1e-4)
    ir.setup(op)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    r = ir.solve(torch.as_tensor(b, device=DEV), x)
    return x.cpu().numpy(), r


def test_block_and_warp_forms_same_bits(prepared):
    """The CG vector kernels take a block per chunk for vectors of at most 1,024 chunks and a warp
    per chunk beyond; both sum in the same order. A small mesh batched beside one of more than 1,024
    chunks runs the engine's warp form, its single solve the block form: the same bits, iterations
    and rounds; the large mesh matches its own single solve too."""
    big = serving.Request(9, 100, 100, 70)
    fb, bb, nb = serving.prepare(big)
    assert nb > 1024 * 2048
    f0, b0, n0 = prepared[0]
    e = engine(capacity=3 << 20)
    s_big = e.admit(fb, bb)
    s0 = e.admit(f0, b0)
    out = run_to_end(e, {s_big: 9, s0: 0}, ticks=4000)
    for rid, (force, b, n) in ((9, (fb, bb, nb)), (0, (f0, b0, n0))):
        x, r = single_ir(force, b, n)
        xe, re = out[rid]
        assert r.converged and re.converged, rid
        assert np.array_equal(xe, x), rid
        assert (re.iterations, re.refinements) == (r.iterations, r.refinements), rid


def test_alone_and_in_mix_are_the_same(prepared, alone):
    e = engine()
    f0, b0, _ = prepared[0]
    f1, b1, _ = prepared[1]
    slots = {e.admit(f0, b0): 0, e.admit(f1, b1): 1}
    e.round()  # requests 2 and 3 arrive while 0 and 1 are on the device
    for rid in (2, 3):
        f, b, _ = prepared[rid]
        slots[e.admit(f, b)] = rid
    out = {}
    for _ in range(200):
        e.round()
        for s in list(slots):
            if e.finished(s):
                out[slots.pop(s)] = e.retire(s)
        if not slots:
            break
    assert sorted(out) == [0, 1, 2, 3]
    for rid, (x, r) in out.items():
        assert np.array_equal(x, alone[rid][0]), rid
        assert r.iterations == alone[rid][1].iterations


def test_fp64_residual_and_plain_cg(prepared, alone):
    k = fx.OperatorCoefficients()
    for rid, (force, b, n) in prepared.items():
        x, r = alone[rid]
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        force.apply_operator(k, torch.as_tensor(x, device=DEV), y)
        res = np.linalg.norm(b - y.cpu().numpy()) / np.linalg.norm(b)
        assert res <= RTOL, (rid, res)
        cg = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=1e-10))
        cg.setup(fx.MatrixFreeOperator(force, k))
        xc = torch.zeros(n, dtype=torch.float64, device=DEV)
        assert cg.solve(torch.as_tensor(b, device=DEV), xc).converged
        xc = xc.cpu().numpy()
        assert np.linalg.norm(x - xc) / np.linalg.norm(xc) <= 1e-6, rid


def test_admission_limits(prepared):
    f0, b0, n0 = prepared[0]
    f1, b1, n1 = prepared[1]
    small = fx.BatchEngine(n0, 4, options=fx.SolveOptions(relative_tolerance=RTOL))
    assert small.try_admit(f1, b1) is None  # larger than the whole capacity
    s0 = small.admit(f0, b0)
    assert small.try_admit(f0, b0) is None  # no free range
    one = fx.BatchEngine(1 << 20, 1, options=fx.SolveOptions(relative_tolerance=RTOL))
    s = one.admit(f0, b0)
    assert one.try_admit(f1, b1) is None  # no free slot
    one.retire(s)
    assert one.admit(f1, b1) == 0
    info = one.info()
    assert info["slots_in_use"] == 1 and info["in_use"] >= n1
    small.retire(s0)


def test_server_stream(alone):
    reqs = [serving.Request(r.id, r.nx, r.ny, r.nz, r.E, r.nu, r.q, r.h, arrival=0.001 * r.id) for r in REQS]
    srv = serving.Server(engine(), hbm_budget=1 << 34)
    served, wall = srv.run(reqs, realtime=False)
    assert sorted(s.id for s in served) == [0, 1, 2, 3]
    for s in served:
        assert s.result.converged
        assert np.array_equal(s.x, alone[s.id][0]), s.id
    summ = serving.summary(served, wall)
    assert summ["converged"] == 4 and summ["p99_s"] >= summ["p50_s"] > 0


def test_fp64_inner_engine(prepared):
    """inner="fp64": the same engine with FP64 inner solves (the batching without reduced
    precision). Every slot meets the 1e-8 FP64 residual in one refinement round, agrees with the
    plain FP64 CG solution to 1e-8 relative, and is bit for bit the same alone and in a mix; the
    same InternalForce admitted into two slots at once gives the same bits in both."""
    def eng():
        return fx.BatchEngine(1 << 20, 8, options=fx.SolveOptions(relative_tolerance=RTOL), inner_tolerance=0.5 * RTOL,
                              inner="fp64")
    alone64 = {}
    for rid, (force, b, n) in prepared.items():
        e = eng()
        s = e.admit(force, b)
        alone64[rid] = run_to_end(e, {s: rid})[rid]
    e = eng()
    slots = {e.admit(f, b): rid for rid, (f, b, _) in prepared.items()}
    f0, b0, _ = prepared[0]
    slots[e.admit(f0, b0)] = "again"
    mix = run_to_end(e, slots)
    assert np.array_equal(mix["again"][0], mix[0][0])
    for rid, (force, b, n) in prepared.items():
        x, r = alone64[rid]
        assert r.converged and r.refinements == 1, (rid, r)
        assert np.array_equal(mix[rid][0], x), rid
        op = fx.MatrixFreeOperator(force, fx.OperatorCoefficients())
        y = torch.zeros(n, dtype=torch.float64, device=DEV)
        op.apply(torch.as_tensor(x, device=DEV), y)
        res = np.linalg.norm(b - y.cpu().numpy()) / np.linalg.norm(b)
        assert res <= RTOL, (rid, res)
        cg = fx.ConjugateGradient(fx.SolveOptions(relative_tolerance=RTOL))
        cg.setup(op)
        xc = torch.zeros(n, dtype=torch.float64, device=DEV)
        assert cg.solve(torch.as_tensor(b, device=DEV), xc).converged
        xc = xc.cpu().numpy()
        assert np.max(np.abs(x - xc)) <= 1e-7 * np.max(np.abs(xc)), rid
    e2 = eng()
    e2.admit(f0, b0)
    with pytest.raises(fx.FxError):  # the precision is fixed while slots are in use
        fx._lib.check(fx._lib.lib().fx_engine_set_precision(e2._h, 0))


def test_persistent_work_list_same_bits(prepared, alone):
    """The batched apply as a persistent wave of CTAs over the work list gives every slot the same bits."""
    e = engine()
    e.set_persistent(True)
    slots = {e.admit(f, b): rid for rid, (f, b, _) in prepared.items()}
    out = run_to_end(e, slots)
    for rid in prepared:
        assert np.array_equal(out[rid][0], alone[rid][0]), rid
        assert out[rid][1].iterations == alone[rid][1].iterations
