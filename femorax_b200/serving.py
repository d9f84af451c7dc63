"""Serving: a request loop over a BatchEngine (continuous batching of static solves).

A request is a structured hex8 block (its model) and a load. The loop
  - prepares each arrived request's resident state (compile step, device maps: an InternalForce;
    this allocates) on a pool of host threads, in arrival order;
  - admits prepared requests, in arrival order, into the engine while their HBM footprint (the
    mesh's device bytes) fits the budget and the engine has a free slot and range;
  - advances every admitted solve by one refinement round per pass (one batched launch per
    operator apply for all of them), so requests that arrive while others run join at the next
    round and their work overlaps on the device;
  - retires finished solves, frees their footprint, and records the latency from arrival to the
    solution on the host.
Each slot's arithmetic does not depend on the others, so a request's solution is bit for bit the
same alone and in any mix (tests/test_gpu_batch.py checks it).

`serve_one_at_a_time` is the comparison: the same stream, first come first served, each request
solved alone by the plain FP64 Jacobi-PCG to the same tolerance.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import dataclasses
import math
import time

import numpy as np

from . import (BatchEngine, ConjugateGradient, InternalForce, MatrixFreeOperator, Model, OperatorCoefficients,
               SolveOptions, SolveResult, meshes)


@dataclasses.dataclass
class Request:
    """A static solve: an nx x ny x nz block of h-metre boxes (base fixed), E, nu, and a uniform
    vertical traction q (Pa) on its top face."""
    id: int
    nx: int
    ny: int
    nz: int
    E: float = 80e6
    nu: float = 0.3
    q: float = -100e3
    h: float = 1.0
    arrival: float = 0.0  # seconds after the stream starts

    @property
    def equations(self) -> int:
        return 3 * (self.nx + 1) * (self.ny + 1) * self.nz


@dataclasses.dataclass
class Served:
    id: int
    x: np.ndarray
    result: SolveResult
    arrival: float
    admitted: float
    done: float

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def equation_map(compiled):
    """eq[tag, dof]: the equation of (node tag, dof 0..2), -1 fixed, as an array indexed by tag,
    from the compile step's arrays."""
    tags = compiled.array("node_tag")
    off = compiled.array("dof_offset")
    eq = compiled.array("eq")
    out = np.full((int(tags.max()) + 1, 3), -1, dtype=np.int64)
    for d in range(3):
        out[tags, d] = eq[off[:-1] + d]
    return out


def top_load(req: Request, eqmap) -> np.ndarray:
    """Equation-space load of the uniform vertical traction q on the top face: each top quad gives
    q h^2 / 4 to each of its 4 nodes (a top node carries the shares of the 1, 2 or 4 quads around it)."""
    share = req.q * req.h * req.h / 4.0
    ci = np.full(req.nx + 1, 2.0)
    cj = np.full(req.ny + 1, 2.0)
    ci[[0, -1]] = 1.0
    cj[[0, -1]] = 1.0
    i, j = np.meshgrid(np.arange(req.nx + 1), np.arange(req.ny + 1), indexing="ij")
    tags = 1 + i + (req.nx + 1) * (j + (req.ny + 1) * req.nz)
    q = eqmap[tags.ravel(), 2]
    f = (share * np.outer(ci, cj)).ravel()
    b = np.zeros(int(eqmap.max()) + 1)
    keep = q >= 0
    np.add.at(b, q[keep], f[keep])
    return b


def prepare(req: Request, device: int = 0):
    """The request's resident state: (InternalForce, right-hand side, equations)."""
    spec = meshes.box_model(req.nx, req.ny, req.nz, (req.nx * req.h, req.ny * req.h, req.nz * req.h), E=req.E,
                            nu=req.nu)
    comp = Model(spec).compile()
    b = top_load(req, equation_map(comp))
    force = InternalForce(comp.mesh(), device=device)
    return force, b, comp.num_equations


def synthetic_stream(count: int, rate: float, min_dof: float = 1e4, max_dof: float = 2e6, seed: int = 0):
    """Poisson arrivals at `rate` requests/s; sizes log-uniform in [min_dof, max_dof] equations on
    near-cubic blocks; E ~ U[50, 200] MPa, nu ~ U[0.25, 0.40]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        dof = math.exp(rng.uniform(math.log(min_dof), math.log(max_dof)))
        n = max(1, int(round((dof / 3.0) ** (1.0 / 3.0))))
        nz = max(1, int(round(dof / (3.0 * (n + 1) ** 2))))
        out.append(Request(i, n, n, nz, E=rng.uniform(50e6, 200e6), nu=rng.uniform(0.25, 0.40), arrival=t))
    return out


def percentile(v, p):
    return float(np.percentile(np.asarray(v), p)) if len(v) else float("nan")


class Server:
    """The continuous-batching loop over one BatchEngine."""

    def __init__(self, engine: BatchEngine, hbm_budget: int, device: int = 0, prep_threads: int = 4,
                 prepare_fn=None):
        self.engine = engine
        self.budget = int(hbm_budget)
        self.device = device
        self.prep_threads = prep_threads
        self.prepare = prepare_fn or prepare
        self.resident = 0  # footprint of the admitted requests

    def run(self, requests, realtime: bool = True):
        """Serve `requests` (sorted by arrival). With realtime, a request becomes visible at its
        arrival time; otherwise all are visible at once. Returns (served list, wall seconds)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        now = (lambda: time.perf_counter() - t0) if realtime else (lambda: math.inf)
        pool = cf.ThreadPoolExecutor(max_workers=self.prep_threads)
        pending = collections.deque()  # (request, future) in arrival order
        slots = {}                     # slot -> (request, footprint, admitted time)
        served = []
        nxt = 0
        try:
            while nxt < len(reqs) or pending or slots:
                # arrivals
                t = now()
                while nxt < len(reqs) and reqs[nxt].arrival <= t:
                    pending.append((reqs[nxt], pool.submit(self.prepare, reqs[nxt], self.device)))
                    nxt += 1
                # admissions in arrival order, while the footprint fits and the engine has room
                while pending and pending[0][1].done():
                    req, fut = pending[0]
                    force, b, n = fut.result()
                    foot = int(force.info()["device_bytes"])
                    if slots and self.resident + foot > self.budget:
                        break
                    slot = self.engine.try_admit(force, b)
                    if slot is None:
                        break
                    pending.popleft()
                    self.resident += foot
                    slots[slot] = (req, foot, time.perf_counter() - t0)
                if not slots and pending and pending[0][1].done():
                    raise RuntimeError(f"request {pending[0][0].id} does not fit the engine even alone")
                if not slots:
                    # nothing on the GPU: wait for the next preparation or arrival
                    if pending:
                        cf.wait([pending[0][1]], return_when=cf.FIRST_COMPLETED)
                    elif nxt < len(reqs) and realtime:
                        time.sleep(max(0.0, min(0.01, reqs[nxt].arrival - now())))
                    continue
                self.engine.round()
                for slot in list(slots):
                    if self.engine.finished(slot):
                        req, foot, adm = slots.pop(slot)
                        x, res = self.engine.retire(slot)
                        self.resident -= foot
                        done = time.perf_counter() - t0
                        served.append(Served(req.id, x, res, req.arrival if realtime else 0.0, adm, done))
        finally:
            pool.shutdown(wait=True)
        return served, time.perf_counter() - t0


def resident(requests, device: int = 0, rtol: float = 1e-8):
    """Prepare every request's mesh up front (the resident state a serving process keeps):
    {id: (force, b, n)}, and for the one-at-a-time arm a plain FP64 CG per mesh, already created
    (its work vectors allocated): {id: solver}."""
    prepared = {r.id: prepare(r, device) for r in requests}
    solvers = {}
    for rid, (force, b, n) in prepared.items():
        cg = ConjugateGradient(SolveOptions(relative_tolerance=rtol))
        cg.setup(MatrixFreeOperator(force, OperatorCoefficients()))
        solvers[rid] = cg
    return prepared, solvers


def serve_one_at_a_time(requests, rtol: float = 1e-8, realtime: bool = True, device: int = 0, prepared=None,
                        solvers=None):
    """The same stream, first come first served, each solved alone by plain FP64 Jacobi-PCG. With
    `prepared` / `solvers` (from resident()) the meshes and solvers are resident; otherwise each
    request is prepared when its turn comes."""
    import torch
    reqs = sorted(requests, key=lambda r: r.arrival)
    dev = torch.device("cuda", device)
    t0 = time.perf_counter()
    served = []
    for req in reqs:
        if realtime:
            wait = req.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        adm = time.perf_counter() - t0
        force, b, n = prepared[req.id] if prepared else prepare(req, device)
        op = MatrixFreeOperator(force, OperatorCoefficients())
        cg = solvers[req.id] if solvers else ConjugateGradient(SolveOptions(relative_tolerance=rtol))
        cg.setup(op)  # the Jacobi diagonal, as the engine builds it at admission
        bt = torch.as_tensor(b, device=dev)
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        res = cg.solve(bt, x)
        xh = x.cpu().numpy()
        done = time.perf_counter() - t0
        served.append(Served(req.id, xh, res, req.arrival if realtime else 0.0, adm, done))
    return served, time.perf_counter() - t0


def summary(served, wall):
    lat = [s.latency for s in served]
    return {"solves": len(served), "solves_per_s": len(served) / wall if wall > 0 else float("nan"),
            "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99),
            "converged": int(sum(s.result.converged for s in served)), "wall_s": wall}
