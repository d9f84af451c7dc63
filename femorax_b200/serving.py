"""Serving: a request loop over a BatchEngine (continuous batching of static solves) and a lane of
batched J2 load paths.

A request is a structured hex8 block (its model) and a load: a static elastic solve (`Request`)
or a quasi-static J2 load path (`J2Request`). For the static solves the loop
  - prepares each arrived request's resident state (compile step, device maps: an InternalForce;
    this allocates) on a pool of host threads, in arrival order;
  - admits prepared requests, in arrival order, into the engine while their HBM footprint (the
    mesh's device bytes) fits the budget and the engine has a free slot and range;
  - advances every admitted solve in ticks of 8 inner iterations (one batched launch per operator
    apply for all of them, each solve in its own phase: outer FP64 residual, inner solve,
    correction), so requests that arrive while others run join at the next tick and their work
    overlaps on the device;
  - retires finished solves, frees their footprint, and records the latency from arrival to the
    solution on the host.
Each slot's arithmetic does not depend on the others, so a request's solution is bit for bit the
same alone and in any mix (tests/test_gpu_batch.py checks it).

J2 load paths run in cohorts: when the J2 lane is idle, the prepared J2 requests waiting (in
arrival order, up to `max_cohort`, the same load path) become one BatchedNewton (one combined
mesh, per-instance Newton and CG on the device), which advances one load step per pass of the
loop, after engine ticks that take as long as its last step did, and retires all its requests at
the end of the path (NativeServer runs each cohort on a thread of its own instead). A cohort
takes no members once it runs, so while the engine is busy an idle lane waits (at most
`cohort_window` seconds) for the requests queued behind a prepared head to be prepared too. Each
instance's arithmetic is that of the load path alone, bit for bit (tests/test_gpu_serving.py).

`serve_one_at_a_time` is the comparison: the same stream, first come first served, each request
solved alone by the plain FP64 path (Jacobi-PCG; for J2, Newton with Jacobi-PCG per load step).
"""
from __future__ import annotations

import collections
import itertools
import concurrent.futures as cf
import dataclasses
import math
import time

import numpy as np

from . import (BatchEngine, BatchedNewton, ConjugateGradient, InternalForce, MatrixFreeOperator, Model,
               OperatorCoefficients, SolveOptions, SolveResult, device_memory, meshes, stages)


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
class J2Request:
    """A quasi-static J2 load path (the batched J2 configuration): an nx x ny x nz block of
    h-metre boxes, base fixed, J2 with yield stress sigma_y, hardening H = 0.05 E and kinematic
    share 0.5, under a horizontal shear traction on its top face totalling `total` newtons, scaled
    by `cycles` triangular load cycles of `steps_per_cycle` steps."""
    id: int
    nx: int
    ny: int
    nz: int
    E: float = 80e6
    sigma_y: float = 100e3
    total: float = 1e3
    h: float = 0.5
    cycles: int = 1
    steps_per_cycle: int = 8
    arrival: float = 0.0

    @property
    def equations(self) -> int:
        return 3 * (self.nx + 1) * (self.ny + 1) * self.nz

    @property
    def path(self):
        return (self.cycles, self.steps_per_cycle)


@dataclasses.dataclass
class J2Result:
    """A served J2 load path: the monitored top displacement after each step and the Newton
    solves per step; converged when every step converged."""
    monitor: np.ndarray
    newton: np.ndarray
    converged: bool


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
    return meshes.equation_map(compiled)


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


def j2_spec(req: J2Request):
    return meshes.box_model(req.nx, req.ny, req.nz, (req.nx * req.h, req.ny * req.h, req.nz * req.h), E=req.E,
                            nu=0.3, kind=1, sigma_y=req.sigma_y, H=0.05 * req.E, hk=0.5)


def prepare_j2(req: J2Request, device: int = 0):
    """A J2 request's host state: (mesh arrays, unit load, monitored equation, equations). The
    device state is the cohort's (BatchedNewton) or, alone, an InternalForce."""
    comp = Model(j2_spec(req)).compile()
    f, mon = stages.top_shear(j2_spec(req), equation_map(comp), req.total)
    return comp.mesh(), f, mon, comp.num_equations


def prepare_any(req, device: int = 0):
    return prepare_j2(req, device) if isinstance(req, J2Request) else prepare(req, device)


def j2_footprint(mesh) -> int:
    """Device bytes of one J2 instance in a cohort: element maps and slots (8 nodes, 24 equations,
    24 slot values), the material state of 8 points (two 13-value states and an 8-value tangent),
    and about 20 vectors of its equations."""
    per_element = 4 * (8 + 24 + 1) + 8 * 24 + 8 * 8 * (2 * 13 + 8)
    return int(mesh.padded * per_element + 8 * 20 * mesh.num_equations)


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


def pooled_stream(count: int, rate: float, models: int = 48, j2_share: float = 0.3, j2_models: int = 16,
                  min_dof: float = 1e4, max_dof: float = 2e6, seed: int = 0, cycles: int = 1, steps_per_cycle: int = 8,
                  j2_sizes=(1, 2, 4, 8), j2_nz=(20, 40)):
    """A served stream over resident models: `models` elastic blocks (sizes log-uniform in [min_dof,
    max_dof] equations, E ~ U[50, 200] MPa, nu ~ U[0.25, 0.40]) and `j2_models` J2 blocks (as
    mixed_stream's J2 requests); Poisson arrivals at `rate`, a share j2_share of the requests J2
    load paths on a J2 model, the others static solves on an elastic model with their own top
    traction q ~ U[-150, -50] kPa. Requests on the same model share its resident state (resident()
    keys it by the model's parameters)."""
    rng = np.random.default_rng(seed)
    pool = synthetic_stream(models, 1.0, min_dof, max_dof, seed + 7)
    j2pool = [r for r in mixed_stream(4 * j2_models, 1.0, j2_share=1.0, seed=seed + 11, cycles=cycles,
                                      steps_per_cycle=steps_per_cycle, j2_sizes=j2_sizes, j2_nz=j2_nz)][:j2_models]
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        if rng.uniform() < j2_share:
            m = j2pool[int(rng.integers(len(j2pool)))]
            out.append(dataclasses.replace(m, id=i, arrival=t))
        else:
            m = pool[int(rng.integers(len(pool)))]
            out.append(dataclasses.replace(m, id=i, q=float(rng.uniform(-150e3, -50e3)), arrival=t))
    return out


def model_key(req):
    """The parameters of a request's model (mesh, material, load pattern), without its load
    magnitude: requests with equal keys share their resident state."""
    if isinstance(req, J2Request):
        return ("j2", req.nx, req.ny, req.nz, req.E, req.sigma_y, req.total, req.h, req.path)
    return ("el", req.nx, req.ny, req.nz, req.E, req.nu, req.h)


def mixed_stream(count: int, rate: float, j2_share: float = 0.3, min_dof: float = 1e4, max_dof: float = 2e6,
                 seed: int = 0, cycles: int = 1, steps_per_cycle: int = 8, j2_sizes=(1, 2, 4, 8, 16, 24),
                 j2_nz=(20, 400)):
    """The served mixed stream: Poisson arrivals at `rate`; a share j2_share of the requests are J2
    load paths (the batched J2 configuration's instances: nx = ny from j2_sizes, nz uniform in
    j2_nz, sigma_y U[50, 200] kPa), the others static elastic solves as synthetic_stream."""
    rng = np.random.default_rng(seed)
    elastic = synthetic_stream(count, rate, min_dof, max_dof, seed)
    j2 = stages.j2_instances(count, seed=seed + 1, sizes=j2_sizes, nz_range=j2_nz)
    out = []
    for i, r in enumerate(elastic):
        if rng.uniform() < j2_share:
            spec, total = j2[i]
            nx, ny, nz, h, _, _ = spec.grid
            g = spec.groups[0]
            out.append(J2Request(r.id, nx, ny, nz, E=g.E, sigma_y=g.sigma_y, total=total, h=h, cycles=cycles,
                                 steps_per_cycle=steps_per_cycle, arrival=r.arrival))
        else:
            out.append(r)
    return out


class J2Lane:
    """A cohort of J2 load paths advancing together, one load step per call of step()."""

    def __init__(self, device: int = 0, tol: float = 1e-6, cg_rtol: float = 1e-12, max_newton: int = 25):
        self.device = device
        self.tol = tol
        self.cg_rtol = cg_rtol
        self.max_newton = max_newton
        self.members = []  # [(request, footprint, admitted)]
        self.batch = None

    @property
    def idle(self) -> bool:
        return not self.members

    def start(self, members, prepared):
        """members: [(request, footprint, admitted)], all with the same load path; prepared: their
        prepare_j2 results."""
        import torch
        self.members = list(members)
        reqs = [m[0] for m in members]
        self.factors = stages.cyclic_factors(*reqs[0].path)
        self.batch = BatchedNewton([p[0] for p in prepared],
                                   SolveOptions(relative_tolerance=self.cg_rtol, max_iterations=20000), self.device)
        dev = torch.device("cuda", self.device)
        self.F = torch.as_tensor(self.batch.combine([p[1] for p in prepared]), device=dev)
        self.u = torch.zeros(self.batch.total, dtype=torch.float64, device=dev)
        self.idx = torch.as_tensor(np.asarray(self.batch.offsets[:-1]) + np.asarray([p[2] for p in prepared]),
                                   device=dev)
        self.k = 0
        self.mon, self.nit = [], []
        self.conv = np.ones(len(members), dtype=bool)

    def step(self):
        """One load step of every member; at the end of the path returns [(request, footprint,
        admitted, final displacement, J2Result)] and the lane becomes idle, else []."""
        it, res = self.batch.step(self.F * float(self.factors[self.k]), self.u, tol=self.tol,
                                  max_newton=self.max_newton)
        self.conv &= np.array([r.converged for r in res], dtype=bool)
        self.batch.commit_state()
        self.mon.append(self.u[self.idx].clone())
        self.nit.append(it)
        self.k += 1
        if self.k < len(self.factors):
            return []
        import torch
        mon = torch.stack(self.mon).cpu().numpy()
        nit = np.array(self.nit)
        us = self.batch.split(self.u.cpu().numpy())
        out = []
        for i, (req, foot, adm) in enumerate(self.members):
            out.append((req, foot, adm, us[i], J2Result(mon[:, i], nit[:, i], bool(self.conv[i]))))
        self.members, self.batch = [], None
        return out


def percentile(v, p):
    return float(np.percentile(np.asarray(v), p)) if len(v) else float("nan")


class Server:
    """The continuous-batching loop over one BatchEngine (static solves) and one J2Lane (J2 load
    paths, in cohorts of up to max_cohort)."""

    def __init__(self, engine: BatchEngine, hbm_budget: int = None, device: int = 0, prep_threads: int = 4,
                 prepare_fn=None, lane=None, max_cohort: int = 32, cohort_window: float = 0.25,
                 reserve: int = 2 << 30):
        """hbm_budget: the bytes the admitted requests' footprints may hold; None sizes it from the
        device's free memory now (fx_device_memory, as the reference sizes against cudaMemGetInfo),
        less `reserve` for the work vectors and the library's own buffers."""
        self.engine = engine
        if hbm_budget is None:
            free, _ = device_memory(device)
            hbm_budget = max(0, free - int(reserve))
        self.budget = int(hbm_budget)
        self.device = device
        self.prep_threads = prep_threads
        self.prepare = prepare_fn or prepare_any
        self.lane = lane if lane is not None else J2Lane(device)
        self.max_cohort = max_cohort
        # a running cohort takes no new members, so an idle lane waits up to this many seconds for
        # the J2 requests queued behind a prepared head (same load path) while the engine is busy
        self.cohort_window = float(cohort_window)
        # while a J2 cohort runs, a pass runs engine ticks (8 inner iterations each) for at least this
        # many seconds (and as long as the cohort's last load step took) before its next load step
        self.tick_budget = 0.02
        self.resident = 0  # footprint of the admitted requests

    def _start_cohort(self, pending_j2, slots, t0):
        """Moves the prepared J2 requests at the head of pending_j2 (same load path, up to
        max_cohort, while the footprint fits) into the idle lane."""
        members, prepared, foot_sum = [], [], 0
        path = pending_j2[0][0].path
        while pending_j2 and len(members) < self.max_cohort and pending_j2[0][1].done():
            req, fut = pending_j2[0]
            if req.path != path:
                break
            prep = fut.result()
            foot = j2_footprint(prep[0])
            if (slots or members) and self.resident + foot_sum + foot > self.budget:
                break
            pending_j2.popleft()
            members.append((req, foot, time.perf_counter() - t0))
            prepared.append(prep)
            foot_sum += foot
        if members:
            self.lane.start(members, prepared)
            self.resident += foot_sum

    def run(self, requests, realtime: bool = True):
        """Serve `requests` (sorted by arrival). With realtime, a request becomes visible at its
        arrival time; otherwise all are visible at once. Returns (served list, wall seconds)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        now = (lambda: time.perf_counter() - t0) if realtime else (lambda: math.inf)
        pool = cf.ThreadPoolExecutor(max_workers=self.prep_threads)
        pending = collections.deque()     # static solves: (request, future) in arrival order
        pending_j2 = collections.deque()  # J2 load paths: (request, future) in arrival order
        slots = {}                        # slot -> (request, footprint, admitted time)
        served = []
        nxt = 0
        head_ready = None  # when the J2 queue's head was first seen prepared with the lane idle
        lane_s = 0.0  # seconds the lane's last load step took
        try:
            while nxt < len(reqs) or pending or pending_j2 or slots or not self.lane.idle:
                # arrivals
                t = now()
                while nxt < len(reqs) and reqs[nxt].arrival <= t:
                    r = reqs[nxt]
                    (pending_j2 if isinstance(r, J2Request) else pending).append(
                        (r, pool.submit(self.prepare, r, self.device)))
                    nxt += 1
                # admissions in arrival order, while the footprint fits and the engine has room
                while pending and pending[0][1].done():
                    req, fut = pending[0]
                    force, b, n = fut.result()
                    foot = int(force.info()["device_bytes"])
                    if (slots or not self.lane.idle) and self.resident + foot > self.budget:
                        break
                    slot = self.engine.try_admit(force, b)
                    if slot is None:
                        break
                    pending.popleft()
                    self.resident += foot
                    slots[slot] = (req, foot, time.perf_counter() - t0)
                if not slots and self.lane.idle and pending and pending[0][1].done():
                    raise RuntimeError(f"request {pending[0][0].id} does not fit the engine even alone")
                # a new J2 cohort when the lane is free: when the requests queued behind a prepared
                # head with its load path are all prepared too, when the engine runs nothing (the
                # GPU would wait), or when the head has waited cohort_window seconds
                if self.lane.idle and pending_j2 and pending_j2[0][1].done():
                    if head_ready is None:
                        head_ready = time.perf_counter()
                    path = pending_j2[0][0].path
                    queued = list(itertools.islice(itertools.takewhile(lambda q: q[0].path == path, pending_j2),
                                                   self.max_cohort))
                    if (all(f.done() for _, f in queued) or not slots
                            or time.perf_counter() - head_ready >= self.cohort_window):
                        self._start_cohort(pending_j2, slots, t0)
                        head_ready = None
                if not slots and self.lane.idle:
                    # nothing on the GPU: wait for the next preparation or arrival
                    heads = [q[0][1] for q in (pending, pending_j2) if q]
                    if heads:
                        cf.wait(heads, return_when=cf.FIRST_COMPLETED)
                    elif nxt < len(reqs) and realtime:
                        time.sleep(max(0.0, min(0.01, reqs[nxt].arrival - now())))
                    continue
                if slots:
                    # engine ticks: one per pass with the J2 lane idle, else for as long as the lane's
                    # last load step took (at least tick_budget seconds): the two share the time
                    until = time.perf_counter() + (0.0 if self.lane.idle else max(self.tick_budget, lane_s))
                    while True:
                        self.engine.round()
                        for slot in list(slots):
                            if self.engine.finished(slot):
                                req, foot, adm = slots.pop(slot)
                                x, res = self.engine.retire(slot)
                                self.resident -= foot
                                done = time.perf_counter() - t0
                                served.append(Served(req.id, x, res, req.arrival if realtime else 0.0, adm, done))
                        if not slots or time.perf_counter() >= until:
                            break
                if not self.lane.idle:
                    t_lane = time.perf_counter()
                    finished = self.lane.step()
                    lane_s = time.perf_counter() - t_lane
                    for req, foot, adm, u, res in finished:
                        self.resident -= foot
                        done = time.perf_counter() - t0
                        served.append(Served(req.id, u, res, req.arrival if realtime else 0.0, adm, done))
        finally:
            pool.shutdown(wait=True)
        return served, time.perf_counter() - t0


class NativeServer:
    """The serving loop in C++ (fx_server_*, serve.cu) over one BatchEngine: the same admission by
    footprint, engine ticks for the static solves and J2 cohorts (up to max_cohort, fx_nbatch) as
    Server, with up to max_lanes cohorts running at once, each on a thread and a stream of its own
    that overlap the engine's work on the device (J2 requests that arrive while one runs start the
    next), the loop, the arrival gating and the clock in the library; latency is measured by
    the host's steady clock inside it. run() takes the requests with their prepared state
    (prepare_fn(request, device) as for Server: (force, b, n) for a static solve, prepare_j2's
    (mesh, unit load, monitored equation, n) for a J2 path) and returns (served, wall seconds)."""

    def __init__(self, engine: BatchEngine, hbm_budget: int = None, device: int = 0, prepare_fn=None,
                 max_cohort: int = 32, max_lanes: int = 4, reserve: int = 2 << 30, tol: float = 1e-6,
                 max_newton: int = 25, cg_rtol: float = 1e-12, cg_max_iterations: int = 20000):
        self.engine = engine
        if hbm_budget is None:
            free, _ = device_memory(device)
            hbm_budget = max(0, free - int(reserve))
        self.budget = int(hbm_budget)
        self.device = device
        self.prepare = prepare_fn or prepare_any
        self.max_cohort = int(max_cohort)
        self.max_lanes = int(max_lanes)
        self.j2_settings = (float(tol), int(max_newton), float(cg_rtol), int(cg_max_iterations))

    def run(self, requests, realtime: bool = True):
        import ctypes as C
        from . import _lib as L
        from ._lib import check, lib
        reqs = sorted(requests, key=lambda r: r.arrival)
        h = C.c_void_p()
        check(lib().fx_server_create(self.engine._h, self.device, self.budget, self.max_cohort, self.max_lanes,
                                     C.byref(h)))
        keep, sizes = [], {}
        try:
            tol, max_newton, cg_rtol, cg_max_it = self.j2_settings
            for r in reqs:
                prep = self.prepare(r, self.device)
                if isinstance(r, J2Request):
                    mesh, f, mon, n = prep
                    cm, k = mesh.to_c()
                    f = np.ascontiguousarray(f, dtype=np.float64)
                    keep += [cm, k, f]
                    check(lib().fx_server_add_j2(h, r.id, C.byref(cm), f.ctypes.data_as(L.p_f64), int(mon), r.cycles,
                                                 r.steps_per_cycle, tol, max_newton, cg_rtol, cg_max_it,
                                                 float(r.arrival) if realtime else 0.0))
                    sizes[r.id] = (n, r.cycles * r.steps_per_cycle)
                else:
                    force, b, n = prep
                    b = np.ascontiguousarray(b, dtype=np.float64)
                    keep += [force, b]
                    check(lib().fx_server_add_static(h, r.id, force._h, b.ctypes.data_as(L.p_f64),
                                                     float(r.arrival) if realtime else 0.0))
                    sizes[r.id] = (n, 0)
            wall = C.c_double()
            check(lib().fx_server_run(h, 1 if realtime else 0, C.byref(wall)))
            served = []
            for r in reqs:
                n, steps = sizes[r.id]
                x = np.empty(n)
                res = L.fx_solve_result()
                t = (C.c_double * 3)()
                mon = np.empty(max(steps, 1))
                nit = np.empty(max(steps, 1), dtype=np.int32)
                check(lib().fx_server_result(h, r.id, x.ctypes.data_as(L.p_f64), C.byref(res), t,
                                             mon.ctypes.data_as(L.p_f64), nit.ctypes.data_as(L.p_i32)))
                if steps:
                    result = J2Result(mon[:steps].copy(), nit[:steps].astype(np.int64), bool(res.converged))
                else:
                    result = SolveResult(bool(res.converged), res.iterations, res.rhs_norm, res.initial_residual,
                                         res.final_residual, bool(res.indefinite), res.refinements)
                served.append(Served(r.id, x, result, t[0], t[1], t[2]))
            return served, wall.value
        finally:
            lib().fx_server_destroy(h)


def resident(requests, device: int = 0, rtol: float = 1e-8, j2_host: bool = False, cache: dict = None):
    """Prepare every request's mesh up front (the resident state a serving process keeps):
    {id: (force, b, n)} for static solves and {id: (force, unit load, monitored equation, n)} for
    J2 paths, and for the one-at-a-time arm a plain FP64 CG per mesh, already created (its work
    vectors allocated): {id: solver}. Requests with the same model_key share the model's force,
    solver and (J2) load; a static solve's right-hand side is its own (the model's unit traction
    load times its q). With j2_host, also {id: prepare_j2 result} (the serving loop's J2 cohorts
    build from these host arrays), shared per model too. `cache` (a dict) keeps the models between
    calls."""
    import torch
    prepared, solvers, host = {}, {}, {}
    models = cache if cache is not None else {}
    for r in requests:
        key = model_key(r)
        if key not in models:
            if isinstance(r, J2Request):
                mesh, f, mon, n = prepare_j2(r, device)
                force = InternalForce(mesh, device=device)
                models[key] = ((force, torch.as_tensor(f, device=torch.device("cuda", device)), mon, n),
                               ConjugateGradient(SolveOptions(relative_tolerance=1e-12, max_iterations=20000)),
                               (mesh, f, mon, n))
            else:
                unit = dataclasses.replace(r, q=1.0)
                force, b1, n = prepare(unit, device)
                cg = ConjugateGradient(SolveOptions(relative_tolerance=rtol))
                cg.setup(MatrixFreeOperator(force, OperatorCoefficients()))
                models[key] = ((force, b1, n), cg, None)
        state, solver, h = models[key]
        if isinstance(r, J2Request):
            prepared[r.id] = state
            host[r.id] = h
        else:
            force, b1, n = state
            prepared[r.id] = (force, r.q * b1, n)
        solvers[r.id] = solver
    if j2_host:
        return prepared, solvers, host
    return prepared, solvers


def solve_j2_alone(req: J2Request, force, f_unit, monitor_eq, solver=None, tol: float = 1e-6):
    """A J2 request alone by the plain FP64 path (stages.load_path from the virgin material state):
    (final displacement, J2Result)."""
    force.set_j2_state(np.zeros_like(force.j2_state("committed")), "committed")
    r = stages.load_path(force, f_unit, stages.cyclic_factors(*req.path), monitor_eq, tol=tol, solver=solver)
    return r.u, J2Result(r.monitor, r.newton, r.converged)


def serve_one_at_a_time(requests, rtol: float = 1e-8, realtime: bool = True, device: int = 0, prepared=None,
                        solvers=None):
    """The same stream, first come first served, each solved alone by the plain FP64 path
    (Jacobi-PCG; J2: Newton with Jacobi-PCG per load step). With `prepared` / `solvers` (from
    resident()) the meshes and solvers are resident; otherwise each request is prepared when its
    turn comes."""
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
        if isinstance(req, J2Request):
            if prepared:
                force, f, mon, n = prepared[req.id]
            else:
                mesh, fh, mon, n = prepare_j2(req, device)
                force, f = InternalForce(mesh, device=device), torch.as_tensor(fh, device=dev)
            xh, res = solve_j2_alone(req, force, f, mon, solvers[req.id] if solvers else None)
        else:
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
    out = {"solves": len(served), "solves_per_s": len(served) / wall if wall > 0 else float("nan"),
           "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99),
           "converged": int(sum(s.result.converged for s in served)), "wall_s": wall}
    j2 = [s.latency for s in served if isinstance(s.result, J2Result)]
    if j2:  # the J2 load paths' latencies apart (a path is many solves)
        out["j2_p50_s"] = percentile(j2, 50)
        out["j2_p99_s"] = percentile(j2, 99)
    return out
