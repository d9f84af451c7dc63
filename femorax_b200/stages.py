"""Implicit stages over the device solvers (ImplicitStage, src/exec/implicit_stage.cpp:118-437):

- `load_path`: quasi-static load steps; for each load factor, Newton iterations to equilibrium
  with the current material state (fx_solver_newton), then commit_state. `cyclic_factors` gives
  the cyclic loading of the batched J2 configuration: `cycles` full cycles 0 -> +1 -> -1 -> 0 in
  `steps_per_cycle` load steps each.
- `newmark_run`: transient Newmark steps (fx_solver_newmark) under a time-dependent load, with the
  plain FP64 CG or the mixed-precision (FP32 CG in FP64 refinement) inner solve.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import (BatchedNewton, ConjugateGradient, MatrixFreeOperator, MixedPrecisionSolver, OperatorCoefficients,
               SolveOptions)


def cyclic_factors(cycles: int, steps_per_cycle: int) -> np.ndarray:
    """Load factors of `cycles` triangular cycles 0 -> 1 -> -1 -> 0, `steps_per_cycle` steps each."""
    t = np.arange(1, cycles * steps_per_cycle + 1) / steps_per_cycle
    ph = t % 1.0
    return np.where(ph <= 0.25, 4 * ph, np.where(ph <= 0.75, 2 - 4 * ph, 4 * ph - 4))


@dataclasses.dataclass
class PathResult:
    factors: np.ndarray
    monitor: np.ndarray          # the monitored equation's displacement after each step
    newton: np.ndarray           # Newton iterations per step
    cg: np.ndarray               # CG iterations per step
    plastic: np.ndarray          # plastic points at each step's last force evaluation
    converged: bool


def load_path(force, fext_unit, factors, monitor_eq: int, tol: float = 1e-6, test: str = "NormUnbalance",
              cg_rtol: float = 1e-12, max_newton: int = 25, stream=None) -> PathResult:
    """Run the load path f_ext = factor * fext_unit (device vector) on `force`; displacements start
    at zero and the material state at its committed state."""
    import torch
    n = force.num_equations
    dev = fext_unit.device
    solver = ConjugateGradient(SolveOptions(relative_tolerance=cg_rtol, max_iterations=20000))
    solver.setup(MatrixFreeOperator(force, OperatorCoefficients(1.0, 0.0, 0.0)), stream)
    u = torch.zeros(n, dtype=torch.float64, device=dev)
    mon, nit, cgit, npl = [], [], [], []
    ok = True
    for lam in factors:
        fext = fext_unit * float(lam)
        it, res = solver.newton(fext, u, tol=tol, test=test, max_newton=max_newton, stream=stream)
        ok = ok and res.converged
        npl.append(force.plastic_points())
        force.commit_state(stream)
        mon.append(float(u[monitor_eq].item()))
        nit.append(it)
        cgit.append(res.iterations)
    return PathResult(np.asarray(factors, float), np.array(mon), np.array(nit), np.array(cgit), np.array(npl), ok)


@dataclasses.dataclass
class NewmarkResult:
    monitor: np.ndarray          # the monitored equation's displacement after each step
    newton: np.ndarray           # Newton iterations per step
    inner: np.ndarray            # linear-solver iterations per step (CG, or inner FP32 CG)
    refinements: np.ndarray      # FP64 refinement rounds per step (mixed precision)
    converged: bool
    seconds: float               # wall time of the steps


def newmark_run(force, load, steps: int, dt: float, monitor_eq: int, mixed: bool = False, beta: float = 0.25,
                gamma: float = 0.5, tol: float = 1e-6, rtol: float = 1e-8, inner_tolerance: float = 1e-4,
                stream=None) -> NewmarkResult:
    """`steps` Newmark steps from rest under f_ext(t) = load(t) (a device vector for each step
    time t = (i + 1) dt); the inner linear solves to rtol (relative, FP64 residual)."""
    import time

    import torch
    n = force.num_equations
    k = OperatorCoefficients(1.0, gamma / (beta * dt), 1.0 / (beta * dt * dt))
    opts = SolveOptions(relative_tolerance=rtol, max_iterations=20000)
    solver = MixedPrecisionSolver(opts, inner_tolerance=inner_tolerance) if mixed else ConjugateGradient(opts)
    solver.setup(MatrixFreeOperator(force, k), stream)
    dev = torch.device("cuda", force.device)
    u, v, a = (torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(3))
    mon, nit, inner, refs = [], [], [], []
    ok = True
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in range(steps):
        it, res = solver.newmark_step(load((i + 1) * dt), u, v, a, dt, beta, gamma, tol=tol, stream=stream)
        ok = ok and res.converged
        force.commit_state(stream)
        mon.append(u[monitor_eq].clone())
        nit.append(it)
        inner.append(res.iterations)
        refs.append(res.refinements)
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    return NewmarkResult(torch.stack(mon).cpu().numpy(), np.array(nit), np.array(inner), np.array(refs), ok, secs)


@dataclasses.dataclass
class BatchedPathResult:
    monitor: np.ndarray          # [steps, instances]: each instance's monitored displacement
    newton: np.ndarray           # [steps, instances]: Newton solves
    converged: bool
    seconds: float               # wall time of the steps


def batched_load_path(meshes, fext_units, factors, monitor_eqs, tol: float = 1e-6, cg_rtol: float = 1e-12,
                      max_newton: int = 25, device: int = 0) -> BatchedPathResult:
    """`load_path` for many meshes at once (BatchedNewton): instance i under factor *
    fext_units[i] (host), monitoring its equation monitor_eqs[i]; per instance the same bits as
    load_path on that mesh alone."""
    import time

    import torch
    b = BatchedNewton(meshes, SolveOptions(relative_tolerance=cg_rtol, max_iterations=20000), device)
    dev = torch.device("cuda", device)
    F = torch.as_tensor(b.combine(fext_units), device=dev)
    u = torch.zeros(b.total, dtype=torch.float64, device=dev)
    idx = torch.as_tensor(np.asarray(b.offsets[:-1]) + np.asarray(monitor_eqs), device=dev)
    mon, nit = [], []
    ok = True
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for lam in factors:
        it, res = b.step(F * float(lam), u, tol=tol, max_newton=max_newton)
        ok = ok and all(r.converged for r in res)
        b.commit_state()
        mon.append(u[idx].clone())
        nit.append(it)
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    return BatchedPathResult(torch.stack(mon).cpu().numpy(), np.array(nit), ok, secs)
