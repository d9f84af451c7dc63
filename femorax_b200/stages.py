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
    u: np.ndarray = None         # the displacements after the last step (host)


def load_path(force, fext_unit, factors, monitor_eq: int, tol: float = 1e-6, test: str = "NormUnbalance",
              cg_rtol: float = 1e-12, max_newton: int = 25, stream=None, solver=None) -> PathResult:
    """Run the load path f_ext = factor * fext_unit (device vector) on `force`; displacements start
    at zero and the material state at its committed state. `solver`: a ConjugateGradient made
    beforehand (its work vectors allocated), or None to make one."""
    import torch
    n = force.num_equations
    dev = fext_unit.device
    if solver is None:
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
    return PathResult(np.asarray(factors, float), np.array(mon), np.array(nit), np.array(cgit), np.array(npl), ok,
                      u.cpu().numpy())


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
    refinements: np.ndarray = None  # [steps, instances]: refinement rounds (mixed)


def batched_load_path(meshes, fext_units, factors, monitor_eqs, tol: float = 1e-6, cg_rtol: float = 1e-12,
                      max_newton: int = 25, device: int = 0, mixed: bool = False,
                      inner_tolerance: float = 1e-4) -> BatchedPathResult:
    """`load_path` for many meshes at once (BatchedNewton): instance i under factor *
    fext_units[i] (host), monitoring its equation monitor_eqs[i]; per instance the same bits as
    load_path on that mesh alone (mixed: with a MixedPrecisionSolver of the same tolerances)."""
    import time

    import torch
    b = BatchedNewton(meshes, SolveOptions(relative_tolerance=cg_rtol, max_iterations=20000), device, mixed=mixed,
                      inner_tolerance=inner_tolerance)
    dev = torch.device("cuda", device)
    F = torch.as_tensor(b.combine(fext_units), device=dev)
    u = torch.zeros(b.total, dtype=torch.float64, device=dev)
    idx = torch.as_tensor(np.asarray(b.offsets[:-1]) + np.asarray(monitor_eqs), device=dev)
    mon, nit, refs = [], [], []
    ok = True
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for lam in factors:
        it, res = b.step(F * float(lam), u, tol=tol, max_newton=max_newton)
        ok = ok and all(r.converged for r in res)
        b.commit_state()
        mon.append(u[idx].clone())
        nit.append(it)
        refs.append([r.refinements for r in res])
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    return BatchedPathResult(torch.stack(mon).cpu().numpy(), np.array(nit), ok, secs, np.array(refs))


def j2_instances(count: int, seed: int = 0, sizes=(1, 2, 4, 8, 16, 24), nz_range=(20, 400), h: float = 0.5,
                 load_ratio: float = 1.2):
    """The batched J2 configuration's instances, seeded: soil columns and blocks of nx = ny drawn
    from `sizes` and nz uniform in nz_range, boxes of h metres, J2 with sigma_y ~ U[50, 200] kPa,
    E ~ U[40, 120] MPa, nu 0.3, H = 0.05 E, hk 0.5, base fixed; each with a uniform horizontal
    shear traction on its top face totalling load_ratio times the force that first yields the
    base in elastic bending, sigma_y b^3 / (6 L) (b the width, L the height).
    Returns [(spec, total top force)]."""
    from . import meshes
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(sizes))
        nz = int(rng.integers(nz_range[0], nz_range[1] + 1))
        sy = rng.uniform(50e3, 200e3)
        E = rng.uniform(40e6, 120e6)
        spec = meshes.box_model(n, n, nz, (n * h, n * h, nz * h), E=E, nu=0.3, kind=1, sigma_y=sy, H=0.05 * E,
                                hk=0.5)
        b, L = n * h, nz * h
        out.append((spec, load_ratio * sy * b ** 3 / (6.0 * L)))
    return out


def top_shear(spec, eqmap, total):
    """x-direction nodal loads of a uniform shear traction on the top face summing to `total`, and
    the equation of the top corner node's x displacement (eqmap: serving.equation_map)."""
    nx, ny, nz, _, _, _ = spec.grid
    ci = np.full(nx + 1, 2.0)
    cj = np.full(ny + 1, 2.0)
    ci[[0, -1]] = 1.0
    cj[[0, -1]] = 1.0
    i, j = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    tags = 1 + i + (nx + 1) * (j + (ny + 1) * nz)
    q = eqmap[tags.ravel(), 0]
    f = np.zeros(int(eqmap.max()) + 1)
    np.add.at(f, q[q >= 0], (total / (4.0 * nx * ny) * np.outer(ci, cj)).ravel()[q >= 0])
    return f, int(eqmap[tags[-1, -1], 0])
