"""Quasi-static load paths (the implicit static stage of the path: ImplicitStage's load steps and
Newton loop, src/exec/implicit_stage.cpp:118-437, without inertia): for each load factor, Newton
iterations to equilibrium with the current material state, then commit_state.

`cyclic_factors` gives the cyclic loading of the batched J2 configuration: `cycles` full cycles
0 -> +1 -> -1 -> 0 in `steps_per_cycle` load steps each.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import ConjugateGradient, MatrixFreeOperator, OperatorCoefficients, SolveOptions


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
