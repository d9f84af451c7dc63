"""Benchmark: the plain FP64 matrix-free apply y = K x on the layered soil box (128 x 128 x 64
stdBrick, 8 layers, ~3.2 M equations), in GDoF/s (equations / apply time).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: one process per GPU (torchrun for N > 1), each GPU applies the operator of its own copy
of the mesh (independent replicas: no data-path collective; weak scaling); the timed region is K
applies with x resident in HBM, L2 flushed (a 256 MB write) between applies, each apply timed by
CUDA events on its stream; value = all ranks' equations x K / the slowest rank's summed time.
`e2e` is the same metric through the public host-buffer call (fx_apply_operator_host: pinned host
x in, y out, copies inside the timed region). `roofline` relates the kernel to the measured HBM
copy bandwidth with the algorithmic bytes of one apply: 8 neq (x) + 8 neq (y) + 32 n_el (8 node
ids) + 12 N (node -> equations) + 4 n_el (parameter index). `cpu_baseline` times the reference's
own InternalForce::apply_operator (built here from its sources, oracle/_ref) on a bounded sample.

`explicit` times the explicit wave configuration's stepping (FP64 and FP32, 4000 steps);
`newmark` compares the Newmark stage with plain FP64 and mixed-precision inner solves;
`pimy` times PressureIndependMultiYield material-point updates on the device (and on one host core) and
an explicit step of a 1 M-element plastic box; `pdmy` the PressureDependMultiYield point updates;
`batched_j2` compares the batched J2 Newton with one instance at a time on a bounded sample;
`served` compares solves/s and p50/p99 latency at a 1e-8 FP64 residual on a stream of static solves:
the batched mixed-precision engine behind the serving loop versus plain FP64 CG one at a time;
`served_mixed` does the same on a stream of 70 % static solves and 30 % J2 load paths (J2 cohorts
beside the engine's slots); `served_rates` serves that mix with Poisson arrivals at 20, 200 and
2000 requests/s in real time.

The reference arm (--impl reference) times that reference CPU path alone, on every host thread.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

WORKLOAD = dict(workload="layered soil box 128x128x64 stdBrick (8 layers, seed 0), plain FP64 y = K x",
                nx=128, ny=128, nz=64, layers=8, seed=0)
METRIC = "K*x GDoF/s (plain FP64 matrix-free apply, layered box 128x128x64)"


def max_over_ranks(values, dist=None, device="cpu"):
    """Each value's maximum over the ranks of the process group (the slowest rank's time); the
    values themselves without a group."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_value(world, neq, steps, total_ms):
    """GDoF/s of `world` independent replicas, each applying its own operator of neq equations
    `steps` times, the slowest taking total_ms in all."""
    return world * neq * steps / (total_ms * 1e-3) / 1e9


def algorithmic_bytes(neq, n_el, n_nodes):
    return 8 * neq + 8 * neq + 32 * n_el + 12 * n_nodes + 4 * n_el


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def load_traffic(variant, kz):
    """DRAM bytes per apply from the committed ncu summary of this kernel and workload, when the
    summary's launch shape (variant, kz) is the one timed; else None. Returns (bytes, source)."""
    p = os.path.join(ROOT, "profiles", "box_apply_layered128.json")
    if not os.path.exists(p):
        return None, "no ncu summary"
    d = json.load(open(p))
    shape = d.get("launch")
    if shape is not None and (int(shape[0]), int(shape[1])) != (int(variant), int(kz)):
        return None, f"ncu summary of launch {shape[0]},{shape[1]}; timed {variant},{kz}: not the same kernel"
    return d.get("dram_bytes_per_launch"), "ncu summary profiles/box_apply_layered128.json (" + d.get("source", "") + ")"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def start(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                           "-i", self.gpu, "-lms", "200"], stdout=subprocess.PIPE,
                                          stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self._proc = None

    def _read(self):
        for line in self._proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def stop(self):
        if self._proc:
            time.sleep(0.25)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=2)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 4 + i and s[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def mesh_builders():
    """The mesh generators (femorax_b200/meshes.py, plain numpy) loaded as a module of their own,
    without importing the package: importing femorax_b200 loads its library, and the reference arm
    maps no file of this library."""
    name = "femorax_mesh_builders"
    if name not in sys.modules:
        import importlib.util
        s = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "femorax_b200", "meshes.py"))
        m = importlib.util.module_from_spec(s)
        sys.modules[name] = m
        s.loader.exec_module(m)
    return sys.modules[name]


def bench_spec():
    return mesh_builders().layered_box(WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nz"], WORKLOAD["layers"],
                                       seed=WORKLOAD["seed"])[0]


def bench_config(neq, n_el, n_nodes, gpus):
    """The workload's `config`, the same dict in both arms."""
    return dict(WORKLOAD, neq=int(neq), elements=int(n_el), nodes=int(n_nodes), parallelism=f"replicas x{gpus}",
                l2="GPU arm: L2 flushed by a 256 MB write between timed applies; host arm: a 1 GB working set "
                   "(maps, geometry cache, slots), past every host cache")


def build_mesh():
    import femorax_b200 as fx
    spec = bench_spec()
    return spec, fx.Model(spec).compile(renumbering="rcm", simd_width=32)


def reference_force(spec):
    """The reference's own compile step and InternalForce (oracle/_ref, every host thread) on `spec`,
    or None where that library is missing."""
    import oracle as O
    if not O.have_ref():
        return None
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    c = O.RefModel(spec).compile(renumbering="rcm", simd_width=32)
    return O.RefForce(c, cache=True)


def grid_order_equations(spec, comp):
    """The free equations of the box's nodes in grid order (z planes, then y rows, then x, then the
    three components): the order in which the apply's tiles gather x."""
    eq = mesh_builders().equation_map(comp)[spec.tags]
    c = spec.coords
    key = [np.rint((c[:, d] - c[:, d].min()) * 1e6).astype(np.int64) for d in range(3)]
    order = np.lexsort((key[0], key[1], key[2]))
    e = eq[order].reshape(-1)
    return e[e >= 0].astype(np.int64)


def gather_floor(spec, comp, x, flush, stream, reps=20):
    """What one pass over x in the apply's access order costs on this device by itself: every free
    equation of the box gathered in grid order (torch.index_select, a library kernel used here as a
    measuring stick only, reading an 8-byte index per value), beside a contiguous copy of the same
    bytes; L2 flushed before each launch as for the timed applies."""
    import torch
    idx = torch.as_tensor(grid_order_equations(spec, comp), device=x.device)
    out = torch.empty(idx.numel(), dtype=x.dtype, device=x.device)
    res = {}
    for name, fn in (("rcm_gather_of_x", lambda: torch.index_select(x, 0, idx, out=out)),
                     ("contiguous_copy_of_x", lambda: out[: x.numel()].copy_(x))):
        for _ in range(3):
            fn()
        ev = []
        for i in range(reps):
            flush.fill_(float(i))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            ev.append((a, b))
        torch.cuda.synchronize(x.device)
        res[name + "_us"] = float(np.median([a.elapsed_time(b) for a, b in ev]) * 1e3)
    res["values"] = int(idx.numel())
    res["what"] = ("x alone, in the apply's gather order (grid order of the RCM-numbered equations) and contiguous; "
                   "library kernels, L2 flushed before each launch; index read 8 B per value")
    return res


def rel_err(a, b):
    """max |a - b| over max |b|."""
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


def cpu_reference_apply(rf, x, max_seconds=20.0, max_reps=5):
    """The reference's InternalForce::apply_operator (gather scatter, cached geometry, constant
    tangent) on the host, OpenMP over every host thread: GDoF/s over a bounded number of applies."""
    if rf is None:
        return None
    threads = os.cpu_count() or 1
    rf.apply_operator((1.0, 0.0, 0.0), x)  # warm-up (first touch of the cache and slots)
    times = []
    t_start = time.perf_counter()
    while len(times) < max_reps and (time.perf_counter() - t_start) < max_seconds:
        t0 = time.perf_counter()
        rf.apply_operator((1.0, 0.0, 0.0), x)
        times.append(time.perf_counter() - t0)
    best = min(times)
    return dict(value=rf.n / best / 1e9, unit="GDoF/s", cores=int(os.environ.get("OMP_NUM_THREADS", threads)),
                kind="reference",
                sample=f"{len(times)} applies of the full 128x128x64 layered box (min time {best * 1e3:.1f} ms) through "
                       "the reference's own InternalForce::apply_operator (gather scatter, geometry cache, constant "
                       "tangent), built from its sources with a serial/OpenMP Kokkos-subset shim")


def layered_parity(rf, force, x, y, device):
    """The timed apply's y on the layered box against the reference's apply_operator on the same x,
    and one FP64 internal force (seeded u, v; the box's alphaM and betaK damping) against the
    reference's InternalForce::compute: max |ours - reference| over max |reference|."""
    import torch
    dev = torch.device("cuda", device)
    y_ref = rf.apply_operator((1.0, 0.0, 0.0), x)
    rng = np.random.default_rng(11)
    u, v = 1e-3 * rng.standard_normal(rf.n), 1e-2 * rng.standard_normal(rf.n)
    f = torch.zeros(rf.n, dtype=torch.float64, device=dev)
    force.compute(torch.as_tensor(u, device=dev), torch.as_tensor(v, device=dev), f)
    torch.cuda.synchronize(dev)
    f_ref = rf.force(u, v)
    return {"apply_max_rel_err": rel_err(y.cpu().numpy(), y_ref),
            "force_max_rel_err": rel_err(f.cpu().numpy(), f_ref),
            "against": "the reference's own InternalForce (apply_operator, compute) built from its sources",
            "tolerance": 1e-12}


# The reference's own 40^3 laminar-column measurements on an H200 (GH200; reference
# benchmarks/baselines/tacc-vista-gh-cuda270336.json, min over 20 calls): its default variant, its
# fastest deterministic (gather) variant and its fastest variant overall, in microseconds.
H200_COLUMN_40 = {
    "operator": {"default": 242.3, "fastest_deterministic": 137.3, "fastest": 73.1,
                 "names": "operator/40^3/gather_cached_constant, gather_recompute_recomputed, "
                          "atomic_recompute_recomputed"},
    "explicit_force": {"default": 335.2, "fastest_deterministic": 173.3, "fastest": 103.3,
                       "names": "explicit_force/40^3/team_gather_ept4_cached, flat_gather, flat_atomic"},
    "operator_ssp": {"default": 142.0, "fastest_deterministic": 142.0, "fastest": 78.0,
                     "names": "operator_ssp/40^3/gather_cached_constant, gather_cached_constant, "
                              "atomic_cached_constant"},
}


def column_40(device, reps=50):
    """The reference's benchmark model, the 40^3 laminar soil column (tests/common/
    synthetic_models.hpp; 64,000 bricks, equalDOF ties, two Rayleigh regions), on the Gauss-point
    path, deterministic, in its exact form (the reference's own arithmetic order) and, for the
    stdBrick legs, its fast form (fx_force_set_general_mode): the stdBrick operator (consistent mass,
    K + 2e3 C + 1.6e7 M, as bench_operator.cpp), the explicit internal force (lumped, damped,
    u = 1e-4, v = 1e-3, as bench_explicit.cpp) and the SSPbrick operator.
    Per leg: min and median over `reps` calls by CUDA events (the reference's harness takes the min
    with the operands warm in cache), the median with L2 flushed before each call, and the result
    against the reference's own InternalForce (oracle/_ref) on the same inputs."""
    import torch
    import femorax_b200 as fx
    mb = mesh_builders()
    dev = torch.device("cuda", device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    out = {"mesh": "laminar column 40^3 (64,000 bricks)", "reference_h200_us": H200_COLUMN_40}
    legs = {"operator": (mb.laminar_column(40, 40, 40, lumped=False), "apply"),
            "explicit_force": (mb.laminar_column(40, 40, 40, lumped=True), "force"),
            "operator_ssp": (mb.laminar_column(40, 40, 40, element=1), "apply")}
    k = (1.0, 2e3, 1.6e7)
    for name, (spec, kind) in legs.items():
        mesh = fx.Model(spec).compile().mesh()
        force = fx.InternalForce(mesh, device=device)
        n = mesh.num_equations
        leg = {}
        for mode in (("exact", "fast") if name != "operator_ssp" else ("exact",)):
            force.set_general_mode(mode)
            leg[mode] = column_leg(force, kind, k, n, dev, flush, reps, spec)
        leg["equations"], leg["elements"], leg["path"] = n, mesh.count, force.info()["path"]
        best = min(leg[m]["us_min"] for m in leg if isinstance(leg[m], dict))
        leg["vs_h200_default"] = H200_COLUMN_40[name]["default"] / best
        leg["vs_h200_fastest"] = H200_COLUMN_40[name]["fastest"] / best
        out[name] = leg
    return out


def column_leg(force, kind, k, n, dev, flush, reps, spec):
    """One leg of column_40 in the force's current form: timings and the error against the
    reference's InternalForce (computed once per leg, cached across the forms)."""
    import torch
    import femorax_b200 as fx
    global _COLUMN_REF
    if kind == "apply":
        xn = np.full(n, 1e-3)
        x, y = torch.as_tensor(xn, device=dev), torch.zeros(n, dtype=torch.float64, device=dev)
        call = lambda: force.apply_operator(fx.OperatorCoefficients(*k), x, y)
    else:
        un, vn = np.full(n, 1e-4), np.full(n, 1e-3)
        u, v = torch.as_tensor(un, device=dev), torch.as_tensor(vn, device=dev)
        y = torch.zeros(n, dtype=torch.float64, device=dev)
        call = lambda: force.compute(u, v, y)
    for _ in range(5):
        call()
    hot, cold = [], []
    for flushed in (False, True):
        for i in range(reps):
            if flushed:
                flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            call()
            e1.record()
            torch.cuda.synchronize(dev)
            (cold if flushed else hot).append(e0.elapsed_time(e1) * 1e3)
    leg = {"us_min": float(np.min(hot)), "us_median": float(np.median(hot)),
           "us_median_l2_flushed": float(np.median(cold))}
    key = (id(spec), kind)
    if _COLUMN_REF.get("key") != key:
        rf = reference_force(spec)
        _COLUMN_REF = {"key": key, "want": None if rf is None else
                       (rf.apply_operator(k, xn) if kind == "apply" else rf.force(un, vn))}
    if _COLUMN_REF["want"] is not None:
        leg["max_rel_err_vs_reference"] = rel_err(y.cpu().numpy(), _COLUMN_REF["want"])
    return leg


_COLUMN_REF = {}


def static_c1(device, solves=10):
    """The static configuration as specified: a 32^3 stdBrick cube (1 m, E 50 MPa, nu 0.3, base fixed)
    under a 100 kPa downward top traction, Jacobi-PCG to a 1e-10 relative residual. Plain FP64 CG and
    FP32 CG inside FP64 refinement, solves/s by CUDA events over `solves` solves from x = 0 after one
    warm-up solve each; the FP64 solution against the reference's own ConjugateGradient (oracle/_ref,
    its host build) on the same compiled model, and each solution's true FP64 residual by the reference's
    operator."""
    import torch
    import femorax_b200 as fx
    mb = mesh_builders()
    spec = mb.static_cube(32)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh, device=device)
    neq = mesh.num_equations
    b = mb.top_traction_vector(spec, mb.equation_map(comp), neq)
    dev = torch.device("cuda", device)
    bt = torch.as_tensor(b, device=dev)
    out = {"mesh": f"cube 32^3, {neq} equations", "rtol": 1e-10, "solves": solves}
    xs = {}
    for name, cls in (("plain_fp64", fx.ConjugateGradient), ("mixed", fx.MixedPrecisionSolver)):
        s = cls(fx.SolveOptions(relative_tolerance=1e-10, max_iterations=20000))
        s.setup(fx.MatrixFreeOperator(force))
        x = torch.zeros(neq, dtype=torch.float64, device=dev)
        r = s.solve(bt, x)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lat = []
        for _ in range(solves):
            x.zero_()
            torch.cuda.synchronize(dev)
            e0.record()
            r = s.solve(bt, x)
            e1.record()
            torch.cuda.synchronize(dev)
            lat.append(e0.elapsed_time(e1) * 1e-3)
        xs[name] = x.cpu().numpy()
        out[name] = {"solves_per_s": solves / sum(lat), "p50_s": float(np.percentile(lat, 50)),
                     "p99_s": float(np.percentile(lat, 99)), "iterations": int(r.iterations),
                     "refinements": int(r.refinements), "converged": bool(r.converged)}
    out["mixed_speedup"] = out["mixed"]["solves_per_s"] / out["plain_fp64"]["solves_per_s"]
    rf = reference_force(spec)
    if rf is not None:
        x_ref, info = rf.solve(b, method="cg", rtol=1e-10, lanes=1)
        nb = float(np.linalg.norm(b))
        out["reference_cg_iterations"] = info["iterations"]
        out["plain_fp64_vs_reference_max_rel_err"] = rel_err(xs["plain_fp64"], x_ref)
        for name in xs:
            out[name]["true_relative_residual"] = float(np.linalg.norm(b - rf.apply_operator((1.0, 0.0, 0.0), xs[name])) / nb)
    return out


def explicit_comparison(force, mesh, comp, device, steps=4000):
    """The explicit wave configuration's time stepping on the bench mesh: ExplicitDifference steps
    (force + update, CUDA graphs of 16 steps) at dt = 0.5 dt_crit under a 5 Hz Ricker base
    acceleration, FP64 and FP32; steps/s by CUDA events around each run, and the FP32 surface-centre
    acceleration history against the FP64 one (max abs difference over the FP64 peak)."""
    import torch
    from femorax_b200 import meshes, serving
    nx, ny, nz = WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nz"]
    eqmap = serving.equation_map(comp)
    rec = int(eqmap[1 + nx // 2 + (nx + 1) * (ny // 2 + (ny + 1) * nz), 0])
    dt = 0.5 * force.min_critical_dt("ExplicitDifference")
    ag = meshes.ricker(np.arange(steps) * dt + dt, f0=5.0, amplitude=1.0)
    dev = torch.device("cuda", device)
    out = {"steps": steps, "dt_s": dt, "record": "surface-centre x acceleration"}
    hist = {}
    for name, dt_ in (("f64", torch.float64), ("f32", torch.float32)):
        n = mesh.num_equations
        mass = torch.as_tensor(mesh.lumped_mass, device=dev).to(dt_)
        u, vh, a, v = (torch.zeros(n, dtype=dt_, device=dev) for _ in range(4))
        force.explicit_run(mass, u, vh, a, v, dt, 32, ag=ag[:32], direction=0)  # warm-up (graphs, modules)
        u.zero_(), vh.zero_(), a.zero_(), v.zero_()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        hist[name] = force.explicit_run(mass, u, vh, a, v, dt, steps, ag=ag, direction=0, record_eq=rec)
        e1.record()
        torch.cuda.synchronize(dev)
        out[f"steps_per_s_{name}"] = steps / (e0.elapsed_time(e1) * 1e-3)
    peak = float(np.max(np.abs(hist["f64"])))
    out["f32_history_max_abs_diff_over_peak"] = float(np.max(np.abs(hist["f32"] - hist["f64"]))) / peak
    return out


PDMY_SAND = (2.0285423037716614, 145000.0, 314166.66666666663, 40.0, 0.1, 80.0, 0.5, 27.0, 0.03, 0.8, 5.0, 0.0, 0.0,
             0.0, 20.0, 0.45, 0.9, 0.02, 0.7, 101.0, 0.3, 0.0, 1.0)  # dense sand of the stored paths


def pdmy_force_box(device, n=40, evals=20):
    """The reference's PressureDependMultiYield force measurement (the internal force of an n^3
    stdBrick box of dense sand, 20 surfaces, in the plastic stage; 7.85 ms at 40^3 on an H200,
    reference benchmarks/baselines/tacc-vista-gh-cuda270336.json:769, explicit_force_pdmy/40^3/plastic):
    the box is confined (a uniform 2e-4 volumetric strain, elastic
    stage, committed), switched to the plastic stage and sheared (committed), then `evals` force
    evaluations at further shear strains (each every point's update from the committed state and the
    element forces), timed by CUDA events."""
    import torch
    import femorax_b200 as fx
    from femorax_b200 import meshes
    G, K = PDMY_SAND[1], PDMY_SAND[2]
    E, nu = 9 * K * G / (3 * K + G), (3 * K - 2 * G) / (2 * (3 * K + G))
    spec = meshes.box_model(n, n, n, size=(float(n), float(n), float(n)), E=E, nu=nu, rho=PDMY_SAND[0], lumped=True)
    mesh = fx.Model(spec).compile().mesh()
    force = fx.InternalForce(mesh, device=device)
    m = fx.PressureDependMultiYield(*PDMY_SAND[:14], noYieldSurf=int(PDMY_SAND[14]), e=PDMY_SAND[15],
                                    cs1=PDMY_SAND[16], cs2=PDMY_SAND[17], cs3=PDMY_SAND[18], pa=PDMY_SAND[19],
                                    c=PDMY_SAND[20])
    force.set_pdmy(0, m)
    dev = torch.device("cuda", device)
    neq, P = mesh.num_equations, mesh.padded
    node, eq, X = mesh.node.reshape(8, P), mesh.eq.reshape(24, P), mesh.coords.reshape(3, -1)
    xq, zq, dof = np.zeros(neq), np.zeros(neq), np.full(neq, -1)
    for a in range(8):
        for d in range(3):
            q = eq[3 * a + d, :mesh.count]
            ok = q >= 0
            xq[q[ok]], zq[q[ok]] = X[0, node[a, :mesh.count][ok]], X[2, node[a, :mesh.count][ok]]
            dof[q[ok]] = d
    conf = np.where(dof == 2, -2e-4 / 3 * zq, 0.0) + np.where(dof == 0, -2e-4 / 3 * xq, 0.0)
    v = torch.zeros(neq, dtype=torch.float64, device=dev)
    f = torch.zeros(neq, dtype=torch.float64, device=dev)

    def u_at(gam):
        return torch.as_tensor(conf + np.where(dof == 0, gam * zq, 0.0), device=dev)

    force.compute(u_at(0.0), v, f)
    force.commit_state()
    force.set_material_stage(0, 1)
    force.compute(u_at(2e-4), v, f)
    force.commit_state()
    us = [u_at(2e-4 + 1e-4 * np.sin(0.3 * k)) for k in range(evals + 3)]
    out = {"elements": int(mesh.count), "points": 8 * int(mesh.count), "reference_h200_ms": 7.85}
    results = {}
    for corrector in ("fused", "compacted"):  # every evaluation from the same committed state
        force.set_soil_corrector(corrector)
        for k in range(3):
            force.compute(us[k], v, f)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(evals):
            force.compute(us[3 + k], v, f)
        e1.record()
        torch.cuda.synchronize(dev)
        results[corrector] = f.cpu().numpy()
        key = "ms_per_force" if corrector == "fused" else "compacted_ms_per_force"
        out[key] = e0.elapsed_time(e1) / evals
    out["compacted_bit_identical"] = bool(np.array_equal(results["fused"], results["compacted"]))
    out["plastic_points"] = int(force.plastic_points())
    out["failed_points"] = int(force.pimy_failed())
    return out


def pdmy_points(device, n=1 << 20, steps=10, sample=4096, seed=0):
    """PressureDependMultiYield material points (fx_pdmy_update): a dense sand (20 surfaces, friction
    angle 40, phase transformation 27 degrees, dilatancy), otherwise as pimy_points."""
    import femorax_b200 as fx
    m = fx.PressureDependMultiYield(2.03, 145000, 314167, 40, 0.1, 80, 0.5, 27, 0.03, 0.8, 5, 0, 0, 0,
                                    noYieldSurf=20, e=0.45)
    return pimy_points(device, n, steps, sample, seed, material=m, amplitude=5e-3)


def pimy_points(device, n=1 << 20, steps=10, sample=8192, seed=0, material=None, amplitude=2e-2):
    """PressureIndependMultiYield material points (fx_pimy_update): n points of a frictional sand
    (20 surfaces, friction angle 30 degrees, pressure-dependent moduli) on seeded strain paths,
    switched to the plastic stage under confinement, then `steps` cyclic-shear updates with the
    tangent, timed by CUDA events on the launching stream. Point-updates/s and the HBM traffic one
    update needs (committed and trial state, strain, stress, tangent); the host restatement of the
    same arithmetic on `sample` points on one core beside it."""
    import torch
    import femorax_b200 as fx
    m = material or fx.PressureIndependMultiYield(2.0, 60000, 150000, 5, 0.1, 30, 80, 0.5, 20)
    dev = torch.device("cuda", device)
    rng = np.random.default_rng(seed)
    amp = torch.as_tensor(rng.uniform(2e-4, amplitude, n), device=dev)
    dirs = torch.as_tensor(rng.standard_normal((3, n)), device=dev)
    dirs /= dirs.norm(dim=0)
    conf = torch.as_tensor(rng.uniform(-2e-3, -5e-4, n), device=dev)
    c, t = m.initial_state(n, device), torch.empty((m.nstate, n), dtype=torch.float64, device=dev)
    sig = torch.empty((6, n), dtype=torch.float64, device=dev)
    tan = torch.empty((36, n), dtype=torch.float64, device=dev)
    failed = torch.zeros(1, dtype=torch.int32, device=dev)

    def strain(k):
        e = torch.zeros((6, n), dtype=torch.float64, device=dev)
        e[0:3] = conf / 3
        e[3:6] = amp * float(np.sin(2 * np.pi * k / steps)) * dirs
        return e.contiguous()

    eps = [strain(k) for k in range(steps + 1)]
    m.update(0, c, t, eps[0], sig, tan, failed)  # confinement, elastic stage
    c, t = t, c
    m.update(1, c, t, eps[0], sig, tan, failed)  # the switch to the plastic stage
    c, t = t, c
    stream = torch.cuda.current_stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize(dev)
    ev[0].record(stream)
    for k in range(1, steps + 1):
        m.update(1, c, t, eps[k], sig, tan, failed, stream)
        c, t = t, c
    ev[1].record(stream)
    torch.cuda.synchronize(dev)
    ms = ev[0].elapsed_time(ev[1])
    per_point = 2 * m.nstate * 8 + 6 * 8 + 6 * 8 + 36 * 8
    # host: the same arithmetic on a sample of the same points, one core
    hs = slice(0, sample)
    hc, ht = m.initial_state(sample), np.zeros((m.nstate, sample))
    hsig, htan = np.zeros((6, sample)), np.zeros((36, sample))
    heps = [np.ascontiguousarray(e[:, hs].cpu().numpy()) for e in eps]
    m.update_host(0, hc, ht, heps[0], hsig, htan)
    hc, ht = ht, hc
    m.update_host(1, hc, ht, heps[0], hsig, htan)
    hc, ht = ht, hc
    t0 = time.perf_counter()
    for k in range(1, steps + 1):
        m.update_host(1, hc, ht, heps[k], hsig, htan)
        hc, ht = ht, hc
    host_s = time.perf_counter() - t0
    dsig = sig[:, hs].cpu().numpy()
    rel = np.max(np.abs(dsig - hsig), axis=0) / float(np.max(np.abs(hsig)))
    rate = n * steps / (ms * 1e-3)
    return {"points": n, "surfaces": m.surfaces, "steps": steps, "ms_per_update": ms / steps,
            "point_updates_per_s": rate, "bytes_per_point_update": per_point,
            "achieved_gbs": rate * per_point / 1e9, "failed_points": int(failed.item()),
            "host_one_core_point_updates_per_s": sample * steps / host_s, "host_sample_points": sample,
            "device_vs_host_sample": {
                "bit_identical": float(np.mean(rel == 0)), "within_1e-12": float(np.mean(rel <= 1e-12)),
                "host": "this library's host restatement with the host C library's elementary functions (the "
                        "device's pow/exp/log/cos are its own, or CUDA's for PressureIndependMultiYield): points on "
                        "another branch after a last-place difference count against both fractions"}}


PIMY_CLAY = (1.8, 40500.0, 108000.0, 8.0, 0.1, 0.0, 100.0, 0.0, 20.0)  # rho t/m3, G, K kPa, cohesion kPa, ...


def pimy_explicit(device, n=100, warm=16, steps=64):
    """pimy_explicit_run with the fused point pass and with the compacted plastic corrector; the two
    runs' final displacements compared bit for bit."""
    fused = pimy_explicit_run(device, n, warm, steps, "fused")
    comp = pimy_explicit_run(device, n, warm, steps, "compacted")
    u_f, u_c = fused.pop("_u"), comp.pop("_u")
    fused["compacted"] = comp
    fused["compacted_bit_identical"] = bool(np.array_equal(u_f, u_c))
    return fused


def pimy_explicit_run(device, n=100, warm=16, steps=64, corrector="fused"):
    """The reference's plastic-box measurement (an n^3 stdBrick box of PressureIndependMultiYield
    clay, 20 surfaces, in the plastic stage, under 0.3 g 2 Hz base shaking, explicit steps of 5e-4 s)
    on the Gauss-point path: ExplicitDifference stage steps (the force with every point's material
    update, the update pass, the commit of the material state), CUDA graphs of 16 steps; ms per
    step by CUDA events after `warm` steps. 1 m elements, fixed base, lumped mass, no laminar ties
    (the reference's generator is not in its repository)."""
    import torch
    import femorax_b200 as fx
    from femorax_b200 import meshes
    G, K = PIMY_CLAY[1], PIMY_CLAY[2]
    E, nu = 9 * K * G / (3 * K + G), (3 * K - 2 * G) / (2 * (3 * K + G))
    spec = meshes.box_model(n, n, n, size=(float(n), float(n), float(n)), E=E, nu=nu, rho=PIMY_CLAY[0], lumped=True)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh, device=device)
    force.set_pimy(0, fx.PressureIndependMultiYield(*PIMY_CLAY[:8], noYieldSurf=int(PIMY_CLAY[8])))
    force.set_material_stage(0, 1)
    force.set_soil_corrector(corrector)
    dev = torch.device("cuda", device)
    dt = 5e-4
    total = warm + steps
    t = np.arange(total + 2) * dt
    motions = fx.GroundMotions([dict(dof=0, fact=1.0, values=0.3 * 9.81 * np.sin(2 * np.pi * 2.0 * t), dt=dt)])
    m = torch.as_tensor(mesh.lumped_mass, device=dev)
    u, v, a = (torch.zeros(mesh.num_equations, dtype=torch.float64, device=dev) for _ in range(3))
    tm, _ = force.explicit_stage("ExplicitDifference", m, u, v, a, dt, warm, motions=motions)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    force.explicit_stage("ExplicitDifference", m, u, v, a, dt, steps, time=tm, motions=motions, resume=True)
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    return {"elements": int(mesh.count), "points": 8 * int(mesh.count), "surfaces": int(PIMY_CLAY[8]),
            "dt_s": dt, "steps_timed": steps, "ms_per_step": ms, "device_bytes": int(force.info()["device_bytes"]),
            "plastic_points_last_step": int(force.plastic_points()), "failed_points": int(force.pimy_failed()),
            "reference_h200_ms_per_step": 23.5, "corrector": corrector, "_u": u.cpu().numpy()}


def newmark_comparison(device, n=100, steps=200, seed=0):
    """The Newmark configuration at its 200 steps: a heterogeneous cube of n^3 boxes (per-element
    E log-normal, median 80 MPa, sigma 0.5; nu 0.3; base fixed), a harmonic horizontal surface load,
    Newmark beta 0.25 gamma 0.5 with one inner solve per step to a 1e-8 relative FP64 residual:
    plain FP64 CG against FP32 CG inside FP64 refinement. Steps/s by wall clock around each run
    (after a 2-step warm-up of each); the monitored top displacement histories compared."""
    import math

    import torch
    import femorax_b200 as fx
    from femorax_b200 import meshes, serving, stages
    spec = meshes.heterogeneous_cube(n, seed=seed, size=0.5 * n)
    comp = fx.Model(spec).compile()
    mesh = comp.mesh()
    force = fx.InternalForce(mesh, device=device)
    f, mon = stages.top_shear(spec, serving.equation_map(comp), 1e6)
    ft = torch.as_tensor(f, device=torch.device("cuda", device))

    def load(t):
        return ft * math.sin(2 * math.pi * 5.0 * t)

    out = {"mesh": f"heterogeneous cube {n}^3, {mesh.num_equations} equations", "steps": steps, "dt_s": 2e-3}
    runs = {}
    for mixed in (False, True):
        stages.newmark_run(force, load, 2, 2e-3, mon, mixed=mixed, rtol=1e-8)
        runs[mixed] = stages.newmark_run(force, load, steps, 2e-3, mon, mixed=mixed, rtol=1e-8)
    out["plain_fp64_steps_per_s"] = steps / runs[False].seconds
    out["mixed_steps_per_s"] = steps / runs[True].seconds
    out["speedup"] = runs[False].seconds / runs[True].seconds
    peak = float(np.max(np.abs(runs[False].monitor)))
    out["mixed_vs_plain_max_abs_diff_over_peak"] = float(np.max(np.abs(runs[True].monitor - runs[False].monitor))) / peak
    out["converged"] = bool(runs[False].converged and runs[True].converged)
    # one FP64 apply of the cube's operator (per-element E) against the reference's apply_operator
    rf = reference_force(spec)
    if rf is not None:
        dev = torch.device("cuda", device)
        xr = np.random.default_rng(5).standard_normal(mesh.num_equations)
        y = torch.zeros(mesh.num_equations, dtype=torch.float64, device=dev)
        force.apply_operator(fx.OperatorCoefficients(1.0, 0.0, 0.0), torch.as_tensor(xr, device=dev), y)
        torch.cuda.synchronize(dev)
        out["apply_parity"] = {"apply_max_rel_err": rel_err(y.cpu().numpy(), rf.apply_operator((1.0, 0.0, 0.0), xr)),
                               "against": "the reference's own InternalForce::apply_operator", "tolerance": 1e-12}
    return out


def batched_j2_comparison(device, count=32, steps=8, seed=1):
    """The batched J2 configuration on a bounded sample: `count` seeded J2 columns and blocks
    (nx = ny in {1, 2, 4, 8}, nz in [20, 40]) on one cyclic top-shear cycle of `steps` load steps
    (load-controlled, 1.2 x the first-yield bending load), Newton to ||r|| <= 1e-6 N per step
    with Jacobi-PCG to 1e-12: the batched Newton (one combined mesh, per-instance Newton and CG on
    the device) against the same instances solved one at a time by the single-instance path, and
    the batch with FP32 CG inside FP64 refinement (the FP32 operator on the point tangents); then
    both batched forms with the linear solves at 1e-8, histories compared with the 1e-12 batch.
    Instance-steps/s by wall clock around each arm; the batched and one-at-a-time histories are
    compared bit for bit."""
    import torch
    import femorax_b200 as fx
    from femorax_b200 import serving, stages
    inst = stages.j2_instances(count, seed=seed, sizes=(1, 2, 4, 8), nz_range=(20, 40))
    meshes, fs, mons = [], [], []
    for spec, total in inst:
        comp = fx.Model(spec).compile()
        f, mon = stages.top_shear(spec, serving.equation_map(comp), total)
        meshes.append(comp.mesh())
        fs.append(f)
        mons.append(mon)
    factors = stages.cyclic_factors(1, steps)
    stages.batched_load_path(meshes[:2], fs[:2], factors[:1], mons[:2], device=device)  # warm-up
    b = stages.batched_load_path(meshes, fs, factors, mons, device=device)
    forces = [fx.InternalForce(m, device=device) for m in meshes]
    dev = torch.device("cuda", device)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    single = [stages.load_path(forces[i], torch.as_tensor(fs[i], device=dev), factors, mons[i])
              for i in range(count)]
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    same = all(np.array_equal(b.monitor[:, i], single[i].monitor) for i in range(count))
    # the same batch with FP32 CG inside FP64 refinement (FP32 apply, FP64 return map)
    stages.batched_load_path(meshes[:2], fs[:2], factors[:1], mons[:2], device=device, mixed=True)  # warm-up
    bm = stages.batched_load_path(meshes, fs, factors, mons, device=device, mixed=True)
    peak = float(np.max(np.abs(b.monitor)))
    # both batched forms with the linear solves at 1e-8 (the Newton test is unchanged)
    loose = {}
    for mixed in (False, True):
        stages.batched_load_path(meshes[:2], fs[:2], factors[:1], mons[:2], cg_rtol=1e-8, device=device, mixed=mixed)
        run = stages.batched_load_path(meshes, fs, factors, mons, cg_rtol=1e-8, device=device, mixed=mixed)
        key = "mixed" if mixed else "plain"
        loose[key + "_instance_steps_per_s"] = count * len(factors) / run.seconds
        loose[key + "_newton_solves"] = int(run.newton.sum())
        loose[key + "_max_abs_diff_over_peak"] = float(np.max(np.abs(run.monitor - b.monitor))) / peak
        if mixed:
            loose["mixed_refinements_per_linear_solve"] = float(run.refinements.sum() / max(1, run.newton.sum()))
        loose[key + "_converged"] = bool(run.converged)
    return {"instances": count, "elements": int(sum(m.count for m in meshes)),
            "mixed_batched_instance_steps_per_s": count * len(factors) / bm.seconds,
            "mixed_refinements_per_linear_solve": float(bm.refinements.sum() / max(1, bm.newton.sum())),
            "mixed_converged": bool(bm.converged),
            "mixed_vs_plain_max_abs_diff_over_peak": float(np.max(np.abs(bm.monitor - b.monitor))) / peak,
            "linear_rtol_1e-8": loose,
            "equations": int(sum(m.num_equations for m in meshes)), "load_steps": len(factors),
            "batched_instance_steps_per_s": count * len(factors) / b.seconds,
            "one_at_a_time_instance_steps_per_s": count * len(factors) / secs,
            "speedup": secs / b.seconds, "newton_solves_per_step_mean": float(b.newton.mean()),
            "converged": bool(b.converged and all(r.converged for r in single)), "bit_identical": bool(same)}


def batched_j2_path(device, count=32, steps=8, seed=1):
    """The batched arm of batched_j2_comparison alone (profiling): the same `count` seeded J2
    instances on one cyclic cycle of `steps` load steps, Newton to ||r|| <= 1e-6 N, Jacobi-PCG to
    1e-12; seconds by wall clock, Newton solves and CG iterations per instance and step."""
    import torch
    import femorax_b200 as fx
    from femorax_b200 import serving, stages
    inst = stages.j2_instances(count, seed=seed, sizes=(1, 2, 4, 8), nz_range=(20, 40))
    meshes, fs = [], []
    for spec, total in inst:
        comp = fx.Model(spec).compile()
        f, _ = stages.top_shear(spec, serving.equation_map(comp), total)
        meshes.append(comp.mesh())
        fs.append(f)
    b = fx.BatchedNewton(meshes, fx.SolveOptions(relative_tolerance=1e-12, max_iterations=20000), device)
    dev = torch.device("cuda", device)
    F = torch.as_tensor(b.combine(fs), device=dev)
    u = torch.zeros(b.total, dtype=torch.float64, device=dev)
    newton, cg = [], []
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for lam in stages.cyclic_factors(1, steps):
        it, res = b.step(F * float(lam), u, tol=1e-6, max_newton=25)
        b.commit_state()
        newton.append([int(v) for v in it])
        cg.append([int(r.iterations) for r in res])
    torch.cuda.synchronize(dev)
    return {"instances": count, "load_steps": steps, "seconds": time.perf_counter() - t0, "newton": newton,
            "cg_iterations": cg}


def served_streams(device, count=1000, rates=((10.0, 40), (100.0, 400), (500.0, 400), (2000.0, 1000)), seed=3,
                   models=32, j2_models=12):
    """The served configuration at its sizes, on resident models (serving.pooled_stream: `models`
    elastic blocks log-uniform in 1e4 - 2e6 equations, `j2_models` J2 blocks as the batched J2
    sample's, every request its own load), each stream through three arms:
      - mixed_batched: the serving loop (in C++, serving.NativeServer over fx_server_*) over the
        batched engine, FP32 inner solves inside FP64 refinement (the served form);
      - fp64_batched: the same loop and engine with FP64 inner solves (batching without reduced
        precision: the ablation that splits the speed-up into batching and precision);
      - plain_fp64_one_at_a_time: first come first served, each request alone by the plain FP64 path.
    Static solves end at a 1e-8 relative FP64 residual; J2 requests run one cyclic top-shear cycle
    of 8 load steps (Newton to 1e-6 N) in cohorts beside them. Streams: `count` static solves all
    at t = 0 ("served"), `count` mixed requests (70 % static, 30 % J2) all at t = 0
    ("served_mixed", the J2 results of the batched and one-at-a-time arms compared bit for bit),
    and the mixed stream with Poisson arrivals at each (rate, requests) of `rates` in real time
    ("served_rates"). Before timing, one request of every model goes through every arm (the
    models' resident state, module loading, each model's first solve). Latency runs from arrival to
    the result on the host; solves/s is requests over the arm's wall time, arrival window included."""
    import femorax_b200 as fx
    from femorax_b200 import serving
    opts = fx.SolveOptions(relative_tolerance=1e-8)
    engines = {"mixed_batched": fx.BatchEngine(1 << 26, 256, options=opts, device=device),
               "fp64_batched": fx.BatchEngine(1 << 26, 256, options=opts, inner_tolerance=0.5e-8, inner="fp64",
                                              device=device)}
    cache = {}

    def arms(reqs, realtime):
        prepared, solvers, host = serving.resident(reqs, device, j2_host=True, cache=cache)
        prep = {r.id: host[r.id] if isinstance(r, serving.J2Request) else prepared[r.id] for r in reqs}
        out = {}
        for name, eng in engines.items():
            srv = serving.NativeServer(eng, device=device, prepare_fn=lambda r, d: prep[r.id])
            out[name] = srv.run(reqs, realtime=realtime)
        out["plain_fp64_one_at_a_time"] = serving.serve_one_at_a_time(reqs, 1e-8, realtime=realtime, device=device,
                                                                      prepared=prepared, solvers=solvers)
        return out

    def report(runs, reqs):
        rep = {}
        for name, (served, wall) in runs.items():
            m = serving.summary(served, wall)
            rep[name] = {k: m[k] for k in ("solves_per_s", "p50_s", "p99_s", "converged", "wall_s", "j2_p50_s",
                                           "j2_p99_s") if k in m}
        plain = rep["plain_fp64_one_at_a_time"]["solves_per_s"]
        for name in engines:
            rep[name]["speedup_solves_per_s"] = rep[name]["solves_per_s"] / plain if plain else None
        rep["requests"] = len(reqs)
        rep["j2_requests"] = sum(isinstance(r, serving.J2Request) for r in reqs)
        rep["equations"] = int(sum(r.equations for r in reqs))
        return rep

    t_prep = time.perf_counter()

    def stream(n, rate, j2_share=0.3, s=seed):
        return serving.pooled_stream(n, rate, models=models, j2_models=j2_models, j2_share=j2_share, seed=s)

    # untimed: one request of every model through every arm
    firsts = {}
    for r in stream(40 * (models + j2_models), 1e9, s=seed):
        firsts.setdefault(serving.model_key(r), r)
    warm = sorted(firsts.values(), key=lambda r: r.id)
    arms(warm, False)
    static = stream(count, 1e9, j2_share=0.0)
    out = {"models": f"{models} elastic blocks (log-uniform 1e4-2e6 equations, E U[50,200] MPa, nu U[0.25,0.40]) and "
                     f"{j2_models} J2 blocks (nx = ny in {{1,2,4,8}}, nz in [20,40], sigma_y U[50,200] kPa, one cycle of "
                     f"8 load steps) resident on the device ({len(warm)} of them in use); each request its own load "
                     f"(static: top traction q U[-150,-50] kPa)",
           "preparation_s": time.perf_counter() - t_prep}
    out["served"] = report(arms(static, False), static)
    mixed = stream(count, 1e9, s=seed + 1)
    runs = arms(mixed, False)
    out["served_mixed"] = report(runs, mixed)
    pm = {x.id: x for x in runs["mixed_batched"][0]}
    pp = {x.id: x for x in runs["plain_fp64_one_at_a_time"][0]}
    j2 = [r.id for r in mixed if isinstance(r, serving.J2Request)]
    out["served_mixed"]["j2_bit_identical"] = bool(all(
        np.array_equal(pm[i].x, pp[i].x) and np.array_equal(pm[i].result.monitor, pp[i].result.monitor) for i in j2))
    rates_out = []
    for i, (rate, n) in enumerate(rates):
        reqs = stream(n, rate, s=seed + 2 + i)
        r = report(arms(reqs, True), reqs)
        r["rate_per_s"] = rate
        rates_out.append(r)
    out["served_rates"] = rates_out
    out["seconds"] = time.perf_counter() - t_prep
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle as O
    if not O.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfxref.so (the reference built from "
                                                               "its sources) is missing"}))
        return 0
    spec = bench_spec()
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    rf = reference_force(spec)
    c = rf.c
    x = np.random.default_rng(0).standard_normal(c.num_equations)
    for _ in range(args.warmup):
        rf.apply_operator((1.0, 0.0, 0.0), x)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rf.apply_operator((1.0, 0.0, 0.0), x)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = c.num_equations * args.steps / total / 1e9
    cores = int(os.environ.get("OMP_NUM_THREADS", threads))
    n_nodes = len(c.array("node_tag"))
    line = {"metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded layer properties)",
            "config": bench_config(c.num_equations, c.count, n_nodes, args.gpus),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "GDoF/s", "cores": cores, "kind": "reference",
                             "sample": f"{args.steps} applies of the full workload, each one step, through the "
                                       "reference's own InternalForce::apply_operator on every host thread"},
            "e2e": {"value": value, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import ctypes as fx_ctypes

    import torch
    import femorax_b200 as fx
    from femorax_b200._lib import check as fx_check, lib as fx_lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    spec, comp = build_mesh()
    mesh = comp.mesh()
    if args.launch:  # pinned before the force is created: no tuning launches
        os.environ["FEMORAX_B200_BOX_LAUNCH"] = args.launch
    force = fx.InternalForce(mesh, device=local)
    if args.launch:
        os.environ.pop("FEMORAX_B200_BOX_LAUNCH")
    launch = (fx_ctypes.c_int32 * 2)()
    fx_check(fx_lib().fx_force_get_launch(force._h, launch))
    shapes = (fx_ctypes.c_int32 * 8)()
    fx_check(fx_lib().fx_force_get_launches(force._h, shapes))
    tuned = {name: [int(shapes[2 * i]), int(shapes[2 * i + 1])]
             for i, name in enumerate(("f64_apply", "f64_force", "f32_apply", "f32_force"))}
    info = force.info()
    neq, n_el, n_nodes = mesh.num_equations, mesh.count, mesh.num_nodes
    dev = torch.device("cuda", local)
    k = fx.OperatorCoefficients(1.0, 0.0, 0.0)
    x = torch.as_tensor(np.random.default_rng(rank).standard_normal(neq), device=dev)
    y = torch.zeros(neq, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    for _ in range(max(args.warmup, 3)):
        force.apply_operator(k, x, y, stream)
    torch.cuda.synchronize(dev)

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    for i in range(args.steps):
        flush.fill_(float(i))  # 256 MB write: L2 (126 MB) holds nothing of the last apply
        starts[i].record(stream)
        force.apply_operator(k, x, y, stream)
        ends[i].record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.stop()
    ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(ms)
    total_ms = max_over_ranks([total_ms], dist, dev)[0]
    value = replica_value(world, neq, args.steps, total_ms)

    floor = gather_floor(spec, comp, x, flush, stream) if world == 1 else None
    # the FP32 apply (the precision form) on the same x, timed the same way, outside the FP64 figures
    x32 = x.float()
    y32 = torch.zeros(neq, dtype=torch.float32, device=dev)
    for _ in range(3):
        force.apply_operator(k, x32, y32, stream)
    f32_ms = []
    for i in range(args.steps):
        flush.fill_(float(i))
        a32, b32 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a32.record(stream)
        force.apply_operator(k, x32, y32, stream)
        b32.record(stream)
        f32_ms.append((a32, b32))
    torch.cuda.synchronize(dev)
    f32_ms = [a32.elapsed_time(b32) for a32, b32 in f32_ms]
    f32_err = float(((y32.double() - y).abs().max() / y.abs().max()).item())
    del x32, y32

    # e2e: the public host-buffer call, copies included
    xh = torch.empty(neq, dtype=torch.float64, pin_memory=True)
    xh.copy_(x.cpu())
    yh = torch.empty(neq, dtype=torch.float64, pin_memory=True)
    xn, yn = xh.numpy(), yh.numpy()
    force.apply_operator_host(k, xn, yn, stream)
    e_ms = []
    for i in range(args.steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        force.apply_operator_host(k, xn, yn, stream)
        e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = replica_value(world, neq, args.steps, max_over_ranks([sum(e_ms)], dist, dev)[0])

    peak, peak_kind = load_peaks()
    alg = algorithmic_bytes(neq, n_el, n_nodes)
    achieved = alg / (total_ms / args.steps * 1e-3) / 1e9
    traffic, traffic_source = load_traffic(launch[0], launch[1])
    alg32 = alg - 8 * neq  # x read and y written as 4-byte values
    ach32 = alg32 / (float(np.mean(f32_ms)) * 1e-3) / 1e9
    f32 = {"ms_per_apply": float(np.mean(f32_ms)), "gdof_per_s": neq / (float(np.mean(f32_ms)) * 1e-3) / 1e9,
           "achieved_gbs": ach32, "frac": ach32 / peak, "algorithmic_bytes_per_launch": alg32,
           "max_rel_err_vs_fp64": f32_err}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    explicit = explicit_comparison(force, mesh, comp, local) if world == 1 and not args.no_serve else None
    streams = served_streams(local) if world == 1 and not args.no_serve else None
    batched_j2 = batched_j2_comparison(local) if world == 1 and not args.no_serve else None
    newmark = newmark_comparison(local) if world == 1 and not args.no_serve else None
    pimy = pimy_points(local) if world == 1 and not args.no_serve else None
    if pimy is not None:
        pimy["explicit_box"] = pimy_explicit(local)
    pdmy = pdmy_points(local) if world == 1 and not args.no_serve else None
    if pdmy is not None:
        pdmy["force_box"] = pdmy_force_box(local)
    rf = reference_force(spec) if world == 1 else None
    xn0 = x.cpu().numpy()
    parity = layered_parity(rf, force, xn0, y, local) if rf is not None else None
    cpu = cpu_reference_apply(rf, xn0) if rf is not None and not args.no_cpu else None
    del rf
    static = static_c1(local) if world == 1 and not args.no_serve else None
    column = column_40(local) if world == 1 and not args.no_serve else None
    line = {"metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded layer properties)",
            "config": bench_config(neq, n_el, n_nodes, world),
            "path": info["path"],
            "launch": {"variant": int(launch[0]), "kz": int(launch[1]),
                       "chosen_by": "option" if args.launch else "autotuner", "all": tuned},
            "parity": parity,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": traffic_source, "peak_source": f"{peak_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": alg},
            "fp32_apply": f32,
            "gather_floor": floor,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "GDoF/s", "h2d_bytes_per_step": 8 * neq, "d2h_bytes_per_step": 8 * neq,
                    "ms_per_step": float(np.mean(e_ms)), "ms_per_step_min": float(np.min(e_ms)),
                    "ms_per_step_median": float(np.median(e_ms)),
                    "copies": "page-locked x in and y out in 8 equation ranges, overlapped with the tiles "
                              "that read the arrived ranges (fx_apply_operator_host)"},
            "gpu_launches": args.steps,
            "clocks": clocks.summary(),
            "explicit": explicit,
            "static_c1": static,
            "column_40": column,
            "batched_j2": batched_j2,
            "newmark": newmark,
            "pimy": pimy,
            "pdmy": pdmy}
    # the served figures last, so that they stay in view at the end of the line
    if streams is not None:
        line["served_models"] = streams["models"]
        line["served_seconds"] = streams["seconds"]
        line["served_preparation_s"] = streams["preparation_s"]
        line["served_rates"] = streams["served_rates"]
        line["served_mixed"] = streams["served_mixed"]
        line["served"] = streams["served"]
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-serve", action="store_true",
                    help="skip the explicit-stepping and served-versus-plain solve comparisons")
    ap.add_argument("--launch", default="", help="pin the box launch shape 'variant,kz' (profiling)")
    ap.add_argument("--batched-j2", action="store_true",
                    help="only the batched J2 path (32 instances, one cycle of 8 load steps; profiling)")
    ap.add_argument("--pimy-box", type=int, default=0,
                    help="only the PressureIndependMultiYield plastic box section, n^3 elements (profiling)")
    ap.add_argument("--served", type=int, default=0,
                    help="only the served streams, this many requests per stream (profiling)")
    ap.add_argument("--column", action="store_true",
                    help="only the 40^3 laminar-column legs (the reference's benchmark model)")
    ap.add_argument("--pdmy-box", type=int, default=0,
                    help="only the PressureDependMultiYield plastic force section, n^3 elements (profiling)")
    args = ap.parse_args()
    if args.served:
        n = args.served
        print(json.dumps(served_streams(int(os.environ.get("LOCAL_RANK", "0")), count=n,
                                        rates=((10.0, max(10, n // 16)), (100.0, max(10, 2 * n // 5)),
                                               (500.0, max(10, 2 * n // 5)), (2000.0, n)))))
        return 0
    if args.column:
        print(json.dumps(column_40(int(os.environ.get("LOCAL_RANK", "0")), reps=args.steps)))
        return 0
    if args.pdmy_box:
        print(json.dumps(pdmy_force_box(int(os.environ.get("LOCAL_RANK", "0")), n=args.pdmy_box, evals=args.steps)))
        return 0
    if args.batched_j2:
        print(json.dumps(batched_j2_path(int(os.environ.get("LOCAL_RANK", "0")))))
        return 0
    if args.pimy_box:
        print(json.dumps(pimy_explicit(int(os.environ.get("LOCAL_RANK", "0")), n=args.pimy_box, warm=args.warmup,
                                       steps=args.steps)))
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
