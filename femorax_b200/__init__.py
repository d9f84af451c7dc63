"""femorax_b200: a B200-native matrix-free hex8 hot path with the reference's element, operator and
solver interface (amnp95/FemoraX: exec::InternalForce, exec::MatrixFreeOperator,
solvers::LinearSolver, solvers::VectorOps), implemented in C++/CUDA behind the C ABI of
include/femorax_b200.h and driven from here through ctypes.

Device vectors are torch tensors (float64, or float32 for the *_f32 forms) on the handle's device;
torch is used for memory and streams only.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib as L
from ._lib import FxError, check, lib
from .meshes import ModelSpec

__all__ = ["Model", "Compiled", "MeshArrays", "InternalForce", "OperatorCoefficients", "MatrixFreeOperator",
           "SolveOptions", "SolveResult", "LinearSolver", "ConjugateGradient", "Gmres", "KrylovSolver",
           "MixedPrecisionSolver", "BatchEngine", "BatchedNewton", "VectorOps", "GroundMotions", "FxError", "ModelSpec",
           "device_memory"]


def _i32(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(L.p_i32)


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(L.p_f64)


def _ptr(t):
    """Device pointer of a torch tensor (or an int address)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_contiguous():
        raise ValueError("tensors must be contiguous")
    return t.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def device_memory(device: int = 0):
    """(free, total) bytes of device memory on `device` (fx_device_memory, cudaMemGetInfo)."""
    fr, tot = C.c_int64(), C.c_int64()
    check(lib().fx_device_memory(device, C.byref(fr), C.byref(tot)))
    return fr.value, tot.value


# ------------------------------------------------------------------ model and compile step
class Model:
    """io::Model for this path, built in memory from a ModelSpec (meshes.py)."""

    def __init__(self, spec: ModelSpec):
        self.spec = spec
        h = C.c_void_p()
        tags, pt = _i32(spec.tags)
        coords, pc = _f64(spec.coords)
        check(lib().fx_model_create(len(tags), pt, pc, C.byref(h)))
        self._h = h
        for g in spec.groups:
            mat = L.fx_material(kind=g.kind, element=g.element, E=g.E, nu=g.nu, rho=g.rho, sigma_y=g.sigma_y, H=g.H,
                                hk=g.hk)
            b, pb = _f64(np.array(g.b, dtype=np.float64))
            et, pet = _i32(g.etags)
            cn, pcn = _i32(np.asarray(g.conn).reshape(-1))
            check(lib().fx_model_add_group(h, C.byref(mat), pb, int(g.lumped), len(et), pet, pcn))
        if len(spec.fix_node):
            a, pa = _i32(spec.fix_node)
            d, pd = _i32(spec.fix_dof)
            check(lib().fx_model_add_fix(h, len(a), pa, pd))
        if len(spec.eqd_retained):
            r, pr = _i32(spec.eqd_retained)
            c, pc2 = _i32(spec.eqd_constrained)
            d, pd = _i32(spec.eqd_dof)
            check(lib().fx_model_add_equal_dof(h, len(r), pr, pc2, pd))
        for r in spec.rayleigh:
            et, pet = _i32(r.etags)
            check(lib().fx_model_add_rayleigh(h, r.alphaM, r.betaK, r.betaKinit, r.betaKcomm, len(et), pet))
        if len(spec.mass_node):
            n, pn = _i32(spec.mass_node)
            d, pd = _i32(spec.mass_dof)
            v, pv = _f64(spec.mass_value)
            check(lib().fx_model_add_mass(h, len(n), pn, pd, pv))

    def compile(self, renumbering="rcm", simd_width=32, coloring=False) -> "Compiled":
        """compile::compile_model (src/compile/batches.cpp:54-393)."""
        r = L.FX_RENUMBER_RCM if renumbering == "rcm" else L.FX_RENUMBER_OFF
        h = C.c_void_p()
        check(lib().fx_compile(self._h, r, simd_width, int(coloring), C.byref(h)))
        return Compiled(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_model_destroy(h)
            except Exception:  # interpreter shutdown: the library may be gone already
                pass
            self._h = None


class Compiled:
    """The compile step's arrays (compile::Compiled, batches.hpp:80-116)."""

    I32 = ("node_tag", "node_order", "element_order", "eq", "dof_offset", "node_model_index", "b_node", "b_eq",
           "b_param", "b_tag", "color_start", "color_elements", "eq_dof")
    F64 = ("coords", "lumped_mass", "lumped_alpha_mass", "nodal_mass", "nodal_alpha_mass")

    def __init__(self, h):
        self._h = h
        s = (C.c_int64 * 8)()
        check(lib().fx_compiled_sizes(h, s))
        (self.num_nodes, self.num_equations, self.num_slots, self.num_batches, self.count, self.padded,
         self.num_params, self.num_colors) = [int(v) for v in s]

    def array(self, name):
        if name in self.I32:
            n = lib().fx_compiled_array_i32(self._h, name.encode(), None)
            out = np.zeros(max(n, 0), np.int32)
            if n > 0:
                lib().fx_compiled_array_i32(self._h, name.encode(), out.ctypes.data_as(L.p_i32))
            return out
        if name in self.F64:
            n = lib().fx_compiled_array_f64(self._h, name.encode(), None)
            out = np.zeros(max(n, 0), np.float64)
            if n > 0:
                lib().fx_compiled_array_f64(self._h, name.encode(), out.ctypes.data_as(L.p_f64))
            return out
        raise KeyError(name)

    def params(self):
        arr = (L.fx_param_set * max(self.num_params, 1))()
        m = L.fx_mesh()
        check(lib().fx_compiled_mesh(self._h, arr, C.byref(m)))
        return [arr[i] for i in range(self.num_params)]

    def mesh(self) -> "MeshArrays":
        ps = self.params()
        return MeshArrays(num_nodes=self.num_nodes, num_equations=self.num_equations,
                          coords=self.array("coords"), count=self.count, padded=self.padded,
                          node=self.array("b_node"), eq=self.array("b_eq"), param=self.array("b_param"),
                          params=params_table(ps), lumped_mass=self.array("lumped_mass"),
                          nodal_mass=self.array("nodal_mass"), nodal_alpha_mass=self.array("nodal_alpha_mass"))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_compiled_destroy(h)
            except Exception:  # interpreter shutdown: the library may be gone already
                pass
            self._h = None


PARAM_FIELDS = ("kind", "mass_type", "E", "nu", "rho", "b0", "b1", "b2", "alphaM", "betaK", "betaKinit",
                "betaKcomm", "sigma_y", "H", "hk", "element")


def params_table(ps) -> np.ndarray:
    """Parameter sets as a float64 table [P, 16] in PARAM_FIELDS order."""
    out = np.zeros((len(ps), len(PARAM_FIELDS)))
    for i, p in enumerate(ps):
        out[i] = [p.kind, p.mass_type, p.E, p.nu, p.rho, p.b[0], p.b[1], p.b[2], p.alphaM, p.betaK, p.betaKinit,
                  p.betaKcomm, p.sigma_y, p.H, p.hk, p.element]
    return out


def ssp_element_constants(xl, E, nu):
    """One SSPbrick element's cached data (fx_ssp_element_constants): (geo[33], con[110]) for corner
    coordinates xl[3][8] and an elastic material."""
    xl, px = _f64(np.asarray(xl, np.float64).reshape(3, 8))
    geo, con = np.zeros(33), np.zeros(110)
    check(lib().fx_ssp_element_constants(px, E, nu, geo.ctypes.data_as(L.p_f64), con.ctypes.data_as(L.p_f64)))
    return geo, con


@dataclasses.dataclass
class MeshArrays:
    """What the device path consumes (fx_mesh): the compile step's arrays, from this library's
    compile step or from the reference's own compile_model."""
    num_nodes: int
    num_equations: int
    coords: np.ndarray  # [3N] SoA
    count: int
    padded: int
    node: np.ndarray  # [8 P]
    eq: np.ndarray  # [24 P]
    param: np.ndarray  # [P]
    params: np.ndarray  # [nparams, 15] (PARAM_FIELDS)
    lumped_mass: np.ndarray = None
    nodal_mass: np.ndarray = None
    nodal_alpha_mass: np.ndarray = None

    def to_c(self):
        """(fx_mesh, keep-alive list)."""
        keep = []
        m = L.fx_mesh()
        m.num_nodes = self.num_nodes
        m.num_equations = self.num_equations
        a, m.coords = _f64(self.coords)
        keep.append(a)
        m.count = self.count
        m.padded = self.padded
        for name in ("node", "eq", "param"):
            a, p = _i32(getattr(self, name))
            keep.append(a)
            setattr(m, name, p)
        P = (L.fx_param_set * max(len(self.params), 1))()
        for i, row in enumerate(self.params):
            q = P[i]
            q.kind, q.mass_type = int(row[0]), int(row[1])
            q.E, q.nu, q.rho = row[2], row[3], row[4]
            q.b[0], q.b[1], q.b[2] = row[5], row[6], row[7]
            q.alphaM, q.betaK, q.betaKinit, q.betaKcomm = row[8], row[9], row[10], row[11]
            q.sigma_y, q.H, q.hk = row[12], row[13], row[14]
            q.element = int(row[15]) if len(row) > 15 else 0
        keep.append(P)
        m.num_params = len(self.params)
        m.params = C.cast(P, C.POINTER(L.fx_param_set))
        for name in ("lumped_mass", "nodal_mass", "nodal_alpha_mass"):
            v = getattr(self, name)
            if v is not None and len(v):
                a, p = _f64(v)
                keep.append(a)
                setattr(m, name, p)
        return m, keep


# ------------------------------------------------------------------ operator and force
@dataclasses.dataclass
class OperatorCoefficients:
    """K_eff = stiffness K_t + damping C + mass M (element_operator.hpp:33-40)."""
    stiffness: float = 1.0
    damping: float = 0.0
    mass: float = 0.0
    initial: bool = False

    def c(self):
        return L.fx_coeffs(self.stiffness, self.damping, self.mass, int(self.initial), 0)


class InternalForce:
    """exec::InternalForce (src/exec/internal_force.hpp:80-213) on one B200."""

    PATHS = {"auto": L.FX_PATH_AUTO, "general": L.FX_PATH_GENERAL, "box": L.FX_PATH_BOX}

    def __init__(self, mesh: MeshArrays, device: int = 0):
        m, keep = mesh.to_c()
        h = C.c_void_p()
        check(lib().fx_force_create(C.byref(m), device, C.byref(h)))
        self._h = h
        self.mesh = mesh
        self.device = device
        self.num_equations = mesh.num_equations

    def set_soil_corrector(self, mode: str):
        """The multi-yield soil points' update: "fused" (one pass) or "compacted" (predictor,
        compaction of the plastic points, corrector on those only); the same bits either way."""
        check(lib().fx_force_set_soil_corrector(self._h, {"fused": 0, "compacted": 1}[mode]))

    def set_general_mode(self, mode: str):
        """The Gauss-point path's form: "exact" (the reference's arithmetic, bit for bit) or "fast"
        (eight threads per element, fused multiply-adds, within 1e-12; elastic stdBrick meshes)."""
        check(lib().fx_force_set_general_mode(self._h, {"exact": 0, "fast": 1}[mode]))

    def set_path(self, path: str):
        check(lib().fx_force_set_path(self._h, self.PATHS[path]))

    def info(self) -> dict:
        s = (C.c_int64 * 9)()
        check(lib().fx_force_info(self._h, s))
        keys = ("num_equations", "num_elements", "path", "box_qualifies", "nx", "ny", "nz", "device_bytes", "box_force")
        d = dict(zip(keys, [int(v) for v in s]))
        d["path"] = {1: "general", 2: "box"}[d["path"]]
        return d

    def apply_operator(self, k: OperatorCoefficients, x, y, stream=None):
        f = lib().fx_apply_operator_f32 if x.dtype.itemsize == 4 else lib().fx_apply_operator
        check(f(self._h, k.c(), _ptr(x), _ptr(y), _stream(stream)))

    def apply_operator_host(self, k: OperatorCoefficients, x: np.ndarray, y: np.ndarray, stream=None):
        """The same apply from host buffers (copies inside)."""
        check(lib().fx_apply_operator_host(self._h, k.c(), x.ctypes.data, y.ctypes.data, _stream(stream)))

    def operator_diagonal(self, k: OperatorCoefficients, d, stream=None):
        check(lib().fx_operator_diagonal(self._h, k.c(), _ptr(d), _stream(stream)))

    def compute(self, u, v, f, stream=None):
        fn = lib().fx_force_compute_f32 if u.dtype.itemsize == 4 else lib().fx_force_compute
        check(fn(self._h, _ptr(u), _ptr(v), _ptr(f), _stream(stream)))

    def mass_times_ground(self, direction: int, y, stream=None):
        check(lib().fx_mass_times_ground(self._h, direction, _ptr(y), _stream(stream)))

    def commit_state(self, stream=None):
        """InternalForce::commit_state (internal_force.cpp:507-509): the trial J2 and
        PressureIndependMultiYield states become the committed ones."""
        check(lib().fx_force_commit(self._h, _stream(stream)))

    def plastic_points(self) -> int:
        n = C.c_int64()
        check(lib().fx_force_plastic_points(self._h, C.byref(n)))
        return n.value

    def set_pimy(self, param_set: int, material: "PressureIndependMultiYield"):
        """Binds a PressureIndependMultiYield material to a parameter set (fx_force_set_pimy): the
        set's elements become stdBrick elements with that material's points, elastic stage."""
        check(lib().fx_force_set_pimy(self._h, int(param_set), material._h))
        self._materials = getattr(self, "_materials", {})
        self._materials[int(param_set)] = material

    def set_pdmy(self, param_set: int, material: "PressureDependMultiYield"):
        """Binds a PressureDependMultiYield material to a parameter set (fx_force_set_pdmy)."""
        check(lib().fx_force_set_pdmy(self._h, int(param_set), material._h))
        self._materials = getattr(self, "_materials", {})
        self._materials[int(param_set)] = material

    def set_material_stage(self, param_set: int, stage: int):
        """updateMaterialStage for a PressureIndependMultiYield set (InternalForce::set_material_stage)."""
        check(lib().fx_force_set_material_stage(self._h, int(param_set), int(stage)))

    def pimy_failed(self) -> int:
        n = C.c_int64()
        check(lib().fx_force_pimy_failed(self._h, C.byref(n)))
        return n.value

    J2_STATE = {"committed": (0, 13), "trial": (1, 13), "tangent": (2, 8)}

    def j2_state(self, which: str = "committed") -> np.ndarray:
        """The J2 state of the Gauss points, component c of point gp of element e at
        [(c * 8 + gp) * padded + e]."""
        w, comps = self.J2_STATE[which]
        out = np.empty(comps * 8 * self.mesh.padded)
        check(lib().fx_force_state(self._h, w, out.ctypes.data_as(L.p_f64), out.size))
        return out

    def set_j2_state(self, values: np.ndarray, which: str = "committed"):
        w, _ = self.J2_STATE[which]
        values = np.ascontiguousarray(values, np.float64)
        check(lib().fx_force_set_state(self._h, w, values.ctypes.data_as(L.p_f64), values.size))

    def min_critical_dt(self, scheme: str = "ExplicitDifference") -> float:
        dt = C.c_double()
        check(lib().fx_min_critical_dt(self._h, 1 if scheme == "ExplicitDifference" else 0, C.byref(dt)))
        return dt.value

    def element_critical_dts(self, scheme: str = "ExplicitDifference"):
        """Every element's stable step (InternalForce::element_critical_dts), a device FP64 tensor
        in batch order."""
        import torch
        out = torch.zeros(max(self.mesh.count, 1), dtype=torch.float64, device=torch.device("cuda", self.device))
        check(lib().fx_element_critical_dts(self._h, 1 if scheme == "ExplicitDifference" else 0, _ptr(out), None))
        return out[:self.mesh.count]

    def stability_may_change(self) -> bool:
        out = C.c_int32()
        check(lib().fx_stability_may_change(self._h, C.byref(out)))
        return bool(out.value)

    def prepare_stability_bounds(self, stream=None):
        check(lib().fx_stability_prepare(self._h, _stream(stream)))

    def min_critical_dt_bound(self, scheme: str = "ExplicitDifference", stream=None) -> float:
        dt = C.c_double()
        check(lib().fx_min_critical_dt_bound(self._h, 1 if scheme == "ExplicitDifference" else 0, C.byref(dt),
                                             _stream(stream)))
        return dt.value

    def set_explicit_checks(self, nan_check_interval: int = 100, stable_step_check_interval: int = 100,
                            allow_unstable_dt: bool = False):
        """The checks of later explicit stages (exec::RunOptions): non-finite displacements every
        nan_check_interval steps and at the end of each call (FX_E_DIVERGED), the stable step at
        the start and every stable_step_check_interval steps where it can change (FX_E_UNSTABLE)."""
        check(lib().fx_explicit_checks(self._h, nan_check_interval, stable_step_check_interval,
                                       1 if allow_unstable_dt else 0))

    def explicit_run(self, mass, u, vh, a, v, dt, steps, ag=None, direction=0, record_eq=None, stream=None):
        """`steps` ExplicitDifference steps (explicit_analysis.cpp:62-84, 687-705) with ground
        acceleration ag[step] (host array) in `direction`; returns the recorded acceleration
        history of equation record_eq (host) when asked."""
        agp = None
        if ag is not None:
            ag = np.ascontiguousarray(ag, np.float64)
            agp = ag.ctypes.data_as(L.p_f64)
        check(lib().fx_explicit_record(self._h, -1 if record_eq is None else int(record_eq), None, 0))
        fn = lib().fx_explicit_run_f32 if u.dtype.itemsize == 4 else lib().fx_explicit_run
        check(fn(self._h, _ptr(mass), direction, agp, steps, dt, _ptr(u), _ptr(vh), _ptr(a), _ptr(v),
                 _stream(stream)))
        if record_eq is not None:
            import torch
            hist = torch.zeros(steps + 1, dtype=torch.float64, device=u.device)
            torch.cuda.synchronize(u.device)
            check(lib().fx_explicit_record(self._h, int(record_eq), _ptr(hist), steps))
            return hist[:steps].cpu().numpy()
        return None

    def explicit_stage(self, scheme, mass, u, v, a, dt, steps, time=0.0, motions=None, alpha_mass=None,
                       resume=False, record_eq=None, stream=None):
        """An explicit stage (explicit_analysis.cpp:665-725): `steps` steps of "ExplicitDifference"
        or "CentralDifference" from `time` with the ground motions of `motions` (a GroundMotions,
        evaluated on the device each step); u, v, a (device FP64) are the committed state in and
        the end state out; alpha_mass is Compiled::lumped_alpha_mass (CentralDifference's damping
        diagonal). resume continues the previous call. Returns (end time, recorded acceleration
        history of record_eq or None)."""
        sc = {"ExplicitDifference": 1, "CentralDifference": 0}[scheme]
        check(lib().fx_explicit_record(self._h, -1 if record_eq is None else int(record_eq), None, 0))
        t = C.c_double(time)
        check(lib().fx_explicit_stage(self._h, sc, _ptr(mass), None if alpha_mass is None else _ptr(alpha_mass),
                                      None if motions is None else motions._h, steps, dt, C.byref(t), _ptr(u), _ptr(v),
                                      _ptr(a), 1 if resume else 0, _stream(stream)))
        hist = None
        if record_eq is not None:
            import torch
            h = torch.zeros(steps + 1, dtype=torch.float64, device=u.device)
            check(lib().fx_explicit_record(self._h, int(record_eq), _ptr(h), steps))
            hist = h[:steps].cpu().numpy()
        return t.value, hist

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_force_destroy(h)
            except Exception:  # interpreter shutdown: the library may be gone already
                pass
            self._h = None


class _MaterialPoints:
    """Material points of a soil model behind fx_<model>_* (the PressureIndependMultiYield and
    PressureDependMultiYield classes below). States are [nstate, npoints] arrays (value-major: value
    k of every point contiguous), strains and stresses [6, npoints] (11 22 33 12 23 31; engineering
    shear strains), tangents [36, npoints] (entry 6 r + c). update() works on device tensors,
    update_host() on numpy arrays; both write the trial state in full, so a commit is a swap of the
    committed and trial arrays. `stage` is the material stage (0 elastic, 1 plastic:
    updateMaterialStage)."""

    _fn = ""
    _nsetup = 0

    def _make(self, values, pairs, surfaces):
        v, pv = _f64(values)
        pp = None
        if pairs is not None and len(pairs):
            self._pairs = np.ascontiguousarray(pairs, np.float64).ravel()
            if self._pairs.size != 2 * int(surfaces):
                raise ValueError("a user backbone has noYieldSurf (gamma, G/Gmax) pairs")
            pp = self._pairs.ctypes.data_as(L.p_f64)
        h = C.c_void_p()
        check(getattr(lib(), self._fn + "_create")(pv, pp, C.byref(h)))
        self._h = h
        ns, nsurf = C.c_int32(), C.c_int32()
        check(getattr(lib(), self._fn + "_info")(h, C.byref(ns), C.byref(nsurf)))
        self.nstate, self.surfaces = ns.value, nsurf.value

    def _setup_values(self):
        out = np.zeros(self._nsetup)
        check(getattr(lib(), self._fn + "_setup_values")(self._h, out.ctypes.data_as(L.p_f64)))
        return out

    def initial_state(self, npoints, device=None):
        """The state of npoints new points: a torch tensor on `device` (an index), or numpy."""
        if device is None:
            s = np.zeros((self.nstate, npoints))
            check(getattr(lib(), self._fn + "_init_host")(self._h, npoints, s.ctypes.data_as(L.p_f64)))
            return s
        import torch
        s = torch.empty((self.nstate, npoints), dtype=torch.float64, device=torch.device("cuda", device))
        check(getattr(lib(), self._fn + "_init")(self._h, npoints, _ptr(s), None))
        return s

    def update(self, stage, committed, trial, strain, stress, tangent=None, failed=None, stream=None):
        n = committed.shape[1]
        check(getattr(lib(), self._fn + "_update")(self._h, int(stage), n, _ptr(committed), _ptr(trial), _ptr(strain),
                                                   _ptr(stress), _ptr(tangent), _ptr(failed), _stream(stream)))

    def update_host(self, stage, committed, trial, strain, stress, tangent=None) -> int:
        """Returns the points that met a state OpenSees stops for (their stress is NaN)."""
        n = committed.shape[1]
        bad = C.c_int32(0)
        arrs = [committed, trial, strain, stress] + ([tangent] if tangent is not None else [])
        for a in arrs:
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("host arrays must be C-contiguous float64")
        check(getattr(lib(), self._fn + "_update_host")(
            self._h, int(stage), n, committed.ctypes.data_as(L.p_f64), trial.ctypes.data_as(L.p_f64),
            strain.ctypes.data_as(L.p_f64), stress.ctypes.data_as(L.p_f64),
            tangent.ctypes.data_as(L.p_f64) if tangent is not None else None, C.byref(bad)))
        return bad.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                getattr(lib(), self._fn + "_destroy")(h)
            except Exception:
                pass
            self._h = None


class PressureIndependMultiYield(_MaterialPoints):
    """OpenSees' nDMaterial PressureIndependMultiYield, 3D (fx_pimy_*; the reference's
    PressureIndependMultiYield<NS>, src/physics/materials/pressure_independ_multi_yield.hpp): the
    constructor's arguments in OpenSees' order and defaults, `pairs` the (gamma, G/Gmax) pairs of a
    user backbone (noYieldSurf pairs) or None. Also bound to mesh parameter sets
    (InternalForce.set_pimy)."""

    _fn = "fx_pimy"
    _nsetup = 83

    def __init__(self, rho, refShearModul, refBulkModul, cohesi, peakShearStra, frictionAng=0.0, refPress=100.0,
                 pressDependCoe=0.0, noYieldSurf=20, pairs=None):
        self._make([rho, refShearModul, refBulkModul, cohesi, peakShearStra, frictionAng, refPress, pressDependCoe,
                    noYieldSurf], pairs, noYieldSurf)

    def setup_values(self):
        """(residual pressure, friction angle, cohesion), surface sizes [40], plastic moduli [40]."""
        out = self._setup_values()
        return out[:3], out[3:43], out[43:83]


class PressureDependMultiYield(_MaterialPoints):
    """OpenSees' nDMaterial PressureDependMultiYield, 3D (fx_pdmy_*; the reference's
    PressureDependMultiYield<NS>, src/physics/materials/pressure_depend_multi_yield.hpp): the
    constructor's arguments in OpenSees' order and the Tcl parser's defaults (liquefac3 is OpenSees'
    liquefactionParam4), hv and pv the volumetric plasticity terms (0 and 1: none)."""

    _fn = "fx_pdmy"
    _nsetup = 85

    def __init__(self, rho, refShearModul, refBulkModul, frictionAng, peakShearStra, refPress, pressDependCoe,
                 PTAng, contrac, dilat1, dilat2, liquefac1, liquefac2, liquefac3, noYieldSurf=20, pairs=None, e=0.6,
                 cs1=0.9, cs2=0.02, cs3=0.7, pa=101.0, c=0.3, hv=0.0, pv=1.0):
        self._make([rho, refShearModul, refBulkModul, frictionAng, peakShearStra, refPress, pressDependCoe, PTAng,
                    contrac, dilat1, dilat2, liquefac1, liquefac2, liquefac3, noYieldSurf, e, cs1, cs2, cs3, pa, c,
                    hv, pv], pairs, noYieldSurf)

    def setup_values(self):
        """(residual pressure, friction angle, phase-transformation angle, its stress ratio, its
        octahedral strain), surface sizes [40], plastic moduli [40]."""
        out = self._setup_values()
        return out[:5], out[5:45], out[45:85]


class GroundMotions:
    """exec::GroundMotions (src/exec/ground_motion.hpp:22-70): UniformExcitation patterns with
    Path series, evaluated on the device. add(): one pattern in DOF `dof` (0-based) with factor
    `fact`; its series is `values` with a uniform spacing `dt` (PathSeries) or at `times`
    (PathTimeSeries), scaled by `factor`."""

    def __init__(self, patterns=()):
        h = C.c_void_p()
        check(lib().fx_motions_create(C.byref(h)))
        self._h = h
        self.count = 0
        for p in patterns:
            self.add(**p)

    def add(self, dof, fact, values, dt=None, times=None, factor=1.0, use_last=False, prepend_zero=False):
        v = np.ascontiguousarray(values, np.float64)
        tp = None
        if times is not None:
            tm = np.ascontiguousarray(times, np.float64)
            if tm.size != v.size:
                raise ValueError("times and values differ in length")
            tp = tm.ctypes.data_as(L.p_f64)
        check(lib().fx_motions_add(self._h, int(dof), float(fact), v.ctypes.data_as(L.p_f64), tp, v.size,
                                   0.0 if dt is None else float(dt), float(factor), int(bool(use_last)),
                                   int(bool(prepend_zero))))
        self.count += 1

    def evaluate(self, t):
        out = np.zeros(max(self.count, 1))
        check(lib().fx_motions_evaluate(self._h, float(t), out.ctypes.data_as(L.p_f64)))
        return out[:self.count]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_motions_destroy(h)
            except Exception:
                pass
            self._h = None


class MatrixFreeOperator:
    """exec::MatrixFreeOperator (src/exec/matrix_free_operator.hpp:16-36)."""

    def __init__(self, force: InternalForce, k: OperatorCoefficients = None):
        self.force = force
        self.k = k or OperatorCoefficients()

    def set_coefficients(self, k):
        self.k = k

    @property
    def rows(self):
        return self.force.num_equations

    def apply(self, x, y, stream=None):
        self.force.apply_operator(self.k, x, y, stream)

    def diagonal(self, d, stream=None):
        self.force.operator_diagonal(self.k, d, stream)


# ------------------------------------------------------------------ solvers
@dataclasses.dataclass
class SolveOptions:
    relative_tolerance: float = 1e-10
    absolute_tolerance: float = 0.0
    max_iterations: int = 10000
    lanes: int = 32
    restart: int = 30


@dataclasses.dataclass
class SolveResult:
    converged: bool
    iterations: int
    rhs_norm: float
    initial_residual: float
    final_residual: float
    indefinite: bool
    refinements: int = 0


class LinearSolver:
    """solvers::LinearSolver with the Jacobi preconditioner (linear_solver.hpp:96-105)."""
    METHOD = L.FX_SOLVER_CG

    def __init__(self, options: SolveOptions = None):
        self.options = options or SolveOptions()
        self._h = None
        self.op = None

    def setup(self, op: MatrixFreeOperator, stream=None):
        o = self.options
        if self._h is None or self.op is None or self.op.force is not op.force:
            if self._h is not None:
                lib().fx_solver_destroy(self._h)
            h = C.c_void_p()
            opts = L.fx_solve_opts(o.relative_tolerance, o.absolute_tolerance, o.max_iterations, o.lanes, o.restart, 0)
            check(lib().fx_solver_create(op.force._h, self.METHOD, opts, C.byref(h)))
            self._h = h
        self.op = op
        check(lib().fx_solver_setup(self._h, op.k.c(), _stream(stream)))

    def solve(self, b, x, stream=None) -> SolveResult:
        r = L.fx_solve_result()
        check(lib().fx_solver_solve(self._h, _ptr(b), _ptr(x), C.byref(r), _stream(stream)))
        return SolveResult(bool(r.converged), r.iterations, r.rhs_norm, r.initial_residual, r.final_residual,
                           bool(r.indefinite), r.refinements)

    def newton(self, fext, u, tol: float = 1e-6, test: str = "NormUnbalance", max_newton: int = 25, stream=None):
        """Newton iterations of one quasi-static load step (fx_solver_newton) with the stage's
        absolute convergence test (NormUnbalance or NormDispIncr); u is updated in place; returns
        (Newton iterations, SolveResult of the Newton test). ConjugateGradient, or
        MixedPrecisionSolver (FP32 CG on the tangent inside FP64 refinement)."""
        r = L.fx_solve_result()
        it = C.c_int32()
        t = L.FX_TEST_NORM_UNBALANCE if test == "NormUnbalance" else L.FX_TEST_NORM_DISP_INCR
        check(lib().fx_solver_newton(self._h, _ptr(fext), _ptr(u), t, tol, max_newton, C.byref(it), C.byref(r),
                                     _stream(stream)))
        return it.value, SolveResult(bool(r.converged), r.iterations, r.rhs_norm, r.initial_residual,
                                     r.final_residual, bool(r.indefinite), r.refinements)

    def newmark_step(self, fext, u, v, a, dt: float, beta: float = 0.25, gamma: float = 0.5, tol: float = 1e-6,
                     test: str = "NormUnbalance", max_newton: int = 25, stream=None):
        """One Newmark time step (fx_solver_newmark); u, v, a updated in place. The solver must be
        set up with OperatorCoefficients(1, gamma / (beta dt), 1 / (beta dt^2))."""
        r = L.fx_solve_result()
        it = C.c_int32()
        t = L.FX_TEST_NORM_UNBALANCE if test == "NormUnbalance" else L.FX_TEST_NORM_DISP_INCR
        check(lib().fx_solver_newmark(self._h, _ptr(fext), _ptr(u), _ptr(v), _ptr(a), dt, beta, gamma, t, tol,
                                      max_newton, C.byref(it), C.byref(r), _stream(stream)))
        return it.value, SolveResult(bool(r.converged), r.iterations, r.rhs_norm, r.initial_residual,
                                     r.final_residual, bool(r.indefinite), r.refinements)

    def newmark_step_recover(self, fext0, fext1, u, v, a, dt: float, beta: float = 0.25, gamma: float = 0.5,
                             tol: float = 1e-6, test: str = "NormUnbalance", max_newton: int = 25,
                             max_retries: int = 0, num_sublevels: int = 0, num_substeps: int = 2, stream=None):
        """One Newmark step with the reference's retry and substep recovery
        (fx_solver_newmark_recover): the load ramps from fext0 (None: fext1) to fext1 over the
        step; a converged step (or substep) commits the materials. Returns (stats, SolveResult),
        stats = dict(attempts, failed, retries, substepped, newton)."""
        r = L.fx_solve_result()
        st = (C.c_int32 * 5)()
        t = L.FX_TEST_NORM_UNBALANCE if test == "NormUnbalance" else L.FX_TEST_NORM_DISP_INCR
        check(lib().fx_solver_newmark_recover(self._h, _ptr(fext0), _ptr(fext1), _ptr(u), _ptr(v), _ptr(a), dt, beta,
                                              gamma, t, tol, max_newton, max_retries, num_sublevels, num_substeps, st,
                                              C.byref(r), _stream(stream)))
        return (dict(zip(("attempts", "failed", "retries", "substepped", "newton"), list(st))),
                SolveResult(bool(r.converged), r.iterations, r.rhs_norm, r.initial_residual, r.final_residual,
                            bool(r.indefinite), r.refinements))

    def newton_recover(self, fext, u, tol: float = 1e-6, test: str = "NormUnbalance", max_newton: int = 25,
                       max_retries: int = 0, stream=None):
        """One quasi-static load step with retries (fx_solver_newton_recover); a converged step
        commits the materials, a failed one leaves u at its committed value."""
        r = L.fx_solve_result()
        st = (C.c_int32 * 5)()
        t = L.FX_TEST_NORM_UNBALANCE if test == "NormUnbalance" else L.FX_TEST_NORM_DISP_INCR
        check(lib().fx_solver_newton_recover(self._h, _ptr(fext), _ptr(u), t, tol, max_newton, max_retries, st,
                                             C.byref(r), _stream(stream)))
        return (dict(zip(("attempts", "failed", "retries", "substepped", "newton"), list(st))),
                SolveResult(bool(r.converged), r.iterations, r.rhs_norm, r.initial_residual, r.final_residual,
                            bool(r.indefinite), r.refinements))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_solver_destroy(h)
            except Exception:  # interpreter shutdown: the library may be gone already
                pass
            self._h = None


class ConjugateGradient(LinearSolver):
    METHOD = L.FX_SOLVER_CG


class Gmres(LinearSolver):
    METHOD = L.FX_SOLVER_GMRES


class KrylovSolver(LinearSolver):
    METHOD = L.FX_SOLVER_KRYLOV


class MixedPrecisionSolver(LinearSolver):
    """FP32 PCG inside FP64 iterative refinement (the FP32 operator: the box kernel, or the FP32
    Gauss-point form on other meshes and J2 sets)."""
    METHOD = L.FX_SOLVER_IR

    def __init__(self, options: SolveOptions = None, inner_tolerance: float = 1e-4):
        super().__init__(options)
        self.inner_tolerance = inner_tolerance

    def setup(self, op, stream=None):
        super().setup(op, stream)
        check(lib().fx_solver_set_inner_tolerance(self._h, self.inner_tolerance))


MATH_FUNCTIONS = {"exp": L.FX_MATH_EXP, "log": L.FX_MATH_LOG, "pow": L.FX_MATH_POW, "cos": L.FX_MATH_COS}


def math_eval(name: str, x, y=None, stream=None):
    """fx_math_eval: the PressureDependMultiYield device update's exp, log, pow or cos (`name`) of a
    float64 device tensor x (and y, for pow), element by element; returns a new tensor."""
    import torch
    fn = MATH_FUNCTIONS[name]
    x = x.contiguous()
    if x.dtype != torch.float64 or (y is not None and (y.dtype != torch.float64 or y.shape != x.shape)):
        raise ValueError("math_eval takes float64 tensors of one shape")
    y = y.contiguous() if y is not None else None
    out = torch.empty_like(x)
    check(lib().fx_math_eval(fn, _ptr(x), _ptr(y) if y is not None else None, _ptr(out), x.numel(), _stream(stream)))
    return out


def math_eval_host(name: str, x: np.ndarray, y: np.ndarray = None) -> np.ndarray:
    """fx_math_eval_host: the same functions on the host (the same bits as math_eval)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    yy = np.ascontiguousarray(y, dtype=np.float64) if y is not None else None
    if yy is not None and yy.shape != x.shape:
        raise ValueError("x and y must have one shape")
    out = np.empty_like(x)
    check(lib().fx_math_eval_host(MATH_FUNCTIONS[name], x.ctypes.data_as(L.p_f64),
                                  yy.ctypes.data_as(L.p_f64) if yy is not None else None, out.ctypes.data_as(L.p_f64),
                                  x.size))
    return out


class BatchEngine:
    """Many box meshes resident on one device and solved together (fx_engine_*): per slot FP32
    Jacobi-PCG inside FP64 iterative refinement, the same bits as MixedPrecisionSolver on that mesh
    alone; one launch per operator apply over every running slot's element tiles.

    admit() takes an InternalForce (kept alive here until its slot is retired) and a host
    right-hand side; round() advances every running slot by one tick (its correction and outer step
    when due, then 8 inner iterations); finished() and retire() hand results back. try_admit()
    returns None instead of raising when the engine is full.
    inner="fp64" makes the inner solves FP64 Jacobi-PCG with the FP64 operator (the batched engine
    without reduced precision; give an inner_tolerance at or below the outer relative tolerance).
    The same InternalForce may be admitted into several slots at once (its maps and tables are only
    read); each slot has its own vectors.
    """

    def __init__(self, capacity: int, max_slots: int, k: OperatorCoefficients = None, options: SolveOptions = None,
                 inner_tolerance: float = 1e-4, device: int = 0, inner: str = "fp32"):
        o = options or SolveOptions(relative_tolerance=1e-8)
        k = k or OperatorCoefficients()
        opts = L.fx_solve_opts(o.relative_tolerance, o.absolute_tolerance, o.max_iterations, o.lanes, o.restart, 0)
        h = C.c_void_p()
        check(lib().fx_engine_create(device, capacity, max_slots, k.c(), opts, inner_tolerance, C.byref(h)))
        self._h = h
        if inner not in ("fp32", "fp64"):
            raise ValueError("inner must be 'fp32' or 'fp64'")
        self.inner = inner
        if inner == "fp64":
            check(lib().fx_engine_set_precision(h, L.FX_ENGINE_INNER_FP64))
        self.device = device
        self._forces = {}

    def set_persistent(self, on: bool = True):
        """The batched apply as a persistent wave of CTAs over the work list (or one CTA per item)."""
        check(lib().fx_engine_set_persistent(self._h, 1 if on else 0))

    def admit(self, force: InternalForce, b: np.ndarray) -> int:
        b = np.ascontiguousarray(b, dtype=np.float64)
        slot = C.c_int32()
        check(lib().fx_engine_admit(self._h, force._h, b.ctypes.data_as(L.p_f64), C.byref(slot)))
        self._forces[slot.value] = force
        return slot.value

    def try_admit(self, force: InternalForce, b: np.ndarray):
        try:
            return self.admit(force, b)
        except FxError as e:
            if e.code == L.FX_E_NOMEM:
                return None
            raise

    def round(self) -> int:
        running = C.c_int32()
        check(lib().fx_engine_round(self._h, C.byref(running)))
        return running.value

    def finished(self, slot: int) -> bool:
        f = C.c_int32()
        check(lib().fx_engine_finished(self._h, slot, C.byref(f)))
        return bool(f.value)

    def retire(self, slot: int, n: int = None):
        force = self._forces[slot]
        n = force.info()["num_equations"] if n is None else n
        x = np.empty(n)
        r = L.fx_solve_result()
        check(lib().fx_engine_retire(self._h, slot, x.ctypes.data_as(L.p_f64), C.byref(r)))
        del self._forces[slot]
        return x, SolveResult(bool(r.converged), r.iterations, r.rhs_norm, r.initial_residual, r.final_residual,
                              bool(r.indefinite), r.refinements)

    def slots(self):
        return list(self._forces)

    def info(self) -> dict:
        a = (C.c_int64 * 6)()
        check(lib().fx_engine_info(self._h, a))
        keys = ["capacity", "in_use", "max_slots", "slots_in_use", "rounds", "vector_bytes"]
        return dict(zip(keys, list(a)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_engine_destroy(h)
            except Exception:  # interpreter shutdown: the library may be gone already
                pass
            self._h = None


class BatchedNewton:
    """Quasi-static load steps of many independent meshes at once (fx_nbatch_*): one combined
    mesh (instance i's equations at offsets[i] .. offsets[i] + equations[i]), one launch per element
    kernel for all instances, per-instance Newton test and Jacobi-PCG on the device; per instance
    bit for bit LinearSolver.newton (NormUnbalance) on that mesh alone. mixed: the Newton steps'
    linear solves by FP32 CG inside FP64 refinement (inner_tolerance), per instance the bits of
    MixedPrecisionSolver.newton on that mesh alone."""

    def __init__(self, meshes, options: SolveOptions = None, device: int = 0, mixed: bool = False,
                 inner_tolerance: float = 1e-4):
        o = options or SolveOptions(relative_tolerance=1e-12, max_iterations=20000)
        arr = (L.fx_mesh * len(meshes))()
        keep = []
        for i, m in enumerate(meshes):
            cm, k = m.to_c()
            arr[i] = cm
            keep.append(k)
        opts = L.fx_solve_opts(o.relative_tolerance, o.absolute_tolerance, o.max_iterations, o.lanes, o.restart, 0)
        h = C.c_void_p()
        check(lib().fx_nbatch_create(arr, len(meshes), device, opts, C.byref(h)))
        self._h = h
        self.count = len(meshes)
        self.device = device
        off = (C.c_int64 * (self.count + 1))()
        neq = (C.c_int64 * self.count)()
        check(lib().fx_nbatch_layout(h, off, neq))
        self.offsets = np.array(off[:])
        self.equations = np.array(neq[:])
        self.total = int(self.offsets[-1])
        self._force = lib().fx_nbatch_force(h)
        if mixed:
            check(lib().fx_nbatch_set_inner(h, L.FX_SOLVER_IR, inner_tolerance))

    def combine(self, per_instance) -> np.ndarray:
        """Host vectors of the instances -> one vector in the combined layout."""
        out = np.zeros(self.total)
        for i, v in enumerate(per_instance):
            out[self.offsets[i]:self.offsets[i] + self.equations[i]] = v
        return out

    def split(self, combined):
        """One vector in the combined layout -> the instances' host vectors."""
        c = np.asarray(combined)
        return [c[self.offsets[i]:self.offsets[i] + self.equations[i]] for i in range(self.count)]

    def step(self, fext, u, tol: float = 1e-6, max_newton: int = 25, stream=None):
        """One load step of every instance (u updated in place): (Newton solves, SolveResults)."""
        it = (C.c_int32 * self.count)()
        res = (L.fx_solve_result * self.count)()
        check(lib().fx_nbatch_step(self._h, _ptr(fext), _ptr(u), tol, max_newton, it, res, _stream(stream)))
        out = [SolveResult(bool(r.converged), r.iterations, r.rhs_norm, r.initial_residual, r.final_residual,
                           bool(r.indefinite), r.refinements) for r in res]
        return np.array(it[:]), out

    def commit_state(self, stream=None):
        check(lib().fx_force_commit(self._force, _stream(stream)))

    def plastic_points(self) -> int:
        n = C.c_int64()
        check(lib().fx_force_plastic_points(self._force, C.byref(n)))
        return n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_nbatch_destroy(h)
            except Exception:  # interpreter shutdown: the library may be gone already
                pass
            self._h = None


class VectorOps:
    """solvers::VectorOps(n, lanes): deterministic dot in the documented order."""

    def __init__(self, n: int, lanes: int = 32, device: int = 0):
        h = C.c_void_p()
        check(lib().fx_vops_create(n, lanes, device, C.byref(h)))
        self._h = h

    def dot(self, x, y, stream=None) -> float:
        r = C.c_double()
        check(lib().fx_vops_dot(self._h, _ptr(x), _ptr(y), x.numel(), None, C.byref(r), _stream(stream)))
        return r.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().fx_vops_destroy(h)
            except Exception:  # interpreter shutdown: the library may be gone already
                pass
            self._h = None
