"""Oracle (test infrastructure only): Python access to
  - _ref/libfxref.so: the reference's own C++ (compile step, InternalForce, CG/GMRES, stdBrick
    physics) built here from its sources with the Kokkos-subset shim (oracle/Makefile), and
  - _ref/libfxport.so: the plain-C restatement of the hot path (port/fx_oracle.c).

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module, as the checker.
The product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libfxref.so")
# the same reference objects with pow, exp, log and cos bound to the device update's functions
REF_FXMATH_LIB = os.path.join(HERE, "_ref", "libfxref_fxmath.so")
PORT_LIB = os.path.join(HERE, "_ref", "libfxport.so")

p_i32 = C.POINTER(C.c_int32)
p_i64 = C.POINTER(C.c_int64)
p_f64 = C.POINTER(C.c_double)
p_i8 = C.POINTER(C.c_int8)
vp = C.c_void_p

_ref = None
_ref_fxmath = None
_port = None


def build(reference_dir: str = None) -> None:
    """Builds the oracle libraries: the C restatement always, the reference's own sources where
    `reference_dir` (default: the environment variable FEMORAX_REFERENCE) holds its checkout."""
    reference_dir = reference_dir or os.environ.get("FEMORAX_REFERENCE", "")
    have = bool(reference_dir) and os.path.isdir(os.path.join(reference_dir, "src"))
    subprocess.run(["make", "-s", "-j8", "port"], cwd=HERE, check=True)
    if have:
        subprocess.run(["make", "-s", "-j8", "ref", f"REF={reference_dir}"], cwd=HERE, check=True)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "femorax_b200", "libfemorax_b200.so")):
            subprocess.run(["make", "-s", "adapter", f"REF={reference_dir}"], cwd=HERE, check=True)


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def have_ref_fxmath() -> bool:
    return os.path.exists(REF_FXMATH_LIB)


def ref(math: str = "libm"):
    """The reference library: with the C library's elementary functions ("libm"), or with pow,
    exp, log and cos bound to those of this library's device PressureDependMultiYield update ("fx")."""
    global _ref, _ref_fxmath
    if math == "fx":
        if _ref_fxmath is None:
            _ref_fxmath = _declare_ref(C.CDLL(REF_FXMATH_LIB))
        return _ref_fxmath
    if _ref is None:
        _ref = _declare_ref(C.CDLL(REF_LIB))
    return _ref


def _declare_ref(L):
    L.fxref_last_error.restype = C.c_char_p
    L.fxref_model_create.restype = vp
    L.fxref_model_create.argtypes = [C.c_int32, p_i32, p_f64]
    L.fxref_model_destroy.argtypes = [vp]
    L.fxref_model_add_group.argtypes = [vp, C.c_double, C.c_double, C.c_double, p_f64, C.c_int, C.c_int32, p_i32,
                                        p_i32, C.c_int]
    L.fxref_ssp_constants.argtypes = [p_f64, C.c_double, C.c_double, p_f64, p_f64]
    L.fxref_model_add_fix.argtypes = [vp, C.c_int32, p_i32, p_i32]
    L.fxref_model_add_equal_dof.argtypes = [vp, C.c_int32, p_i32, p_i32, p_i32]
    L.fxref_model_add_rayleigh.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32, p_i32]
    L.fxref_model_add_mass.argtypes = [vp, C.c_int32, p_i32, p_i32, p_f64]
    L.fxref_motions_create.restype = vp
    L.fxref_motions_destroy.argtypes = [vp]
    L.fxref_motions_add.argtypes = [vp, C.c_int32, C.c_double, p_f64, p_f64, C.c_int32, C.c_double, C.c_double,
                                    C.c_int32, C.c_int32]
    L.fxref_motions_evaluate.argtypes = [vp, C.c_double, p_f64]
    L.fxref_compile.restype = vp
    L.fxref_compile.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.fxref_compiled_destroy.argtypes = [vp]
    L.fxref_compiled_sizes.argtypes = [vp, p_i64]
    L.fxref_compiled_array_i32.restype = C.c_int64
    L.fxref_compiled_array_i32.argtypes = [vp, C.c_char_p, p_i32]
    L.fxref_compiled_array_f64.restype = C.c_int64
    L.fxref_compiled_array_f64.argtypes = [vp, C.c_char_p, p_f64]
    L.fxref_compiled_param.argtypes = [vp, C.c_int32, p_f64]
    L.fxref_force_create.restype = vp
    L.fxref_force_create.argtypes = [vp, C.c_int]
    L.fxref_force_destroy.argtypes = [vp]
    L.fxref_apply_operator.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, p_f64, p_f64]
    L.fxref_operator_diagonal.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_int, p_f64]
    L.fxref_mass_times_ground.argtypes = [vp, C.c_int, p_f64]
    L.fxref_force_compute.argtypes = [vp, p_f64, p_f64, C.c_int, p_f64]
    L.fxref_element_critical_dts.argtypes = [vp, C.c_int, p_f64]
    L.fxref_stability_may_change.argtypes = [vp]
    L.fxref_prepare_stability_bounds.argtypes = [vp]
    L.fxref_min_critical_dt_bound.restype = C.c_double
    L.fxref_min_critical_dt_bound.argtypes = [vp, C.c_int]
    L.fxref_min_critical_dt.restype = C.c_double
    L.fxref_min_critical_dt.argtypes = [vp, C.c_int]
    L.fxref_solve.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                              C.c_int, C.c_int, p_f64, p_f64, p_f64]
    L.fxref_host_dot.restype = C.c_double
    L.fxref_host_dot.argtypes = [p_f64, p_f64, C.c_int64, C.c_int]
    L.fxref_brick_compute.argtypes = [p_f64, p_f64, p_f64, p_f64, p_f64, p_f64, p_f64]
    L.fxref_brick_mass.argtypes = [p_f64, p_f64, p_f64, p_f64]
    L.fxref_brick_operator.argtypes = [p_f64, p_f64, p_f64, p_f64, p_f64, p_f64, C.c_int, p_i32]
    L.fxref_brick_critical_dt.restype = C.c_double
    L.fxref_brick_critical_dt.argtypes = [p_f64, p_f64, C.c_int, p_f64]
    L.fxref_pimy_create.argtypes = [p_f64, p_f64, C.c_int32, C.POINTER(vp)]
    L.fxref_pdmy_create.argtypes = [p_f64, p_f64, C.c_int32, C.POINTER(vp)]
    L.fxref_pdmy_destroy.argtypes = [vp]
    L.fxref_pdmy_nstate.restype = C.c_int32
    L.fxref_pdmy_setup_values.argtypes = [vp, p_f64]
    L.fxref_pdmy_initial_state.argtypes = [vp, p_f64]
    L.fxref_pdmy_update.argtypes = [vp, C.c_int32, p_f64, p_f64, p_f64, p_f64, p_f64]
    L.fxref_model_add_group_pimy.argtypes = [vp, p_f64, p_f64, C.c_int32, p_f64, C.c_int, C.c_int32, p_i32, p_i32]
    L.fxref_model_add_group_pdmy.argtypes = [vp, p_f64, p_f64, C.c_int32, p_f64, C.c_int, C.c_int32, p_i32, p_i32]
    L.fxref_force_set_stage.argtypes = [vp, C.c_int32, C.c_int32]
    L.fxref_force_commit.argtypes = [vp]
    L.fxref_apply_operator_at.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_int, p_f64, p_f64, p_f64]
    L.fxref_operator_diagonal_at.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_int, p_f64, p_f64]
    L.fxref_pimy_destroy.argtypes = [vp]
    L.fxref_pimy_nstate.restype = C.c_int32
    L.fxref_pimy_setup_values.argtypes = [vp, p_f64]
    L.fxref_pimy_initial_state.argtypes = [vp, p_f64]
    L.fxref_pimy_update.argtypes = [vp, C.c_int32, p_f64, p_f64, p_f64, p_f64, p_f64]
    return L


def _f(a):
    a = np.ascontiguousarray(a, np.float64)
    return a, a.ctypes.data_as(p_f64)


def _i(a):
    a = np.ascontiguousarray(a, np.int32)
    return a, a.ctypes.data_as(p_i32)


class RefModel:
    """io::Model in the reference's own structures, from a ModelSpec (femorax_b200.meshes)."""

    def __init__(self, spec):
        L = ref()
        t, pt = _i(spec.tags)
        c, pc = _f(np.asarray(spec.coords).reshape(-1))
        self.h = L.fxref_model_create(len(t), pt, pc)
        for g in spec.groups:
            if g.kind != 0:
                raise ValueError("the reference has no J2 material")
            b, pb = _f(np.array(g.b, np.float64))
            et, pet = _i(g.etags)
            cn, pcn = _i(np.asarray(g.conn).reshape(-1))
            if getattr(g, "pdmy", None) is not None:
                in23, pairs = g.pdmy
                p23, pp23 = _f(in23)
                pr = np.ascontiguousarray(pairs if pairs is not None else [], np.float64)
                L.fxref_model_add_group_pdmy(self.h, pp23, pr.ctypes.data_as(p_f64) if pr.size else None, pr.size // 2,
                                             pb, int(g.lumped), len(et), pet, pcn)
            elif getattr(g, "pimy", None) is not None:
                in9, pairs = g.pimy
                p9, pp9 = _f(in9)
                pr = np.ascontiguousarray(pairs if pairs is not None else [], np.float64)
                L.fxref_model_add_group_pimy(self.h, pp9, pr.ctypes.data_as(p_f64) if pr.size else None, pr.size // 2,
                                             pb, int(g.lumped), len(et), pet, pcn)
            else:
                L.fxref_model_add_group(self.h, g.E, g.nu, g.rho, pb, int(g.lumped), len(et), pet, pcn,
                                        int(getattr(g, "element", 0)))
        if len(spec.fix_node):
            a, pa = _i(spec.fix_node)
            d, pd = _i(spec.fix_dof)
            L.fxref_model_add_fix(self.h, len(a), pa, pd)
        if len(spec.eqd_retained):
            r, pr = _i(spec.eqd_retained)
            c2, pc2 = _i(spec.eqd_constrained)
            d, pd = _i(spec.eqd_dof)
            L.fxref_model_add_equal_dof(self.h, len(r), pr, pc2, pd)
        for r in spec.rayleigh:
            et, pet = _i(r.etags)
            L.fxref_model_add_rayleigh(self.h, r.alphaM, r.betaK, r.betaKinit, r.betaKcomm, len(et), pet)
        if len(spec.mass_node):
            n, pn = _i(spec.mass_node)
            d, pd = _i(spec.mass_dof)
            v, pv = _f(spec.mass_value)
            L.fxref_model_add_mass(self.h, len(n), pn, pd, pv)

    def compile(self, renumbering="rcm", simd_width=32, coloring=False):
        h = ref().fxref_compile(self.h, 1 if renumbering == "rcm" else 0, simd_width, int(coloring))
        if not h:
            raise RuntimeError(ref().fxref_last_error().decode())
        return RefCompiled(h)

    def __del__(self):
        if getattr(self, "h", None):
            ref().fxref_model_destroy(self.h)
            self.h = None


class RefCompiled:
    I32 = ("node_tag", "node_order", "element_order", "eq", "dof_offset", "node_model_index", "b_node", "b_eq",
           "b_param", "b_tag", "color_start", "color_elements", "eq_dof")

    def __init__(self, h):
        self.h = h
        s = (C.c_int64 * 8)()
        ref().fxref_compiled_sizes(h, s)
        (self.num_nodes, self.num_equations, self.num_slots, self.num_batches, self.count, self.padded,
         self.num_params, self.num_colors) = [int(v) for v in s]

    def array(self, name):
        L = ref()
        if name in self.I32:
            n = L.fxref_compiled_array_i32(self.h, name.encode(), None)
            out = np.zeros(max(n, 0), np.int32)
            if n > 0:
                L.fxref_compiled_array_i32(self.h, name.encode(), out.ctypes.data_as(p_i32))
            return out
        n = L.fxref_compiled_array_f64(self.h, name.encode(), None)
        out = np.zeros(max(n, 0), np.float64)
        if n > 0:
            L.fxref_compiled_array_f64(self.h, name.encode(), out.ctypes.data_as(p_f64))
        return out

    def params(self) -> np.ndarray:
        """[P, 15] in femorax_b200.PARAM_FIELDS order."""
        out = np.zeros((self.num_params, 15))
        buf = (C.c_double * 14)()
        for p in range(self.num_params):
            ref().fxref_compiled_param(self.h, p, buf)
            E, nu, rho, b0, b1, b2, mt, aM, bK, bKi, bKc = list(buf)[:11]
            out[p] = [0, mt, E, nu, rho, b0, b1, b2, aM, bK, bKi, bKc, 0, 0, 0]
        return out

    def mesh_fields(self) -> dict:
        """The fields of femorax_b200.MeshArrays, from the reference's compile step."""
        return dict(num_nodes=self.num_nodes, num_equations=self.num_equations, coords=self.array("coords"),
                    count=self.count, padded=self.padded, node=self.array("b_node"), eq=self.array("b_eq"),
                    param=self.array("b_param"), params=self.params(), lumped_mass=self.array("lumped_mass"),
                    nodal_mass=self.array("nodal_mass"), nodal_alpha_mass=self.array("nodal_alpha_mass"))

    def __del__(self):
        if getattr(self, "h", None):
            ref().fxref_compiled_destroy(self.h)
            self.h = None


class RefForce:
    """The reference's exec::InternalForce on the host (OpenMP threads through the shim)."""

    def __init__(self, compiled: RefCompiled, cache: bool = True):
        self.c = compiled
        self.h = ref().fxref_force_create(compiled.h, int(cache))
        if not self.h:
            raise RuntimeError(ref().fxref_last_error().decode())
        self.n = compiled.num_equations

    def apply_operator(self, k, x, scatter=0, geometry=1):
        x, px = _f(x)
        y = np.zeros(self.n)
        rc = ref().fxref_apply_operator(self.h, k[0], k[1], k[2], scatter, geometry, px, y.ctypes.data_as(p_f64))
        if rc:
            raise RuntimeError(ref().fxref_last_error().decode())
        return y

    def operator_diagonal(self, k, geometry=1):
        d = np.zeros(self.n)
        ref().fxref_operator_diagonal(self.h, k[0], k[1], k[2], geometry, d.ctypes.data_as(p_f64))
        return d

    def mass_times_ground(self, direction):
        y = np.zeros(self.n)
        ref().fxref_mass_times_ground(self.h, direction, y.ctypes.data_as(p_f64))
        return y

    def force(self, u, v, geometry=1):
        u, pu = _f(u)
        v, pv = _f(v)
        f = np.zeros(self.n)
        ref().fxref_force_compute(self.h, pu, pv, geometry, f.ctypes.data_as(p_f64))
        return f

    def set_stage(self, material, stage):
        """updateMaterialStage of model material `material` (0-based)."""
        assert ref().fxref_force_set_stage(self.h, material, stage) == 0

    def commit(self):
        assert ref().fxref_force_commit(self.h) == 0

    def apply_operator_at(self, k, u, x, initial=False):
        """K_eff x with every point's tangent recomputed at displacement u (TangentSource::Recomputed)."""
        u, pu = _f(u)
        x, px = _f(x)
        y = np.zeros(self.n)
        rc = ref().fxref_apply_operator_at(self.h, k[0], k[1], k[2], int(initial), pu, px, y.ctypes.data_as(p_f64))
        if rc:
            raise RuntimeError(ref().fxref_last_error().decode())
        return y

    def operator_diagonal_at(self, k, u, initial=False):
        u, pu = _f(u)
        d = np.zeros(self.n)
        rc = ref().fxref_operator_diagonal_at(self.h, k[0], k[1], k[2], int(initial), pu, d.ctypes.data_as(p_f64))
        if rc:
            raise RuntimeError(ref().fxref_last_error().decode())
        return d

    def min_critical_dt(self, scheme="ExplicitDifference"):
        return ref().fxref_min_critical_dt(self.h, 1 if scheme == "ExplicitDifference" else 0)

    def element_critical_dts(self, scheme="ExplicitDifference"):
        out = np.zeros(self.c.count)
        k = ref().fxref_element_critical_dts(self.h, 1 if scheme == "ExplicitDifference" else 0,
                                             out.ctypes.data_as(p_f64))
        if k < 0:
            raise RuntimeError(ref().fxref_last_error().decode())
        return out[:k]

    def stability_may_change(self):
        return bool(ref().fxref_stability_may_change(self.h))

    def prepare_stability_bounds(self):
        assert ref().fxref_prepare_stability_bounds(self.h) == 0

    def min_critical_dt_bound(self, scheme="ExplicitDifference"):
        return ref().fxref_min_critical_dt_bound(self.h, 1 if scheme == "ExplicitDifference" else 0)

    def solve(self, b, x0=None, k=(1.0, 0.0, 0.0), method="cg", rtol=1e-10, atol=0.0, max_it=10000, lanes=1,
              restart=30):
        b, pb = _f(b)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        res = (C.c_double * 6)()
        rc = ref().fxref_solve(self.h, 0 if method == "cg" else 1, k[0], k[1], k[2], rtol, atol, max_it, lanes,
                               restart, pb, x.ctypes.data_as(p_f64), res)
        if rc:
            raise RuntimeError(ref().fxref_last_error().decode())
        return x, dict(converged=bool(res[0]), iterations=int(res[1]), rhs_norm=res[2], initial_residual=res[3],
                       final_residual=res[4], indefinite=bool(res[5]))

    def __del__(self):
        if getattr(self, "h", None):
            ref().fxref_force_destroy(self.h)
            self.h = None


def ref_host_dot(x, y, lanes):
    x, px = _f(x)
    y, py = _f(y)
    return ref().fxref_host_dot(px, py, len(x), lanes)


# ------------------------------------------------------------------ the C restatement
class fxo_param(C.Structure):
    _fields_ = [("E", C.c_double), ("nu", C.c_double), ("rho", C.c_double), ("b", C.c_double * 3),
                ("mass_type", C.c_int32), ("pad_", C.c_int32), ("alphaM", C.c_double), ("betaK", C.c_double),
                ("betaKinit", C.c_double), ("betaKcomm", C.c_double)]


class fxo_mesh(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_equations", C.c_int32), ("count", C.c_int32), ("padded", C.c_int32),
                ("num_params", C.c_int32), ("pad_", C.c_int32), ("coords", p_f64), ("node", p_i32), ("eq", p_i32),
                ("param", p_i32), ("params", C.POINTER(fxo_param)), ("nodal_mass", p_f64),
                ("nodal_alpha_mass", p_f64)]


def port():
    global _port
    if _port is None:
        L = C.CDLL(PORT_LIB)
        L.fxo_libm_eval.argtypes = [C.c_int, p_f64, p_f64, p_f64, C.c_int64]
        P = C.POINTER(fxo_param)
        M = C.POINTER(fxo_mesh)
        L.fxo_brick_compute.argtypes = [P, p_f64, p_f64, p_f64, p_f64, p_f64]
        L.fxo_brick_operator.argtypes = [P, p_f64, p_f64, p_f64, p_f64]
        L.fxo_brick_diagonal.argtypes = [P, p_f64, p_f64, p_i32, p_f64]
        L.fxo_brick_mass.argtypes = [P, p_f64, p_f64]
        L.fxo_brick_lumped_mass.argtypes = [P, p_f64, p_f64]
        L.fxo_apply_operator.argtypes = [M, p_f64, p_f64, p_f64]
        L.fxo_operator_diagonal.argtypes = [M, p_f64, p_f64]
        L.fxo_force.argtypes = [M, p_f64, p_f64, p_f64]
        L.fxo_force_j2.argtypes = [M, p_f64, p_f64, p_f64, p_f64, p_f64, p_f64, p_f64, C.POINTER(C.c_int)]
        L.fxo_apply_j2.argtypes = [M, p_f64, p_f64, p_f64, C.c_int, p_f64, p_f64]
        L.fxo_diagonal_j2.argtypes = [M, p_f64, p_f64, p_f64, C.c_int, p_f64]
        L.fxo_mass_times_ground.argtypes = [M, C.c_int, p_f64]
        L.fxo_dot.restype = C.c_double
        L.fxo_dot.argtypes = [p_f64, p_f64, C.c_int64, C.c_int, C.c_int]
        L.fxo_cg.argtypes = [M, p_f64, p_f64, p_f64, C.c_double, C.c_double, C.c_int, C.c_int, p_f64]
        L.fxo_gmres.argtypes = [M, p_f64, p_f64, p_f64, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, p_f64]
        L.fxo_ed_step.argtypes = [M, p_f64, p_i8, p_f64, C.c_double, p_f64, p_f64, p_f64, p_f64, p_f64]
        L.fxo_newmark_predict.argtypes = [C.c_int64, p_f64, p_f64, p_f64, p_f64, p_f64, p_f64, C.c_double, C.c_double,
                                          C.c_double, C.c_double]
        L.fxo_newmark_update.argtypes = [C.c_int64, p_f64, p_f64, p_f64, p_f64, C.c_double, C.c_double]
        L.fxo_j2_update.restype = C.c_int
        L.fxo_j2_update.argtypes = [C.c_double] * 5 + [p_f64, p_f64, p_f64, p_f64, p_f64]
        L.fxo_path_uniform.restype = C.c_double
        L.fxo_path_uniform.argtypes = [p_f64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double]
        L.fxo_path_time.restype = C.c_double
        L.fxo_path_time.argtypes = [p_f64, p_f64, C.c_int64, C.c_double, C.POINTER(C.c_int), C.c_double]
        L.fxo_ed_stage_step.argtypes = [M, p_f64, p_i8, p_f64, p_i32, C.c_int, C.c_double, p_f64, p_f64, p_f64, p_f64,
                                        p_f64]
        L.fxo_cd_stage_step.argtypes = [M, p_f64, p_f64, p_i8, p_f64, p_i32, C.c_int, C.c_double, p_f64, p_f64, p_f64,
                                        p_f64, p_f64, p_f64]
        _port = L
    return _port


def make_param(row) -> fxo_param:
    """fxo_param from a femorax_b200.PARAM_FIELDS row."""
    p = fxo_param()
    p.mass_type = int(row[1])
    p.E, p.nu, p.rho = row[2], row[3], row[4]
    p.b[0], p.b[1], p.b[2] = row[5], row[6], row[7]
    p.alphaM, p.betaK, p.betaKinit, p.betaKcomm = row[8], row[9], row[10], row[11]
    return p


class PortMesh:
    """The C restatement's view of mesh arrays (fields of femorax_b200.MeshArrays)."""

    def __init__(self, m):
        self.keep = []
        s = fxo_mesh()
        s.num_nodes, s.num_equations, s.count, s.padded = m.num_nodes, m.num_equations, m.count, m.padded
        a, s.coords = _f(m.coords)
        self.keep.append(a)
        for name in ("node", "eq", "param"):
            a, p = _i(getattr(m, name))
            self.keep.append(a)
            setattr(s, name, p)
        P = (fxo_param * max(len(m.params), 1))()
        for i, row in enumerate(m.params):
            P[i] = make_param(row)
        self.keep.append(P)
        s.num_params = len(m.params)
        s.params = C.cast(P, C.POINTER(fxo_param))
        for name in ("nodal_mass", "nodal_alpha_mass"):
            v = getattr(m, name, None)
            if v is not None and len(v) and np.any(v != 0):
                a, p = _f(v)
                self.keep.append(a)
                setattr(s, name, p)
        self.s = s
        self.n = m.num_equations
        # J2 table: kind, sigma_y, H, hk per parameter set; per-point arrays [(c * 8 + gp) * padded + e]
        self.j2 = np.ascontiguousarray(np.array([[r[0], r[12], r[13], r[14]] for r in m.params],
                                                np.float64).reshape(-1))
        self.points = 8 * m.padded

    def j2_state(self):
        """A virgin J2 state (13 components per point)."""
        return np.zeros(13 * self.points)

    def force_j2(self, committed, u, v):
        """(f, trial state, point tangents (36 per point), plastic points) at u, v."""
        committed, pc = _f(committed)
        u, pu = _f(u)
        v, pv = _f(v)
        trial = np.zeros(13 * self.points)
        D = np.zeros(36 * self.points)
        f = np.zeros(self.n)
        npl = C.c_int()
        port().fxo_force_j2(C.byref(self.s), self.j2.ctypes.data_as(p_f64), pc, trial.ctypes.data_as(p_f64),
                            D.ctypes.data_as(p_f64), pu, pv, f.ctypes.data_as(p_f64), C.byref(npl))
        return f, trial, D, npl.value

    def apply_j2(self, D, k, x, initial=False):
        D, pD = _f(D)
        k, pk = _f(np.array(k, np.float64))
        x, px = _f(x)
        y = np.zeros(self.n)
        port().fxo_apply_j2(C.byref(self.s), self.j2.ctypes.data_as(p_f64), pD, pk, int(initial), px,
                            y.ctypes.data_as(p_f64))
        return y

    def diagonal_j2(self, D, k, initial=False):
        D, pD = _f(D)
        k, pk = _f(np.array(k, np.float64))
        d = np.zeros(self.n)
        port().fxo_diagonal_j2(C.byref(self.s), self.j2.ctypes.data_as(p_f64), pD, pk, int(initial),
                               d.ctypes.data_as(p_f64))
        return d

    def apply_operator(self, k, x):
        k, pk = _f(np.array(k, np.float64))
        x, px = _f(x)
        y = np.zeros(self.n)
        port().fxo_apply_operator(C.byref(self.s), pk, px, y.ctypes.data_as(p_f64))
        return y

    def operator_diagonal(self, k):
        k, pk = _f(np.array(k, np.float64))
        d = np.zeros(self.n)
        port().fxo_operator_diagonal(C.byref(self.s), pk, d.ctypes.data_as(p_f64))
        return d

    def force(self, u, v):
        u, pu = _f(u)
        v, pv = _f(v)
        f = np.zeros(self.n)
        port().fxo_force(C.byref(self.s), pu, pv, f.ctypes.data_as(p_f64))
        return f

    def mass_times_ground(self, direction):
        y = np.zeros(self.n)
        port().fxo_mass_times_ground(C.byref(self.s), direction, y.ctypes.data_as(p_f64))
        return y

    def cg(self, b, x0=None, k=(1.0, 0.0, 0.0), rtol=1e-10, atol=0.0, max_it=10000, lanes=1):
        k, pk = _f(np.array(k, np.float64))
        b, pb = _f(b)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        r = (C.c_double * 6)()
        port().fxo_cg(C.byref(self.s), pk, pb, x.ctypes.data_as(p_f64), rtol, atol, max_it, lanes, r)
        return x, dict(converged=bool(r[0]), iterations=int(r[1]), rhs_norm=r[2], initial_residual=r[3],
                       final_residual=r[4], indefinite=bool(r[5]))

    def gmres(self, b, x0=None, k=(1.0, 0.0, 0.0), rtol=1e-10, atol=0.0, max_it=10000, lanes=1, restart=30):
        k, pk = _f(np.array(k, np.float64))
        b, pb = _f(b)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        r = (C.c_double * 6)()
        port().fxo_gmres(C.byref(self.s), pk, pb, x.ctypes.data_as(p_f64), rtol, atol, max_it, lanes, restart, r)
        return x, dict(converged=bool(r[0]), iterations=int(r[1]), rhs_norm=r[2], initial_residual=r[3],
                       final_residual=r[4])

    def stage(self, scheme, mass, cm, eq_dof, patterns, dt, steps, time=0.0, u=None, v=None, a=None,
              record_eq=None):
        """An explicit stage as ExplicitAnalysis runs it (src/exec/explicit_analysis.cpp:665-725,
        no LTS, constraints or recorders): ExplicitDifference (scheme 1) starts the half-step
        velocity from the committed one; CentralDifference (scheme 0) starts Utm1 = Ut. Returns
        (u, v_rec, a, time, hist)."""
        n = self.n
        u = np.zeros(n) if u is None else np.array(u, np.float64)
        v = np.zeros(n) if v is None else np.array(v, np.float64)
        a = np.zeros(n) if a is None else np.array(a, np.float64)
        f = np.zeros(n)
        m, pm = _f(mass)
        c, pc = _f(cm)
        dof = np.ascontiguousarray(eq_dof, np.int8)
        mot = PortMotions(patterns)
        gd, pgd = mot.dof, mot.dof.ctypes.data_as(p_i32)
        P = lambda x: x.ctypes.data_as(p_f64)
        hist = []
        if scheme == 1:
            vh = v.copy()
        else:
            um = u.copy()
            ve = np.zeros(n)
        for _ in range(steps):
            if scheme == 1:
                time += dt
                g, pg = _f(mot.evaluate(time))
                port().fxo_ed_stage_step(C.byref(self.s), pm, dof.ctypes.data_as(p_i8), pg, pgd, len(gd), dt, P(u),
                                         P(vh), P(a), P(v), P(f))
            else:
                g, pg = _f(mot.evaluate(time))
                port().fxo_cd_stage_step(C.byref(self.s), pm, pc, dof.ctypes.data_as(p_i8), pg, pgd, len(gd), dt,
                                         P(u), P(um), P(ve), P(a), P(v), P(f))
                time += dt
            if record_eq is not None:
                hist.append(a[record_eq])
        return u, v, a, time, np.array(hist)

    def ed_steps(self, mass, eq_dof, dt, steps, ag=None, direction=0, u=None, vh=None, a=None, record_eq=None):
        n = self.n
        u = np.zeros(n) if u is None else u.copy()
        vh = np.zeros(n) if vh is None else vh.copy()
        a = np.zeros(n) if a is None else a.copy()
        v = np.zeros(n)
        f = np.zeros(n)
        m, pm = _f(mass)
        dof = np.ascontiguousarray(eq_dof, np.int8)
        hist = []
        for s in range(steps):
            g = np.zeros(3)
            if ag is not None:
                g[direction] = ag[s]
            g, pg = _f(g)
            port().fxo_ed_step(C.byref(self.s), pm, dof.ctypes.data_as(p_i8), pg, dt, u.ctypes.data_as(p_f64),
                               vh.ctypes.data_as(p_f64), a.ctypes.data_as(p_f64), v.ctypes.data_as(p_f64),
                               f.ctypes.data_as(p_f64))
            if record_eq is not None:
                hist.append(a[record_eq])
        return u, vh, a, v, np.array(hist)


class PortMotions:
    """UniformExcitation patterns evaluated by the port's restatement of GroundMotions::evaluate
    (src/exec/ground_motion.cpp:150-175): accel[p] = fact_p * series_p(t), 0 for t < 0. A pattern
    is a dict: dof (0-based), fact, values, and dt (PathSeries) or times (PathTimeSeries), factor,
    use_last, prepend_zero."""

    def __init__(self, patterns):
        self.patterns = [dict(p) for p in patterns]
        self.loc = [C.c_int(0) for _ in self.patterns]
        self.dof = np.array([p["dof"] for p in self.patterns], np.int32)

    def evaluate(self, t):
        out = np.zeros(len(self.patterns))
        for i, p in enumerate(self.patterns):
            a = 0.0
            if t >= 0.0:
                vals = np.asarray(p["values"], np.float64)
                if p.get("times") is None:
                    if p.get("prepend_zero"):
                        vals = np.concatenate([[0.0], vals])
                    v, pv = _f(vals)
                    a = port().fxo_path_uniform(pv, len(v), p["dt"], p.get("factor", 1.0), 0.0,
                                                int(bool(p.get("use_last"))), t)
                else:
                    v, pv = _f(vals)
                    tm, pt = _f(p["times"])
                    a = port().fxo_path_time(pv, pt, len(v), p.get("factor", 1.0), C.byref(self.loc[i]), t)
            out[i] = p["fact"] * a
        return out


class RefMotions:
    """The same patterns through the reference's own exec::GroundMotions (oracle/_ref)."""

    def __init__(self, patterns):
        self.n = len(patterns)
        self.h = ref().fxref_motions_create()
        for p in patterns:
            v, pv = _f(p["values"])
            if p.get("times") is None:
                pt, dt = None, p["dt"]
            else:
                tm, pt = _f(p["times"])
                dt = 0.0
            rc = ref().fxref_motions_add(self.h, p["dof"], p["fact"], pv, pt, len(v), dt, p.get("factor", 1.0),
                                         int(bool(p.get("use_last"))), int(bool(p.get("prepend_zero"))))
            assert rc == 0, ref().fxref_last_error()

    def evaluate(self, t):
        out = np.zeros(self.n)
        rc = ref().fxref_motions_evaluate(self.h, t, out.ctypes.data_as(p_f64))
        assert rc == 0, ref().fxref_last_error()
        return out

    def __del__(self):
        if getattr(self, "h", None):
            ref().fxref_motions_destroy(self.h)


class RefPimy:
    """The reference's PressureIndependMultiYield (40-surface bucket) at one material point
    (oracle/_ref): params9 = rho, refShearModul, refBulkModul, cohesi, peakShearStra, frictionAng,
    refPress, pressDependCoe, noYieldSurf; pairs: (gamma, G/Gmax) pairs or empty."""

    def __init__(self, params9, pairs=()):
        p9, pp = _f(params9)
        pr = np.ascontiguousarray(pairs, np.float64)
        h = vp()
        rc = ref().fxref_pimy_create(pp, pr.ctypes.data_as(p_f64) if pr.size else None, pr.size // 2, C.byref(h))
        assert rc == 0, rc
        self.h = h
        self.nstate = ref().fxref_pimy_nstate()

    def setup_values(self):
        """residualPress, frictionAngle, cohesion; surface sizes and plastic moduli (1..40)."""
        out = np.zeros(83)
        ref().fxref_pimy_setup_values(self.h, out.ctypes.data_as(p_f64))
        return out[:3], out[3:43], out[43:83]

    def initial_state(self):
        s = np.zeros(self.nstate)
        ref().fxref_pimy_initial_state(self.h, s.ctypes.data_as(p_f64))
        return s

    def update(self, stage, committed, eps):
        """(trial state, stress, tangent) at total strain eps from the committed state."""
        committed, pc = _f(committed)
        eps, pe = _f(eps)
        trial, sig, D = np.zeros(self.nstate), np.zeros(6), np.zeros((6, 6))
        ref().fxref_pimy_update(self.h, stage, pc, trial.ctypes.data_as(p_f64), pe, sig.ctypes.data_as(p_f64),
                                D.ctypes.data_as(p_f64))
        return trial, sig, D

    def replay(self, stage, pre, pre_eps, eps):
        """A golden path: per step the stage, an optional discarded trial, the update, the commit.
        Returns the stresses [n, 6] and tangents [n, 6, 6]."""
        c = self.initial_state()
        sig, D = np.zeros((len(eps), 6)), np.zeros((len(eps), 6, 6))
        for k in range(len(eps)):
            if pre[k]:
                self.update(int(stage[k]), c, pre_eps[k])
            c, sig[k], D[k] = self.update(int(stage[k]), c, eps[k])
        return sig, D

    def __del__(self):
        if getattr(self, "h", None):
            ref().fxref_pimy_destroy(self.h)


class RefPdmy(RefPimy):
    """The reference's PressureDependMultiYield (40-surface bucket) at one material point
    (oracle/_ref): params23 = the 21 constructor values of the stored paths' header (rho ... c)
    then hv, pv; pairs: (gamma, G/Gmax) pairs or empty. math: "libm" (the C library's elementary
    functions, as the reference ships) or "fx" (pow, exp, log and cos bound to those of this
    library's device update, oracle/_ref/libfxref_fxmath.so)."""

    def __init__(self, params23, pairs=(), math="libm"):
        self.L = ref(math)
        p, pp = _f(params23)
        pr = np.ascontiguousarray(pairs, np.float64)
        h = vp()
        rc = self.L.fxref_pdmy_create(pp, pr.ctypes.data_as(p_f64) if pr.size else None, pr.size // 2, C.byref(h))
        assert rc == 0, rc
        self.h = h
        self.nstate = self.L.fxref_pdmy_nstate()

    def setup_values(self):
        """residualPress, frictionAngle, phaseTransfAngle, stressRatioPT, strainPTOcta; sizes and
        plastic moduli (1..40)."""
        out = np.zeros(85)
        self.L.fxref_pdmy_setup_values(self.h, out.ctypes.data_as(p_f64))
        return out[:5], out[5:45], out[45:85]

    def initial_state(self):
        s = np.zeros(self.nstate)
        self.L.fxref_pdmy_initial_state(self.h, s.ctypes.data_as(p_f64))
        return s

    def update(self, stage, committed, eps):
        committed, pc = _f(committed)
        eps, pe = _f(eps)
        trial, sig, D = np.zeros(self.nstate), np.zeros(6), np.zeros((6, 6))
        self.L.fxref_pdmy_update(self.h, stage, pc, trial.ctypes.data_as(p_f64), pe, sig.ctypes.data_as(p_f64),
                                D.ctypes.data_as(p_f64))
        return trial, sig, D

    def __del__(self):
        if getattr(self, "h", None):
            self.L.fxref_pdmy_destroy(self.h)
            self.h = None


def libm_eval(fn: int, x, y=None):
    """The host C library's exp (0), log (1), pow (2) or cos (3) of x (and y), element by element."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(x if y is None else y, np.float64)
    out = np.empty_like(x)
    port().fxo_libm_eval(fn, x.ctypes.data_as(p_f64), y.ctypes.data_as(p_f64), out.ctypes.data_as(p_f64), x.size)
    return out


def ref_ssp_constants(xl, E, nu):
    """The reference's SSPbrick geometry record (33) and element constants (110) of one element."""
    xl, px = _f(np.asarray(xl, np.float64).reshape(3, 8))
    geo, con = np.zeros(33), np.zeros(110)
    ref().fxref_ssp_constants(px, E, nu, geo.ctypes.data_as(p_f64), con.ctypes.data_as(p_f64))
    return geo, con


def port_dot(x, y, lanes, fused):
    x, px = _f(x)
    y, py = _f(y)
    return port().fxo_dot(px, py, len(x), lanes, int(fused))


def port_brick_compute(row, damp, xe, u, v, want_k=True):
    p = make_param(row)
    p.alphaM, p.betaK, p.betaKinit, p.betaKcomm = damp
    xe, px = _f(xe)
    u, pu = _f(u)
    v, pv = _f(v)
    fe = np.zeros(24)
    Ke = np.zeros(576) if want_k else None
    port().fxo_brick_compute(C.byref(p), px, pu, pv, fe.ctypes.data_as(p_f64),
                             Ke.ctypes.data_as(p_f64) if want_k else None)
    return fe, (Ke.reshape(24, 24) if want_k else None)


def port_brick_mass(row, xe):
    p = make_param(row)
    xe, px = _f(xe)
    Me = np.zeros(576)
    port().fxo_brick_mass(C.byref(p), px, Me.ctypes.data_as(p_f64))
    return Me.reshape(24, 24)


def port_brick_operator(row, damp, k, xe, ve):
    p = make_param(row)
    p.alphaM, p.betaK, p.betaKinit, p.betaKcomm = damp
    k, pk = _f(np.array(k, np.float64))
    xe, px = _f(xe)
    ve, pv = _f(ve)
    ye = np.zeros(24)
    port().fxo_brick_operator(C.byref(p), pk, px, pv, ye.ctypes.data_as(p_f64))
    return ye


def port_j2(E, nu, sy, H, hk, committed, eps):
    committed, pc = _f(committed)
    eps, pe = _f(eps)
    trial = np.zeros(13)
    sig = np.zeros(6)
    D = np.zeros(36)
    plastic = port().fxo_j2_update(E, nu, sy, H, hk, pc, trial.ctypes.data_as(p_f64), pe, sig.ctypes.data_as(p_f64),
                                   D.ctypes.data_as(p_f64))
    return sig, D.reshape(6, 6), trial, bool(plastic)
