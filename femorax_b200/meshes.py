"""In-memory model descriptions (the fields of the reference's io::Model the hot path reads) and
builders for structured hex8 blocks: nodes on a grid, stdBrick elements in stdBrick corner
order, materials per element group, fixes, Rayleigh regions.

A ``ModelSpec`` feeds both this library's compile step (``femorax_b200.Model``) and the oracle
(the reference's own compile step), so the two can be compared array by array.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Group:
    """One stdBrick element group with its own material (io::ElementGroup + NDMaterial)."""
    E: float
    nu: float
    rho: float
    etags: np.ndarray  # [M] int32
    conn: np.ndarray  # [M, 8] int32 node tags, stdBrick order
    b: tuple = (0.0, 0.0, 0.0)
    lumped: bool = False
    kind: int = 0  # 0 ElasticIsotropic, 1 J2
    element: int = 0  # 0 stdBrick, 1 SSPbrick (one point, physical stabilization; always lumped)
    sigma_y: float = 0.0
    H: float = 0.0
    hk: float = 0.0
    # PressureIndependMultiYield: (the 9 constructor values, pairs or None). The library compiles
    # the group as an elastic set (E, nu, rho) and binds the material to its parameter set
    # (InternalForce.set_pimy); the reference's model gets the material itself.
    pimy: tuple = None
    pdmy: tuple = None  # PressureDependMultiYield: (the 23 values of fx_pdmy_create, pairs or None), likewise


@dataclasses.dataclass
class Rayleigh:
    alphaM: float
    betaK: float
    betaKinit: float
    betaKcomm: float
    etags: np.ndarray


@dataclasses.dataclass
class ModelSpec:
    tags: np.ndarray  # [N] int32
    coords: np.ndarray  # [N, 3] float64
    groups: list
    fix_node: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    fix_dof: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    eqd_retained: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    eqd_constrained: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    eqd_dof: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    rayleigh: list = dataclasses.field(default_factory=list)
    mass_node: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    mass_dof: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))
    mass_value: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.float64))
    grid: tuple = None  # (nx, ny, nz, hx, hy, hz) for structured blocks

    @property
    def num_elements(self) -> int:
        return sum(len(g.etags) for g in self.groups)


def node_tag(i, j, k, nx, ny):
    """Tag of grid node (i, j, k): 1 + i + (nx+1) (j + (ny+1) k)."""
    return 1 + i + (nx + 1) * (j + (ny + 1) * k)


def block_connectivity(nx, ny, nz, k0=0, k1=None):
    """Element tags (1-based, lexicographic i fastest) and stdBrick connectivity of element
    layers k0 <= k < k1 of an nx x ny x nz grid."""
    k1 = nz if k1 is None else k1
    k, j, i = np.meshgrid(np.arange(k0, k1), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    t = lambda a, b, c: node_tag(a, b, c, nx, ny)
    conn = np.stack([t(i, j, k), t(i + 1, j, k), t(i + 1, j + 1, k), t(i, j + 1, k),
                     t(i, j, k + 1), t(i + 1, j, k + 1), t(i + 1, j + 1, k + 1), t(i, j + 1, k + 1)],
                    axis=1).astype(np.int32)
    etags = (1 + i + nx * (j + ny * k)).astype(np.int32)
    return etags, conn


def block_nodes(nx, ny, nz, hx, hy, hz, origin=(0.0, 0.0, 0.0)):
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    tags = node_tag(i, j, k, nx, ny).astype(np.int32)
    coords = np.stack([origin[0] + i * hx, origin[1] + j * hy, origin[2] + k * hz], axis=1).astype(np.float64)
    return tags, coords


def fix_base(nx, ny):
    """All three DOFs of the nodes at k = 0."""
    j, i = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    nodes = node_tag(i.ravel(), j.ravel(), 0, nx, ny).astype(np.int32)
    return np.repeat(nodes, 3), np.tile(np.array([1, 2, 3], np.int32), len(nodes))


def box_model(nx, ny, nz, size=(1.0, 1.0, 1.0), E=50e6, nu=0.3, rho=2000.0, lumped=False, b=(0.0, 0.0, 0.0),
              fixed_base=True, kind=0, sigma_y=0.0, H=0.0, hk=0.0):
    """One material over an nx x ny x nz block of size `size` (metres), base z = 0 fixed; kind 1
    makes it J2 with yield stress sigma_y, hardening H and kinematic share hk."""
    hx, hy, hz = size[0] / nx, size[1] / ny, size[2] / nz
    tags, coords = block_nodes(nx, ny, nz, hx, hy, hz)
    etags, conn = block_connectivity(nx, ny, nz)
    group = Group(E, nu, rho, etags, conn, b=b, lumped=lumped, kind=kind, sigma_y=sigma_y, H=H, hk=hk)
    spec = ModelSpec(tags=tags, coords=coords, groups=[group], grid=(nx, ny, nz, hx, hy, hz))
    if fixed_base:
        spec.fix_node, spec.fix_dof = fix_base(nx, ny)
    return spec


# ------------------------------------------------------------------ the benchmark configurations
def static_cube(n=32, E=50e6, nu=0.3, rho=2000.0):
    """Static linear-elastic block: n^3 stdBrick on a 1 m cube, E = 50 MPa, nu = 0.3, base fixed."""
    return box_model(n, n, n, (1.0, 1.0, 1.0), E=E, nu=nu, rho=rho)


def top_traction_rhs(spec, eq_of, q=-100e3):
    """Equation-space load of a uniform vertical traction q (Pa) on the top face z = max:
    each top quad gives q h^2 / 4 to each of its 4 nodes (the harness builds this RHS: the
    reference's model file has no surface loads). eq_of(node_tag, dof) -> equation or -1."""
    nx, ny, nz, hx, hy, _ = spec.grid
    f = {}
    share = q * hx * hy / 4.0
    for j in range(ny):
        for i in range(nx):
            for (a, c) in ((i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)):
                t = node_tag(a, c, nz, nx, ny)
                f[t] = f.get(t, 0.0) + share
    return f


def equation_map(compiled):
    """eq[tag, dof]: the equation of (node tag, dof 0..2), -1 fixed, from a compile step's arrays
    (`node_tag`, `dof_offset`, `eq` by name: this library's Compiled or the reference's)."""
    tags = compiled.array("node_tag")
    off = compiled.array("dof_offset")
    eq = compiled.array("eq")
    out = np.full((int(tags.max()) + 1, 3), -1, dtype=np.int64)
    for d in range(3):
        out[tags, d] = eq[off[:-1] + d]
    return out


def top_traction_vector(spec, eqmap, neq, q=-100e3):
    """top_traction_rhs as an equation-space vector of neq entries (vertical DOF of each top node)."""
    b = np.zeros(neq)
    for tag, f in top_traction_rhs(spec, None, q).items():
        e = int(eqmap[tag, 2])
        if e >= 0:
            b[e] += f
    return b


def rayleigh_coefficients(xi, f1, f2):
    """alphaM, betaK for damping ratio xi at frequencies f1 and f2 (Hz)."""
    w1, w2 = 2 * math.pi * f1, 2 * math.pi * f2
    return 2 * xi * w1 * w2 / (w1 + w2), 2 * xi / (w1 + w2)


def layered_box(nx=128, ny=128, nz=64, layers=8, h=1.0, seed=0, lumped=True, damping=(0.02, 1.0, 10.0)):
    """Layered soil box (explicit wave propagation): nx x ny x nz elements of h metres, `layers`
    horizontal layers with Vs ~ U[150, 600] m/s, rho ~ U[1800, 2100] kg/m^3, nu ~ U[0.30, 0.45]
    from `seed`, G = rho Vs^2, E = 2 G (1 + nu); lumped mass; Rayleigh 2 % at 1 and 10 Hz; base
    fixed. Returns (spec, layer properties)."""
    rng = np.random.default_rng(seed)
    tags, coords = block_nodes(nx, ny, nz, h, h, h)
    groups = []
    props = []
    per = nz // layers
    for L in range(layers):
        vs = rng.uniform(150.0, 600.0)
        rho = rng.uniform(1800.0, 2100.0)
        nu = rng.uniform(0.30, 0.45)
        G = rho * vs * vs
        E = 2.0 * G * (1.0 + nu)
        k0, k1 = L * per, (L + 1) * per if L < layers - 1 else nz
        et, cn = block_connectivity(nx, ny, nz, k0, k1)
        groups.append(Group(E, nu, rho, et, cn, lumped=lumped))
        props.append(dict(vs=vs, rho=rho, nu=nu, E=E))
    spec = ModelSpec(tags=tags, coords=coords, groups=groups, grid=(nx, ny, nz, h, h, h))
    spec.fix_node, spec.fix_dof = fix_base(nx, ny)
    if damping:
        aM, bK = rayleigh_coefficients(*damping)
        all_e = np.concatenate([g.etags for g in groups])
        spec.rayleigh.append(Rayleigh(aM, bK, 0.0, 0.0, all_e))
    return spec, props


def heterogeneous_cube(n=100, median_E=80e6, sigma=0.5, nu=0.3, rho=2000.0, seed=0, size=1.0):
    """Heterogeneous elastic cube: n^3 elements, per-element E log-normal (median 80 MPa,
    sigma 0.5) from `seed`, nu = 0.3, base fixed. Each element is a group with its own material,
    as a model file with per-element materials holds it."""
    rng = np.random.default_rng(seed)
    h = size / n
    tags, coords = block_nodes(n, n, n, h, h, h)
    etags, conn = block_connectivity(n, n, n)
    Es = median_E * np.exp(sigma * rng.standard_normal(len(etags)))
    groups = [Group(float(Es[e]), nu, rho, etags[e:e + 1], conn[e:e + 1]) for e in range(len(etags))]
    spec = ModelSpec(tags=tags, coords=coords, groups=groups, grid=(n, n, n, h, h, h))
    spec.fix_node, spec.fix_dof = fix_base(n, n)
    return spec


def laminar_column(nx=2, ny=2, nz=8, dx=1.0, dy=1.0, dz=0.5, lumped=True, damping=True, element=0):
    """The layered soil column of the reference's tests and benchmarks (tests/common/
    synthetic_models.hpp:24-94): nx x ny x nz bricks (stdBrick, or SSPbrick with element 1, always
    lumped) of dx x dy x dz with the top at z = 0, a lower and an upper material (E 377 and 109.2 kPa,
    nu 0.3), body force, base fixed, the side nodes of every elevation above the base tied to the
    first side node in DOFs 1 2 3 (equalDOF stars), Rayleigh damping over everything and a second
    region over the top layer (the later region wins)."""
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    tags, coords = block_nodes(nx, ny, nz, dx, dy, dz, origin=(0.0, 0.0, -nz * dz))
    groups = []
    for layer in range(2):
        k0, k1 = (0, nz // 2) if layer == 0 else (nz // 2, nz)
        et, cn = block_connectivity(nx, ny, nz, k0, k1)
        groups.append(Group(377000.0 if layer == 0 else 109200.0, 0.3, 2.0285 if layer == 0 else 2.0183, et, cn,
                            b=(0.0, 0.0, -19.9 if layer == 0 else -19.8), lumped=lumped or element == 1,
                            element=element))
    spec = ModelSpec(tags=tags, coords=coords, groups=groups)
    spec.fix_node, spec.fix_dof = fix_base(nx, ny)
    ret, con, dof = [], [], []
    for k in range(1, NZ):
        master = -1
        for j in range(NY):
            for i in range(NX):
                if not (i == 0 or i == nx or j == 0 or j == ny):
                    continue
                t = node_tag(i, j, k, nx, ny)
                if master < 0:
                    master = t
                    continue
                for d in (1, 2, 3):
                    ret.append(master)
                    con.append(t)
                    dof.append(d)
    spec.eqd_retained, spec.eqd_constrained, spec.eqd_dof = [np.array(a, np.int32) for a in (ret, con, dof)]
    if damping:
        all_e = np.concatenate([g.etags for g in groups])
        spec.rayleigh = [Rayleigh(0.6, 5.8e-4, 0.0, 0.0, all_e),
                         Rayleigh(0.9, 3e-4, 1e-4, 0.0, groups[1].etags[-nx * ny:])]
    return spec


def ricker(t, f0=5.0, t0=None, amplitude=1.0):
    """Ricker wavelet of peak frequency f0 (Hz), centred at t0 (default 1.2 / f0)."""
    t0 = 1.2 / f0 if t0 is None else t0
    a = (math.pi * f0 * (np.asarray(t) - t0)) ** 2
    return amplitude * (1.0 - 2.0 * a) * np.exp(-a)


def distort(spec, amount, seed=0):
    """Perturb every node not on the fixed base by up to `amount` times the spacing (a general,
    non-box mesh for the Gauss-point path)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz, hx, hy, hz = spec.grid
    c = spec.coords.copy()
    free = c[:, 2] > 0
    c[free] += amount * np.array([hx, hy, hz]) * rng.uniform(-1, 1, (int(free.sum()), 3))
    out = dataclasses.replace(spec, coords=c, grid=None)
    return out
