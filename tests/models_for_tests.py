"""Small models the tests share: the reference's synthetic soil column shape (two materials,
laminar equalDOF ties at every elevation, two Rayleigh regions, body force, lumped mass) and a
block with two overlapping Rayleigh regions and nodal masses."""
import numpy as np

from femorax_b200 import meshes


def soil_column(nx=3, ny=2, nz=8, lumped=True):
    """The layered column the reference's tests build in memory (tests/common/synthetic_models.hpp
    shape; meshes.laminar_column): stdBrick, lower and upper material, fixed base, side nodes at
    each elevation tied to the first side node in DOFs 1 2 3, a Rayleigh region over everything and
    one over the top layer."""
    return meshes.laminar_column(nx, ny, nz, lumped=lumped)


def two_region_block(nx=4, ny=3, nz=5, lumped=False):
    """A consistent-mass block with two overlapping Rayleigh regions (all four factors used)
    and nodal masses on a few nodes."""
    spec = meshes.box_model(nx, ny, nz, (2.0, 1.5, 2.5), E=2.0e5, nu=0.25, rho=1.9, lumped=lumped, b=(0.1, -0.2, -9.8))
    et = spec.groups[0].etags
    spec.rayleigh = [meshes.Rayleigh(0.3, 1e-3, 0.0, 0.0, et), meshes.Rayleigh(0.5, 2e-3, 5e-4, 1e-4, et[::3])]
    top = [meshes.node_tag(i, j, nz, nx, ny) for i in (0, nx) for j in (0, ny)]
    spec.mass_node = np.repeat(np.array(top, np.int32), 3)
    spec.mass_dof = np.tile(np.array([1, 2, 3], np.int32), len(top))
    spec.mass_value = np.linspace(0.5, 2.0, len(spec.mass_node))
    return spec


def j2_column(nx=2, ny=3, nz=6, lumped=False, hk=0.5, h=0.5):
    """A column with an elastic lower half and a J2 upper half (sigma_y 60 kPa, H = 0.05 E, kinematic
    share hk), base fixed, mass-proportional Rayleigh damping on the J2 half."""
    tags, coords = meshes.block_nodes(nx, ny, nz, h, h, h)
    groups = []
    for layer in range(2):
        k0, k1 = (0, nz // 2) if layer == 0 else (nz // 2, nz)
        et, cn = meshes.block_connectivity(nx, ny, nz, k0, k1)
        if layer == 0:
            groups.append(meshes.Group(80e6, 0.3, 2000.0, et, cn, b=(0.0, 0.0, -19.6e3), lumped=lumped))
        else:
            groups.append(meshes.Group(40e6, 0.33, 1900.0, et, cn, b=(0.0, 0.0, -18.6e3), lumped=lumped, kind=1,
                                       sigma_y=60e3, H=0.05 * 40e6, hk=hk))
    spec = meshes.ModelSpec(tags=tags, coords=coords, groups=groups)
    spec.fix_node, spec.fix_dof = meshes.fix_base(nx, ny)
    spec.rayleigh = [meshes.Rayleigh(0.4, 0.0, 0.0, 0.0, groups[1].etags)]
    spec.grid = (nx, ny, nz, h, h, h)
    return spec



def roller_block(nx=5, ny=4, nz=6):
    """A box-grid block on rollers: base fixed, the x faces fixed in x and the y faces in y, so
    side nodes keep two free DOFs and corner columns one (nodes neither fully free nor fixed)."""
    spec = meshes.box_model(nx, ny, nz, (2.0, 1.5, 3.0), E=3.0e5, nu=0.3, rho=1.8, lumped=False)
    nodes, dofs = [], []
    for k in range(1, nz + 1):
        for j in range(ny + 1):
            for i in (0, nx):
                nodes.append(meshes.node_tag(i, j, k, nx, ny))
                dofs.append(1)
        for i in range(nx + 1):
            for j in (0, ny):
                nodes.append(meshes.node_tag(i, j, k, nx, ny))
                dofs.append(2)
    spec.fix_node = np.concatenate([spec.fix_node, np.array(nodes, np.int32)])
    spec.fix_dof = np.concatenate([spec.fix_dof, np.array(dofs, np.int32)])
    return spec


def as_ssp(spec):
    """The same model with every group an SSPbrick group (lumped by construction)."""
    for g in spec.groups:
        g.element = 1
        g.lumped = True
    return spec


def ssp_block(nx=4, ny=3, nz=5, distort=0.0, seed=0):
    """An SSPbrick block on a fixed base (optionally distorted: a general mesh), two Rayleigh regions
    (all four factors) and a body force."""
    spec = meshes.box_model(nx, ny, nz, (2.0, 1.5, 2.5), E=2.0e5, nu=0.3, rho=1.9, lumped=True, b=(0.1, -0.2, -9.8))
    if distort:
        spec = meshes.distort(spec, distort, seed=seed)
    as_ssp(spec)
    et = spec.groups[0].etags
    spec.rayleigh = [meshes.Rayleigh(0.3, 1e-3, 0.0, 0.0, et), meshes.Rayleigh(0.5, 2e-3, 5e-4, 1e-4, et[::3])]
    return spec
