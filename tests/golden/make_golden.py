"""Generates the committed golden fixtures of tests/golden/ (run in the build container, where
the reference checkout and the oracle library exist):

  brick_elements.npz  the reference's stored OpenSees Brick data for stdBrick
                      (tests/reference/data/element/Brick_*_{state,mass}.txt, read as text):
                      per case the coordinates, material, body force, Rayleigh factors, the four
                      (u, v) fields and f, K, damping forces (consistent, lumped), and the
                      consistent and lumped mass matrices.
  compile_maps.npz    the reference's compile_model output (oracle/_ref/libfxref.so) for two
                      small models: a 4 x 3 x 5 block with two Rayleigh regions (RCM, coloring)
                      and a 3 x 2 x 8 soil column with laminar equalDOF ties.
  compile_digests.json  sha256 digests of every compile_model array (oracle/_ref/libfxref.so)
                      for the three benchmark configurations' models (the 32^3 static cube,
                      the 128 x 128 x 64 layered box, the 100^3 per-element-E cube).
  pdmy_paths.npz      the same for PressureDependMultiYield (tests/reference/data/nd/
                      PressureDependMultiYield_*.txt).
  pimy_paths.npz      the reference's stored OpenSees PressureIndependMultiYield strain paths
                      (tests/reference/data/nd/PressureIndependMultiYield_*.txt, read as text):
                      per path the material's parameters and backbone pairs, and per step the
                      load stage, the discarded trial strain (if any), the strain, and OpenSees'
                      stress and tangent.

    FEMORAX_REFERENCE=<reference checkout> python tests/golden/make_golden.py [bricks|compile_maps|pimy_paths|pdmy_paths ...]
"""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
REFERENCE = os.environ.get("FEMORAX_REFERENCE", "")  # the reference checkout (read as text)
DATA = os.path.join(REFERENCE, "tests/reference/data/element")
ND = os.path.join(REFERENCE, "tests/reference/data/nd")
PDMY_PARAMS = ("rho", "refShearModul", "refBulkModul", "frictionAng", "peakShearStra", "refPress", "pressDependCoe",
               "PTAng", "contrac", "dilat1", "dilat2", "liquefac1", "liquefac2", "liquefac3", "noYieldSurf", "e", "cs1",
               "cs2", "cs3", "pa", "c")
PIMY_PARAMS = ("rho", "refShearModul", "refBulkModul", "cohesi", "peakShearStra", "frictionAng", "refPress",
               "pressDependCoe", "noYieldSurf")


def read_reference_file(path):
    header, rows = {}, []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                parts = line[1:].split()
                if parts:
                    header[parts[0]] = parts[1:]
            elif line.strip():
                rows.append([float(v) for v in line.split()])
    return header, np.array(rows)


def bricks():
    out = {}
    cases = []
    for state in sorted(glob.glob(os.path.join(DATA, "Brick_*_state.txt"))):
        name = os.path.basename(state)[len("Brick_"):-len("_state.txt")]
        h, rows = read_reference_file(state)
        cols = h["columns"]
        col = {c: i for i, c in enumerate(cols)}
        p = h["params"]
        params = dict(zip(p[0::2], map(float, p[1::2])))
        coords = np.array(list(map(float, h["coords"]))).reshape(8, 3)
        body = np.array(list(map(float, h["body_force"])))
        ray = np.array(list(map(float, h["rayleigh"])))

        def block(prefix, n):
            return rows[:, col[prefix + "0"]:col[prefix + "0"] + n]

        hm, mrows = read_reference_file(state.replace("_state.txt", "_mass.txt"))
        mcol = {c: i for i, c in enumerate(hm["columns"])}
        Mc = mrows[0, mcol["Mc0"]:mcol["Mc0"] + 576].reshape(24, 24)
        Ml = mrows[0, mcol["Ml0"]:mcol["Ml0"] + 576].reshape(24, 24)
        out[name + "/coords"] = coords
        out[name + "/material"] = np.array([params["E"], params["nu"], params["rho"]])
        out[name + "/body"] = body
        out[name + "/rayleigh"] = ray
        out[name + "/u"] = block("u", 24)
        out[name + "/v"] = block("v", 24)
        out[name + "/f"] = block("f", 24)
        out[name + "/K"] = block("K", 576).reshape(-1, 24, 24)
        out[name + "/dc"] = block("dc", 24)
        out[name + "/dl"] = block("dl", 24)
        out[name + "/Mc"] = Mc
        out[name + "/Ml"] = Ml
        cases.append(name)
    out["cases"] = np.array(cases)
    np.savez_compressed(os.path.join(HERE, "brick_elements.npz"), **out)
    print("brick_elements.npz:", len(cases), "cases")


def compile_maps():
    import oracle as O
    from femorax_b200 import meshes
    from tests.models_for_tests import soil_column, two_region_block
    out = {}
    for name, spec, kw in (("block", two_region_block(), dict(renumbering="rcm", simd_width=32, coloring=True)),
                           ("column", soil_column(), dict(renumbering="rcm", simd_width=32, coloring=True))):
        c = O.RefModel(spec).compile(**kw)
        for a in O.RefCompiled.I32:
            out[f"{name}/{a}"] = c.array(a)
        for a in ("coords", "lumped_mass", "lumped_alpha_mass", "nodal_mass", "nodal_alpha_mass"):
            out[f"{name}/{a}"] = c.array(a)
        out[f"{name}/params"] = c.params()
    np.savez_compressed(os.path.join(HERE, "compile_maps.npz"), **out)
    print("compile_maps.npz written")


CONFIG_MODELS = ("static_cube_32", "layered_box_128x128x64", "heterogeneous_cube_100")


def config_model(name):
    """The models of the benchmark configurations: the 32^3 static cube, the 128 x 128 x 64 layered
    box (seed 0) and the 100^3 cube with per-element E (seed 0)."""
    from femorax_b200 import meshes
    if name == "static_cube_32":
        return meshes.static_cube(32)
    if name == "layered_box_128x128x64":
        return meshes.layered_box(128, 128, 64, 8, seed=0)[0]
    return meshes.heterogeneous_cube(100, seed=0, size=50.0)


def array_digest(a):
    """sha256 of an array's dtype, shape and little-endian bytes."""
    import hashlib
    a = np.ascontiguousarray(a)
    h = hashlib.sha256(f"{a.dtype.str}{a.shape}".encode())
    h.update(a.astype(a.dtype.newbyteorder("<")).tobytes())
    return h.hexdigest()


def compile_digests():
    """compile_digests.json: digests of every array the reference's compile_model returns (RCM,
    SIMD width 32) for the benchmark configurations' models; the arrays themselves are too large
    to commit."""
    import json
    import oracle as O
    out = {}
    for name in CONFIG_MODELS:
        c = O.RefModel(config_model(name)).compile(renumbering="rcm", simd_width=32)
        names = O.RefCompiled.I32 + ("coords", "lumped_mass", "lumped_alpha_mass", "nodal_mass", "nodal_alpha_mass")
        out[name] = {a: array_digest(c.array(a)) for a in names}
    json.dump(out, open(os.path.join(HERE, "compile_digests.json"), "w"), indent=1, sort_keys=True)
    print("compile_digests.json written")


def pimy_paths(material="PressureIndependMultiYield", names=None, out_name="pimy_paths.npz"):
    names = names or PIMY_PARAMS
    out, cases = {}, []
    for path in sorted(glob.glob(os.path.join(ND, material + "_*.txt"))):
        name = os.path.basename(path)[len(material) + 1:-len(".txt")]
        h, rows = read_reference_file(path)
        col = {c: i for i, c in enumerate(h["columns"])}
        p = h["params"]
        params = dict(zip(p[0::2], map(float, p[1::2])))
        out[name + "/params"] = np.array([params[k] for k in names])
        out[name + "/pairs"] = np.array(list(map(float, h.get("pairs", []))))
        out[name + "/stage"] = rows[:, col["stage"]].astype(np.int8)
        out[name + "/pre"] = rows[:, col["pre"]].astype(np.int8)
        out[name + "/pre_eps"] = rows[:, col["pre0"]:col["pre0"] + 6]
        out[name + "/eps"] = rows[:, col["eps0"]:col["eps0"] + 6]
        out[name + "/sig"] = rows[:, col["sig0"]:col["sig0"] + 6]
        out[name + "/D"] = rows[:, col["D00"]:col["D00"] + 36].reshape(-1, 6, 6)
        cases.append(name)
    out["cases"] = np.array(cases)
    out["param_names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, out_name), **out)
    print(out_name + ":", len(cases), "paths")


def pdmy_paths():
    pimy_paths("PressureDependMultiYield", PDMY_PARAMS, "pdmy_paths.npz")


if __name__ == "__main__":
    what = sys.argv[1:] or ["bricks", "compile_maps", "compile_digests", "pimy_paths", "pdmy_paths"]
    for w in what:
        globals()[w]()
