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
  pdmy_paths.npz      the same for PressureDependMultiYield (tests/reference/data/nd/
                      PressureDependMultiYield_*.txt).
  pimy_paths.npz      the reference's stored OpenSees PressureIndependMultiYield strain paths
                      (tests/reference/data/nd/PressureIndependMultiYield_*.txt, read as text):
                      per path the material's parameters and backbone pairs, and per step the
                      load stage, the discarded trial strain (if any), the strain, and OpenSees'
                      stress and tangent.

    python tests/golden/make_golden.py [bricks|compile_maps|pimy_paths|pdmy_paths ...]
"""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
DATA = "/root/reference/tests/reference/data/element"
ND = "/root/reference/tests/reference/data/nd"
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
    what = sys.argv[1:] or ["bricks", "compile_maps", "pimy_paths", "pdmy_paths"]
    for w in what:
        globals()[w]()
