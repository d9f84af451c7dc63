"""The compile step's arrays are the reference's (compile::compile_model) value for value: against
the stored fixtures (tests/golden/compile_maps.npz), and against the reference built here on a
range of block sizes when its library is present."""
import json
import os

import numpy as np
import pytest

import femorax_b200 as fx
from femorax_b200 import meshes
from tests.models_for_tests import soil_column, two_region_block

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "compile_maps.npz"))
ARRAYS = fx.Compiled.I32 + fx.Compiled.F64


@pytest.mark.parametrize("name,build", [("block", two_region_block), ("column", soil_column)])
def test_maps_match_stored_reference(name, build):
    c = fx.Model(build()).compile(renumbering="rcm", simd_width=32, coloring=True)
    for a in ARRAYS:
        got, want = c.array(a), GOLD[f"{name}/{a}"]
        assert got.shape == want.shape and np.array_equal(got, want), a
    p = fx.params_table(c.params())
    assert np.array_equal(p[:, 1:12], GOLD[f"{name}/params"][:, 1:12])


@pytest.mark.parametrize("dims,kw", [((5, 4, 3), dict(renumbering="rcm", simd_width=32, coloring=True)),
                                     ((7, 2, 6), dict(renumbering="off", simd_width=1, coloring=True)),
                                     ((1, 1, 12), dict(renumbering="rcm", simd_width=4, coloring=False)),
                                     ((6, 6, 6), dict(renumbering="rcm", simd_width=32, coloring=False))])
def test_maps_match_live_reference(dims, kw, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference library not built")
    spec = meshes.box_model(*dims, lumped=True)
    mine = fx.Model(spec).compile(**kw)
    theirs = oracle_mod.RefModel(spec).compile(**kw)
    for a in ARRAYS:
        assert np.array_equal(mine.array(a), theirs.array(a)), a


def test_layered_and_heterogeneous_configs(oracle_mod, ref_available):
    """Small instances of the layered box and the per-element-material cube."""
    if not ref_available:
        pytest.skip("reference library not built")
    for spec in (meshes.layered_box(6, 5, 8, layers=4, seed=2)[0], meshes.heterogeneous_cube(4, seed=1)):
        mine = fx.Model(spec).compile()
        theirs = oracle_mod.RefModel(spec).compile()
        for a in ARRAYS:
            assert np.array_equal(mine.array(a), theirs.array(a)), a
        assert np.array_equal(fx.params_table(mine.params())[:, 1:12], theirs.params()[:, 1:12])


def test_invalid_models_are_refused():
    spec = meshes.box_model(2, 2, 2)
    spec.eqd_retained = np.array([1, 2], np.int32)
    spec.eqd_constrained = np.array([5, 5], np.int32)
    spec.eqd_dof = np.array([1, 1], np.int32)
    with pytest.raises(fx.FxError) as e:
        fx.Model(spec).compile()
    assert e.value.code == 1
    bad = meshes.box_model(2, 2, 2)
    bad.groups[0].conn = bad.groups[0].conn.copy()
    bad.groups[0].conn[0, 0] = 99999
    with pytest.raises(fx.FxError):
        fx.Model(bad).compile()


@pytest.mark.parametrize("name", ["static_cube_32", "layered_box_128x128x64", "heterogeneous_cube_100"])
def test_maps_at_benchmark_configs(name):
    """Every compile array of the benchmark configurations' models (the 32^3 static cube, the
    128 x 128 x 64 layered box, the 100^3 per-element-E cube) has the digest of the reference's
    compile_model output (tests/golden/compile_digests.json, written from oracle/_ref)."""
    from tests.golden import make_golden as G
    want = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "compile_digests.json")))[name]
    c = fx.Model(G.config_model(name)).compile(renumbering="rcm", simd_width=32)
    got = {a: G.array_digest(c.array(a)) for a in want}
    assert set(want) == set(ARRAYS)
    assert got == want
