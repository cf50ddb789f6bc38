"""The tuning cache (the autotuner's choices kept per device, precision and p, the
reference's FmmBuilder::tuning_cache) and the Helmholtz tables in the table cache (needs
a B200: -m gpu)."""
import os

import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def test_tuning_cache_keeps_the_choice(tmp_path):
    d = str(tmp_path)
    x = np.random.default_rng(4).uniform(size=(30000, 3))
    q = np.random.default_rng(5).standard_normal(30000)
    a = F.FmmBuilder(6).gradients().max_points_per_leaf(64).precision("mixed").autotune().tuning_cache(d).build(x)
    ia = a.info()
    assert ia["tuning_loaded"] == 0
    files = os.listdir(d)
    assert len(files) == 1 and files[0].startswith("tuning-cuda-") and files[0].endswith("-mixed-p06.txt")
    text = open(os.path.join(d, files[0])).read()
    assert f"gradients:p2p_warps {ia['p2p_warps']}" in text and f"gradients:leaf_block {ia['leaf_block']}" in text
    assert f"gradients:m2l_tile {0 if ia['m2l_tile_columns'] == 128 else 1}" in text
    b = F.FmmBuilder(6).gradients().max_points_per_leaf(64).precision("mixed").autotune().tuning_cache(d).build(x)
    ib = b.info()
    assert ib["tuning_loaded"] == 1
    assert (ib["p2p_warps"], ib["leaf_block"], ib["m2l_tile_columns"]) == (
        ia["p2p_warps"], ia["leaf_block"], ia["m2l_tile_columns"])
    oa, ob = a.evaluate(q), b.evaluate(q)
    assert np.array_equal(oa.potential, ob.potential) and np.array_equal(oa.gradient, ob.gradient)
    # a corrupted file is rejected and the shapes timed again (and stored again)
    path = os.path.join(d, files[0])
    open(path, "w").write(text.replace("p 6", "p 7"))
    c = F.FmmBuilder(6).gradients().max_points_per_leaf(64).precision("mixed").autotune().tuning_cache(d).build(x)
    assert c.info()["tuning_loaded"] == 0
    assert open(path).read() != text.replace("p 6", "p 7")


def test_helmholtz_tables_in_the_table_cache(tmp_path):
    d = str(tmp_path)
    rng = np.random.default_rng(6)
    x = rng.uniform(size=(8000, 3))
    q = rng.standard_normal(8000) + 1j * rng.standard_normal(8000)
    a = F.FmmBuilder(6).gradients().max_points_per_leaf(32).table_cache(d).build(x)
    oa = a.helmholtz_evaluate(10.0, q)
    names = os.listdir(d)
    assert any(n.startswith("hh-m2l-p06-k") for n in names) and any(n.startswith("hh-octant-p06-k") for n in names)
    b = F.FmmBuilder(6).gradients().max_points_per_leaf(32).table_cache(d).build(x)
    assert b.info()["tables_loaded"] == 7
    ob = b.helmholtz_evaluate(10.0, q)
    assert np.array_equal(oa.potential, ob.potential) and np.array_equal(oa.gradient, ob.gradient)
