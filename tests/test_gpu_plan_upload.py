"""An FMM on a plan given from outside (fmmgpu_upload_plan, the reference's
DeviceOperator::new on its own plan), needs a B200: -m gpu.  The library's plan exported
and uploaded again gives the library's bits (fused evaluation and level calls); the
oracle's plan (its tree and brute-force lists, boxes without sources kept in the rows)
gives the oracle FMM's result within 1e-12."""
import numpy as np
import pytest

import fmm_b200 as F
from tests.plan_arrays import oracle_plan

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_uploaded_library_plan_gives_the_same_bits(precision):
    rng = np.random.default_rng(8)
    x = rng.uniform(size=(20000, 3))
    q = rng.standard_normal(20000)
    own = F.FmmBuilder(6).gradients().max_points_per_leaf(32).precision(precision).build(x)
    arrays = own.plan_arrays()
    up = F.FmmBuilder(6).gradients().precision(precision).upload(arrays, x)
    a, b = own.evaluate(q), up.evaluate(q)
    assert np.array_equal(a.potential, b.potential) and np.array_equal(a.gradient, b.gradient)
    c = up.evaluate_levels(q)
    assert np.array_equal(c.potential, a.potential) and np.array_equal(c.gradient, a.gradient)


def test_uploaded_oracle_plan_matches_the_oracle_fmm(oracle):
    x, q = oracle.point_sets("sphere", 12000, 9)
    arrays = oracle_plan(oracle, x, x, 24)
    up = F.FmmBuilder(6).gradients().precision("f64").upload(arrays, x)
    out = up.evaluate(q)
    phi, g = oracle.fmm(x, q, x, 6, 24, gradients=True, threads=8)
    assert rel(out.potential, phi) < 1e-12 and rel(out.gradient, g) < 1e-12
