"""Helmholtz on the device: the f64 direct sum against FMM3D's values, and the near field
of the plan (f64 and complex64) against the oracle's."""
import numpy as np
import pytest

import fmm_b200 as F
from tests.test_helmholtz_oracle import golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_gpu_direct_sum_matches_fmm3d():
    src, points, cases = golden()
    for label, k, q, idx, pot, g in cases:
        phi, grad = F.helmholtz_direct_sum(k, src, q, points[idx])
        assert rel(phi, pot) < 1e-13, label
        assert rel(grad, g) < 1e-13, label


@pytest.mark.parametrize("precision,tol,k,m", [
    ("f64", 1e-12, 20.0, 1),
    ("f64", 1e-12, 8.0 + 2.0j, 2),
    ("mixed", 2e-6, 20.0, 1),
    ("mixed", 2e-6, 8.0 + 2.0j, 2),
])
def test_near_field_matches_oracle(oracle, precision, tol, k, m):
    x, _ = oracle.point_sets("cube", 20000, 31)
    rng = np.random.default_rng(32)
    q = rng.normal(size=(len(x), m)) + 1j * rng.normal(size=(len(x), m))
    fmm = F.FmmBuilder(3).gradients().vectors(m).max_points_per_leaf(64).precision(precision).build(x)
    out = fmm.helmholtz_near(k, q)
    phi, g = oracle.helmholtz_near(x, q, x, k, 64, gradients=True, threads=8)
    assert rel(out.potential, phi) < tol
    assert rel(out.gradient, g) < tol


def test_near_field_of_one_leaf_is_the_direct_sum(oracle):
    rng = np.random.default_rng(5)
    x = rng.uniform(size=(300, 3))
    q = rng.normal(size=300) + 1j * rng.normal(size=300)
    fmm = F.FmmBuilder(3).gradients().max_points_per_leaf(512).build(x)
    assert fmm.info()["nleaves"] == 1
    out = fmm.helmholtz_near(5.0 + 0.5j, q)
    d, dg = F.helmholtz_direct_sum(5.0 + 0.5j, x, q, x)
    assert rel(out.potential[0], d) < 1e-13 and rel(out.gradient[0], dg) < 1e-13
