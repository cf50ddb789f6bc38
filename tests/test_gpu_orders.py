"""Every compiled expansion order (3 to 12) against the oracle (needs a B200: -m gpu):
f64 within 1e-12 and the mixed form within 2e-6 relative L2 over all targets, with
gradients; the mixed M2L runs on the tensor cores at every order (above p = 10, where
(p+1)^2 > 128 output slots, each tile once per half of them); the level calls and the
tuner's alternative M2L tile give the fused evaluation's bits."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def points(oracle):
    return oracle.point_sets("sphere", 12000, 23)


@pytest.mark.parametrize("p", [4, 5, 7, 9, 10, 11, 12])
def test_order_matches_oracle(oracle, points, p):
    x, q = points
    phi, g = oracle.fmm(x, q, x, p, 32, gradients=True, threads=8)
    for precision, tol in (("f64", 1e-12), ("mixed", 2e-6)):
        fmm = F.FmmBuilder(p).gradients().max_points_per_leaf(32).precision(precision).build(x)
        out = fmm.evaluate(q)
        ep, eg = rel(out.potential, phi), rel(out.gradient, g)
        print(f"p={p} {precision}: phi {ep:.2e} grad {eg:.2e}")
        assert ep < tol and eg < tol, (precision, ep, eg)
        if p in (10, 12):
            lv = fmm.evaluate_levels(q)
            assert np.array_equal(lv.potential, out.potential) and np.array_equal(lv.gradient, out.gradient)
        if precision == "mixed" and p in (7, 11, 12):
            fmm.set_m2l_tile(1)
            alt = fmm.evaluate(q)
            assert np.array_equal(alt.potential, out.potential) and np.array_equal(alt.gradient, out.gradient)
        fmm.close()


def test_order_outside_the_compiled_range_is_refused(points):
    x, _ = points
    with pytest.raises(F.FmmError) as e:
        F.FmmBuilder(13).build(x[:100])
    assert e.value.status == 2  # FMMGPU_UNSUPPORTED


def test_p8_alternative_tile_same_bits(oracle):
    """p = 8's alternative tensor-core M2L tile (80 columns, three raw stages, where the
    default has 96 and two) gives the default tile's bits."""
    x, q = oracle.point_sets("sphere", 20000, 29)
    fmm = F.FmmBuilder(8).gradients().max_points_per_leaf(32).precision("mixed").build(x)
    assert fmm.info()["m2l_tile_columns"] == 96
    out = fmm.evaluate(q)
    fmm.set_m2l_tile(1)
    assert fmm.info()["m2l_tile_columns"] == 80
    alt = fmm.evaluate(q)
    assert np.array_equal(alt.potential, out.potential) and np.array_equal(alt.gradient, out.gradient)
    fmm.close()
