"""Fused tensor-core M2L (path 2 of the mixed form): the V products added into the locals
straight from tensor memory, in each target's row order, give the floats of the product
path (products stored, then the ordered local reduce, the default), bit for bit."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def _charges(q, m):
    return np.stack([q * (1.0 + 0.25 * v) * (-1) ** v for v in range(m)], axis=1) if m > 1 else q


@pytest.mark.parametrize("p,m", [(3, 1), (6, 1), (8, 1), (6, 3), (6, 16), (8, 16), (3, 16)])
def test_fused_equals_product_path(oracle, p, m):
    x, q = oracle.point_sets("sphere", 30000, 11)
    q = _charges(q, m)
    fmm = F.FmmBuilder(p).gradients().vectors(m).max_points_per_leaf(32).precision("mixed").build(x)
    prod = fmm.evaluate(q)  # the default path
    fmm.set_m2l_path(2)
    fused = fmm.evaluate(q)
    assert np.array_equal(fused.potential, prod.potential)
    assert np.array_equal(fused.gradient, prod.gradient)
    fmm.set_m2l_path(1)
    again = fmm.evaluate(q)
    assert np.array_equal(again.potential, prod.potential)
    if m == 1:
        phi, g = oracle.fmm(x, q, x, p, 32, gradients=True, threads=8)
        err = np.linalg.norm(fused.potential[0] - phi[0]) / np.linalg.norm(phi[0])
        assert err < 2e-6, err
    fmm.close()


def test_fused_level_calls_and_graph(oracle):
    """The per-level M2L call adds the fused products: level calls in the reference's
    schedule give the fused evaluation's floats; graph replays too."""
    x, q = oracle.point_sets("cube", 25000, 12)
    q = _charges(q, 4)
    fmm = F.FmmBuilder(6).gradients().vectors(4).max_points_per_leaf(32).precision("mixed").build(x)
    fmm.set_m2l_path(2)
    want = fmm.evaluate(q)
    got = fmm.evaluate_levels(q)
    assert np.array_equal(got.potential, want.potential) and np.array_equal(got.gradient, want.gradient)
    fmm.set_graph(True)
    for _ in range(2):
        got = fmm.evaluate(q)
        assert np.array_equal(got.potential, want.potential)
    fmm.close()


def test_fused_batch_many_vectors(oracle):
    """A forest of clouds with 16 vectors (every vector in one pass) equals the product path."""
    rng = np.random.default_rng(5)
    clouds = [rng.uniform(-1, 1, (n, 3)) for n in (3000, 17000, 9000)]
    clouds.append(oracle.point_sets("sphere", 12000, 3)[0])
    n = sum(len(c) for c in clouds)
    q = rng.uniform(-1, 1, (n, 16))
    fmm = F.FmmBuilder(6).vectors(16).max_points_per_leaf(32).precision("mixed").build_batch(clouds)
    assert fmm.info()["vectors_per_pass"] == 16
    a = fmm.evaluate(q)
    fmm.set_m2l_path(2)
    b = fmm.evaluate(q)
    assert np.array_equal(a.potential, b.potential)
    fmm.close()


def test_fused_vectors_beyond_one_tile(oracle):
    """Many vectors a pass (65 of 130): a tile holds one pair's 65 columns."""
    x, q = oracle.point_sets("cube", 4000, 13)
    m = 130
    qq = np.stack([q * (v + 1) for v in range(m)], axis=1)
    fmm = F.FmmBuilder(6).vectors(m).max_points_per_leaf(32).precision("mixed").vectors_per_pass(65).build(x)
    assert fmm.info()["vectors_per_pass"] == 65
    a = fmm.evaluate(qq)
    fmm.set_m2l_path(2)
    b = fmm.evaluate(qq)
    assert np.array_equal(a.potential, b.potential)
    with pytest.raises(F.FmmError):
        fmm.set_m2l_path(3)
    fmm.close()


def test_pass_holds_at_most_a_tile_of_vectors(oracle):
    """A pass holds at most a tensor-core tile's columns of vectors (96 at p = 8), and the
    fused M2L (tiles of 64 columns there) refuses a pass wider than its tile."""
    x, q = oracle.point_sets("cube", 3000, 14)
    fmm = F.FmmBuilder(8).vectors(100).max_points_per_leaf(32).precision("mixed").build(x)
    assert fmm.info()["vectors_per_pass"] == 50
    fmm.close()
    fmm = F.FmmBuilder(8).vectors(96).max_points_per_leaf(32).precision("mixed").build(x)
    assert fmm.info()["vectors_per_pass"] == 96
    with pytest.raises(F.FmmError, match="at most 64"):
        fmm.set_m2l_path(2)
    fmm.close()
