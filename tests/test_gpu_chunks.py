"""Chunked M2L product path (settings.product_bytes): the products made and reduced level by
level in chunks of target boxes through one small buffer give the floats of the products
held for every V pair at once, for both precisions, one and many charge vectors (the
tensor-core tiles gather rows one by one below four vectors and a pair's vectors as one
block from four), through the evaluation, the level calls and graph replay."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def _charges(q, m):
    return np.stack([q * (1.0 + 0.5 * v) * (-1) ** v for v in range(m)], axis=1) if m > 1 else q


@pytest.mark.parametrize("p,precision,m", [(6, "mixed", 1), (6, "mixed", 3), (6, "mixed", 16), (8, "mixed", 16),
                                           (6, "f64", 1), (6, "f64", 4)])
def test_chunked_products_equal_whole(oracle, p, precision, m):
    x, q = oracle.point_sets("sphere", 30000, 21)
    q = _charges(q, m)
    b = F.FmmBuilder(p).gradients().vectors(m).max_points_per_leaf(32).precision(precision)
    whole = b.build(x)
    assert whole.info()["product_chunks"] == 0 and whole.info()["vectors_per_pass"] == m
    want = whole.evaluate(q)
    small = b.product_bytes(2 << 20).build(x)
    info = small.info()
    assert info["product_chunks"] > 5 and info["vectors_per_pass"] == m
    got = small.evaluate(q)
    assert np.array_equal(got.potential, want.potential)
    assert np.array_equal(got.gradient, want.gradient)
    lv = small.evaluate_levels(q)
    assert np.array_equal(lv.potential, want.potential) and np.array_equal(lv.gradient, want.gradient)
    small.set_graph(True)
    for _ in range(2):
        g = small.evaluate(q)
        assert np.array_equal(g.potential, want.potential)
    if m == 1:
        phi, _ = oracle.fmm(x, q, x, p, 32, gradients=True, threads=8)
        err = np.linalg.norm(want.potential[0] - phi[0]) / np.linalg.norm(phi[0])
        assert err < (1e-12 if precision == "f64" else 2e-6), err
    whole.close()
    small.close()


def test_chunked_batch_with_fused_option(oracle):
    """A batch with 16 vectors in chunks: the tensor-core products, the SIMT products and
    the fused M2L all give the same floats (the first two through the chunked buffer)."""
    rng = np.random.default_rng(9)
    clouds = [rng.uniform(-1, 1, (n, 3)) for n in (4000, 15000, 7000)]
    n = sum(len(c) for c in clouds)
    q = rng.uniform(-1, 1, (n, 16))
    f = F.FmmBuilder(6).vectors(16).max_points_per_leaf(32).precision("mixed").product_bytes(4 << 20) \
        .build_batch(clouds)
    assert f.info()["product_chunks"] > 3
    a = f.evaluate(q)
    f.set_m2l_path(2)
    b = f.evaluate(q)
    assert np.array_equal(a.potential, b.potential)
    f.set_m2l_path(1)
    c = f.evaluate(q)
    assert np.array_equal(a.potential, c.potential)
    f.close()
