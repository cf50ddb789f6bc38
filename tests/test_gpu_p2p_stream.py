"""The mixed P2P's source streams: every near row's sources mapped into its target leaf's
frame once, at build time, and copied per flush (path 1, the default when the streams fit)
give the bits of the per-flush map (path 0), for potentials and gradients, one and several
vectors, items of fewer than 32 targets, the level calls, graph replays and batches."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def _both(fmm, q):
    assert fmm.info()["p2p_stream_bytes"] > 0
    streamed = fmm.evaluate(q)
    fmm.set_p2p_path(0)
    mapped = fmm.evaluate(q)
    fmm.set_p2p_path(1)
    again = fmm.evaluate(q)
    return streamed, mapped, again


@pytest.mark.parametrize("geometry,n,leaf,grad,m", [
    ("sphere", 40000, 128, True, 1),
    ("sphere", 40000, 128, False, 1),
    ("cube", 30000, 32, True, 3),
    ("cube", 30000, 32, False, 7),
    ("clusters", 20000, 64, True, 1),
    ("cube", 500, 7, True, 2),     # odd leaves: padded pairs at every row's end
])
def test_streamed_equals_mapped(oracle, geometry, n, leaf, grad, m):
    if geometry == "clusters":  # dense Gaussian clumps: deep, unbalanced leaves
        rng = np.random.default_rng(21)
        cen = rng.uniform(-1, 1, (6, 3))
        x = cen[rng.integers(0, 6, n)] + 0.02 * rng.standard_normal((n, 3))
        q = rng.standard_normal(n)
    else:
        x, q = oracle.point_sets(geometry, n, 21)
    if m > 1:
        q = np.stack([q * (1.0 + 0.5 * v) * (-1) ** v for v in range(m)], axis=1)
    b = F.FmmBuilder(6).vectors(m).max_points_per_leaf(leaf).precision("mixed")
    if grad:
        b = b.gradients()
    fmm = b.build(x)
    s, p, a = _both(fmm, q)
    assert np.array_equal(s.potential, p.potential) and np.array_equal(a.potential, p.potential)
    if grad:
        assert np.array_equal(s.gradient, p.gradient)
    if m == 1 and n <= 40000:
        phi, _ = oracle.fmm(x, q, x, 6, leaf, gradients=False, threads=8)
        err = np.linalg.norm(s.potential[0] - phi[0]) / np.linalg.norm(phi[0])
        assert err < 2e-6, err
    fmm.close()


def test_streamed_level_calls_graph_and_shapes(oracle):
    x, q = oracle.point_sets("sphere", 30000, 22)
    fmm = F.FmmBuilder(8).gradients().max_points_per_leaf(64).precision("mixed").build(x)
    fmm.set_p2p_path(0)
    want = fmm.evaluate(q)
    fmm.set_p2p_path(1)
    got = fmm.evaluate_levels(q)
    assert np.array_equal(got.potential, want.potential) and np.array_equal(got.gradient, want.gradient)
    for w in (1, 2, 4):
        fmm.set_launch_shapes(w, 64)
        fmm.set_graph(True)
        for _ in range(2):
            got = fmm.evaluate(q)
            assert np.array_equal(got.potential, want.potential) and np.array_equal(got.gradient, want.gradient)
        fmm.set_graph(False)
    fmm.close()


def test_streamed_batch_and_separate_targets(oracle):
    rng = np.random.default_rng(23)
    clouds = [rng.uniform(-1, 1, (k, 3)) for k in (2000, 9000, 5000)]
    n = sum(len(c) for c in clouds)
    q = rng.uniform(-1, 1, (n, 4))
    fmm = F.FmmBuilder(6).vectors(4).max_points_per_leaf(32).precision("mixed").build_batch(clouds)
    s, p, _ = _both(fmm, q)
    assert np.array_equal(s.potential, p.potential)
    fmm.close()
    # targets apart from the sources
    xs, qs = oracle.point_sets("cube", 20000, 24)
    xt = rng.uniform(-1, 1, (7000, 3))
    fmm = F.FmmBuilder(6).gradients().max_points_per_leaf(48).precision("mixed").build(xs, xt)
    s, p, _ = _both(fmm, qs)
    assert np.array_equal(s.potential, p.potential) and np.array_equal(s.gradient, p.gradient)
    fmm.close()


def test_p2p_path_hook_rejects_unbuilt_forms():
    x = np.random.default_rng(25).uniform(-1, 1, (3000, 3))
    fmm = F.FmmBuilder(3).max_points_per_leaf(32).precision("f64").build(x)
    assert fmm.info()["p2p_stream_bytes"] == 0
    with pytest.raises(F.FmmError):
        fmm.set_p2p_path(1)
    with pytest.raises(F.FmmError):
        fmm.set_p2p_path(2)
    fmm.set_p2p_path(0)
    fmm.close()


def test_plan_without_near_singular_pairs(oracle):
    """Targets apart from every source (no near-singular pair, no near pair at all): the
    P2P adds no near-singular sums, on either path, and the result is the far field."""
    rng = np.random.default_rng(26)
    xs = rng.uniform(0.0, 1.0, (5000, 3))
    xt = rng.uniform(1.5, 2.5, (3000, 3))
    q = rng.standard_normal(5000)
    fmm = F.FmmBuilder(6).gradients().max_points_per_leaf(32).precision("mixed").build(xs, xt)
    assert fmm.info()["close_pairs"] == 0
    s, p, _ = _both(fmm, q)
    assert np.array_equal(s.potential, p.potential) and np.array_equal(s.gradient, p.gradient)
    phi, g = oracle.fmm(xs, q, xt, 6, 32, gradients=True, threads=8)
    assert np.linalg.norm(s.potential[0] - phi[0]) / np.linalg.norm(phi[0]) < 2e-6
    assert np.linalg.norm(s.gradient[0] - g[0]) / np.linalg.norm(g[0]) < 2e-6
    fmm.close()
