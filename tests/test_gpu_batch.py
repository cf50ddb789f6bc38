"""Multi-cloud batches on the device: each cloud's results in the forest are the floats
of its own FMM (f64 and mixed, one and several charge vectors), and match the oracle."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def make_clouds(oracle, sizes):
    out = []
    for i, n in enumerate(sizes):
        kind = ("cube", "sphere")[i % 2]
        x, _ = oracle.point_sets(kind, n, 100 + i)
        out.append(x * (0.5 + 0.25 * i) + i)  # different scales and places
    return out


@pytest.mark.parametrize("precision,p,m", [("f64", 6, 1), ("mixed", 8, 1), ("mixed", 6, 3)])
def test_batch_equals_separate_fmms(oracle, precision, p, m):
    cs = make_clouds(oracle, [12000, 3000, 20000, 700])
    rng = np.random.default_rng(5)
    qs = [rng.uniform(-1, 1, (len(c), m)) for c in cs]
    builder = F.FmmBuilder(p).gradients().vectors(m).max_points_per_leaf(64).precision(precision)
    batch = builder.build_batch(cs)
    out = batch.evaluate(np.concatenate(qs))
    off = 0
    for c, q in zip(cs, qs):
        single = builder.build(c).evaluate(q)
        n = len(c)
        assert np.array_equal(out.potential[:, off:off + n], single.potential)
        assert np.array_equal(out.gradient[:, off:off + n], single.gradient)
        off += n


def test_batch_with_distinct_targets_matches_oracle(oracle):
    cs = make_clouds(oracle, [8000, 5000])
    rng = np.random.default_rng(8)
    ts = [c[::3] + 1e-3 for c in cs]
    qs = [rng.normal(size=len(c)) for c in cs]
    batch = F.FmmBuilder(6).gradients().max_points_per_leaf(32).build_batch(cs, ts)
    out = batch.evaluate(np.concatenate(qs))
    off = 0
    for c, t, q in zip(cs, ts, qs):
        phi, g = oracle.fmm(c, q, t, 6, 32, gradients=True, threads=8)
        assert rel(out.potential[0, off:off + len(t)], phi) < 1e-12
        assert rel(out.gradient[0, off:off + len(t)], g) < 1e-12
        off += len(t)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_vector_passes_give_the_same_floats(oracle, precision):
    """Charge vectors evaluated in passes (vectors_per_pass) equal the one-pass results."""
    x, _ = oracle.point_sets("sphere", 15000, 41)
    q = np.random.default_rng(6).uniform(-1, 1, (len(x), 6))
    base = F.FmmBuilder(6).gradients().vectors(6).max_points_per_leaf(64).precision(precision)
    one = base.build(x).evaluate(q)
    # 4 is rounded down to 3, a divisor of 6: two passes of three vectors
    two = F.FmmBuilder(6).gradients().vectors(6).max_points_per_leaf(64).precision(precision) \
        .vectors_per_pass(4).build(x)
    assert two.info()["vectors_per_pass"] == 3
    out = two.evaluate(q)
    assert np.array_equal(out.potential, one.potential) and np.array_equal(out.gradient, one.gradient)
    two.set_graph(True)
    for _ in range(2):
        out = two.evaluate(q)
        assert np.array_equal(out.potential, one.potential)
    hq = q + 0.5j * q[::-1]
    assert np.array_equal(two.helmholtz_near(3.0, hq).potential, base.build(x).helmholtz_near(3.0, hq).potential)


def test_potentials_multi_vector_kernels_independent_of_pass_size(oracle):
    """Mixed potentials of 8 vectors: the P2P and L2P/M2P kernels share the pair geometry
    and the harmonics across vectors; 1, 2 or 8 vectors a pass give the same bits, and the
    FMM agrees with the oracle."""
    x, q = oracle.point_sets("cube", 25000, 17)
    m = 8
    qq = np.stack([q * (1.0 + 0.3 * v) * (-1) ** v for v in range(m)], axis=1)
    outs = []
    for vpp in (1, 2, 8):
        f = F.FmmBuilder(6).vectors(m).max_points_per_leaf(32).precision("mixed").vectors_per_pass(vpp).build(x)
        assert f.info()["vectors_per_pass"] == vpp
        outs.append(f.evaluate(qq).potential)
        f.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    phi, _ = oracle.fmm(x, qq, x, 6, 32, gradients=False, threads=8)
    for v in (0, 5):
        err = np.linalg.norm(outs[2][v] - phi[v]) / np.linalg.norm(phi[v])
        assert err < 2e-6, (v, err)
