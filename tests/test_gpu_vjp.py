"""Vector-Jacobian products (fmmgpu_fmm_vjp) on the device, against the f64 direct sum,
its analytic gradients and central finite differences (eps = 1e-4).

The energy check follows the differentiated workload (loss L = 0.5 sum_i q_i phi_i on
Gaussian clusters, p = 8): with w = q / 2 the VJP gives dL/dq = phi / 2 + dcharges and
dL/dx = dsources + dtargets, whose exact values are phi and q grad phi."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu

FOUR_PI = 4.0 * np.pi


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def clusters(n, k, seed):
    """Seeded isotropic Gaussian clusters (centres in the unit cube, sigma log-uniform in
    [0.005, 0.05]), the shape of the differentiated workload's points."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, 1, (k, 3))
    sigma = np.exp(rng.uniform(np.log(0.005), np.log(0.05), k))
    which = rng.integers(0, k, n)
    return centres[which] + sigma[which, None] * rng.normal(size=(n, 3))


@pytest.mark.parametrize("precision,tol", [("f64", 2e-5), ("mixed", 2e-5)])
def test_energy_gradient_matches_direct_sum_and_finite_differences(oracle, precision, tol):
    x = clusters(20000, 8, 3)
    q = np.random.default_rng(4).normal(size=len(x))
    fmm = F.FmmBuilder(8).gradients().max_points_per_leaf(64).precision(precision).build(x)
    phi = fmm.evaluate(q).potential[0]
    dq, dxs, dxt = fmm.vjp(q, 0.5 * q[None, :])
    dl_dq = 0.5 * phi + dq[:, 0]
    dl_dx = dxs + dxt
    d, g = oracle.direct_sum(x, q, x, gradients=True)
    phi_ex, grad_ex = d / FOUR_PI, g / FOUR_PI
    assert rel(dl_dq, phi_ex) < tol
    assert rel(dl_dx, q[:, None] * grad_ex) < 10 * tol
    # central differences of the f64 energy on random coordinates: moving point k changes
    # only its pairs, so dL/dx_kc = q_k (phi_k(x + eps) - phi_k(x - eps)) / (2 eps) with
    # phi_k the potential of the other points
    rng = np.random.default_rng(9)
    eps = 1e-4
    scale = np.abs(dl_dx).max()
    for k in rng.choice(len(x), 8, replace=False):
        c = int(rng.integers(0, 3))
        others = np.delete(np.arange(len(x)), k)
        probe = np.repeat(x[k][None, :], 2, axis=0)
        probe[0, c] += eps
        probe[1, c] -= eps
        pk, _ = oracle.direct_sum(x[others], q[others], probe, gradients=False)
        fd = q[k] * (pk[0] - pk[1]) / FOUR_PI / (2 * eps)
        assert abs(fd - dl_dx[k, c]) < 1e-3 * scale, (k, c, fd, dl_dx[k, c])


def test_vjp_with_distinct_sources_and_targets(oracle):
    rng = np.random.default_rng(12)
    src = clusters(9000, 5, 13)
    tgt = rng.uniform(0, 1, (5000, 3))
    q = rng.normal(size=len(src))
    w = rng.normal(size=len(tgt))
    fmm = F.FmmBuilder(8).gradients().max_points_per_leaf(48).build(src, tgt)
    dq, dxs, dxt = fmm.vjp(q, w[None, :])
    # the transpose pass is the FMM of the swapped problem: its floats, and the oracle's
    swapped = F.FmmBuilder(8).gradients().max_points_per_leaf(48).build(tgt, src).evaluate(w)
    assert np.array_equal(dq[:, 0], swapped.potential[0])
    assert np.array_equal(dxs, q[:, None] * swapped.gradient[0])
    phi_o, _ = oracle.fmm(tgt, w, src, 8, 48, gradients=False, threads=8)
    assert rel(dq[:, 0], phi_o[0]) < 1e-12
    # and within the FMM's truncation error of the exact sums
    _, g_t = oracle.direct_sum(src, q, tgt, gradients=True)  # grad phi at the targets
    psi, g_s = oracle.direct_sum(tgt, w, src, gradients=True)  # the transpose problem
    assert rel(dq[:, 0], psi / FOUR_PI) < 1e-4
    assert rel(dxt, w[:, None] * g_t / FOUR_PI) < 5e-4
    assert rel(dxs, q[:, None] * g_s / FOUR_PI) < 5e-4
    # a second call reuses the transpose FMM built by the first
    dq2, _, _ = fmm.vjp(q, w[None, :])
    assert np.array_equal(dq, dq2)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("symmetric", [True, False])
def test_stored_forward_pass_gives_the_same_vjp(precision, symmetric):
    """With the forward pass stored, a VJP whose charges are those of the last evaluation
    takes the kept target gradients instead of its own forward FMM: the same bits as
    recomputing it; other charges are recomputed (and then kept)."""
    x = clusters(12000, 6, 7)
    y = x if symmetric else clusters(9000, 5, 8)
    rng = np.random.default_rng(9)
    q, q2 = rng.normal(size=len(x)), rng.normal(size=len(x))
    w = rng.normal(size=(1, len(y)))
    build = lambda: F.FmmBuilder(6).gradients().max_points_per_leaf(64).precision(precision).build(
        x, None if symmetric else y)
    ref, st = build(), build()
    want = ref.vjp(q, w)
    want2 = ref.vjp(q2, w)
    st.set_vjp_store(True)
    st.evaluate(q)
    got = st.vjp(q, w)
    assert st.info()["vjp_forward_reused"] == 1
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    got2 = st.vjp(q2, w)  # other charges: recomputed
    assert st.info()["vjp_forward_reused"] == 1
    for a, b in zip(got2, want2):
        assert np.array_equal(a, b)
    got3 = st.vjp(q2, w)  # the VJP's own forward pass was kept
    assert st.info()["vjp_forward_reused"] == 2
    for a, b in zip(got3, want2):
        assert np.array_equal(a, b)
    st.set_vjp_store(False)
    st.vjp(q2, w)
    assert st.info()["vjp_forward_reused"] == 2
    ref.close()
    st.close()
