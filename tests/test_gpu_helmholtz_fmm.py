"""The Helmholtz FMM on the device (real k), against the oracle's Helmholtz FMM on the
same tree and lists and against the f64 direct sum (itself pinned to FMM3D's values in
test_gpu_helmholtz / test_helmholtz_oracle).  Needs a B200: -m gpu.

The oracle translates each pair by projection in absolute units while the device applies
per-level tables built by projection in box units (the same quadrature rule, another
evaluation order), so the f64 FMMs agree to rounding (within 1e-12 relative), not bit for
bit; the mixed form (f32 expansions and translations, complex64 near field) stays within
1e-5 of the f64 FMM."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def cloud():
    """1,000 points of a clipped Gaussian cluster: an adaptive tree of five levels (M2L on
    three, L2L on two, W and X lists) that the oracle's Python-level FMM runs in seconds."""
    rng = np.random.default_rng(31)
    x = np.clip(rng.normal(0.5, 0.12, (1000, 3)), 0.0, 1.0)
    q = rng.standard_normal(1000) + 1j * rng.standard_normal(1000)
    return x, q


def test_f64_matches_the_oracle_fmm(oracle, cloud):
    x, q = cloud
    k, p = 5.0, 6
    fmm = F.FmmBuilder(p).gradients().max_points_per_leaf(24).precision("f64").build(x)
    info = fmm.info()
    assert info["nlevels"] == 5 and info["w_pairs"] > 0 and info["x_pairs"] > 0
    out = fmm.helmholtz_evaluate(k, q)
    ophi, og = oracle.helmholtz_fmm(x, q, x, k, p, 24)
    ophi, og = ophi / (4 * np.pi), og / (4 * np.pi)
    ep, eg = rel(out.potential[0], ophi), rel(out.gradient[0], og)
    print(f"p={p}: f64 vs oracle FMM phi {ep:.2e} grad {eg:.2e}")
    assert ep < 1e-12 and eg < 1e-12  # measured 1.6e-15 and 1.3e-14
    fmm.close()


@pytest.mark.parametrize("p,tol", [(6, 2e-4), (10, 1e-5)])
def test_against_the_direct_sum(cloud, p, tol):
    x, q = cloud
    k = 5.0
    dphi, dg = F.helmholtz_direct_sum(k, x, q, x)
    for precision in ("f64", "mixed"):
        fmm = F.FmmBuilder(p).gradients().max_points_per_leaf(24).precision(precision).build(x)
        out = fmm.helmholtz_evaluate(k, q)
        ep, eg = rel(out.potential[0], dphi), rel(out.gradient[0], dg)
        print(f"p={p} {precision}: vs direct phi {ep:.2e} grad {eg:.2e}")
        assert ep < tol and eg < 10 * tol
        fmm.close()


def test_mixed_close_to_f64_and_repeatable():
    rng = np.random.default_rng(5)
    x = rng.uniform(0.0, 1.0, (20000, 3))
    q = rng.standard_normal((20000, 2)) + 1j * rng.standard_normal((20000, 2))
    k = 20.0
    outs = {}
    for precision in ("f64", "mixed"):
        fmm = F.FmmBuilder(8).gradients().vectors(2).max_points_per_leaf(48).precision(precision).build(x)
        a = fmm.helmholtz_evaluate(k, q)
        b = fmm.helmholtz_evaluate(k, q)  # tables kept for the same k: the same bits
        assert np.array_equal(a.potential, b.potential) and np.array_equal(a.gradient, b.gradient)
        outs[precision] = a
        fmm.close()
    ep = rel(outs["mixed"].potential, outs["f64"].potential)
    eg = rel(outs["mixed"].gradient, outs["f64"].gradient)
    print(f"mixed vs f64: phi {ep:.2e} grad {eg:.2e}")
    assert ep < 1e-5 and eg < 1e-5
    pick = np.arange(0, 20000, 97)
    dphi, _ = F.helmholtz_direct_sum(k, x, q[:, 1], x[pick], gradients=False)
    assert rel(outs["f64"].potential[1][pick], dphi) < 5e-4  # p = 8 at k = 20: measured 1.7e-4


def test_complex_wavenumber_is_refused(cloud):
    x, q = cloud
    fmm = F.FmmBuilder(6).max_points_per_leaf(32).build(x)
    with pytest.raises(F.FmmError) as e:
        fmm.helmholtz_evaluate(5.0 + 0.5j, q)
    assert e.value.status == 2
    fmm.close()


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_complex64_call_is_the_complex128_call_rounded(cloud, precision):
    """fmmgpu_helmholtz_evaluate_f32: complex64 charges in, every complex64 output the
    complex128 call's result on the widened charges, rounded (real and imaginary parts)."""
    x, q = cloud
    q64 = q.astype(np.complex64)
    fmm = F.FmmBuilder(6).gradients().max_points_per_leaf(24).precision(precision).build(x)
    want = fmm.helmholtz_evaluate(5.0, q64.astype(np.complex128))
    got = fmm.helmholtz_evaluate(5.0, q64)
    assert got.potential.dtype == np.complex64 and got.gradient.dtype == np.complex64
    assert np.array_equal(got.potential, want.potential.astype(np.complex64))
    assert np.array_equal(got.gradient, want.gradient.astype(np.complex64))
    fmm.close()
