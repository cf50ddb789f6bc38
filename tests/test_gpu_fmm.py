"""GPU parity of the evaluator against the oracle (needs a B200: -m gpu).

The f64 evaluator must match the restated reference host FMM on the same tree and p
within 1e-12 relative L2 over all targets (the reference's own device
matched its host within 1.2e-14, fmm-bench/results/phase4s-gh200.md:448).  The mixed
evaluator (f32 points and expansions, f64 per-target accumulation) must stay within
2e-6 relative L2 of the f64 oracle at p <= 8 on these problems, so that its error
against the direct sum is the FMM's own truncation error.
"""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def run_both(oracle, src, q, tgt, p, mk, grad, precision="f64", m=1):
    fmm = F.FmmBuilder(p).gradients(grad).vectors(m).max_points_per_leaf(mk).precision(precision).build(src, tgt)
    out = fmm.evaluate(q)
    phi, g = oracle.fmm(src, q, tgt, p, mk, gradients=grad, threads=8)
    return fmm, out, phi, g


CASES = [
    ("cube", 20000, 6, 64, False),
    ("cube", 20000, 3, 32, True),
    ("sphere", 30000, 8, 64, True),
    ("sphere", 12000, 6, 16, True),
]


@pytest.mark.parametrize("kind,n,p,mk,grad", CASES)
def test_f64_matches_oracle(oracle, kind, n, p, mk, grad):
    x, q = oracle.point_sets(kind, n, 17)
    fmm, out, phi, g = run_both(oracle, x, q, x, p, mk, grad)
    assert rel(out.potential, phi) < 1e-12
    if grad:
        assert rel(out.gradient, g) < 1e-12


def test_f64_distinct_targets_and_vectors(oracle):
    rng = np.random.default_rng(9)
    src = rng.uniform(-1, 1, (15000, 3))
    tgt = np.concatenate([rng.normal(0.2, 0.3, (6000, 3)), src[:2000]])  # some coincide with sources
    q = rng.normal(size=(15000, 2))
    fmm, out, phi, g = run_both(oracle, src, q, tgt, 6, 24, True, m=2)
    assert rel(out.potential, phi) < 1e-12
    assert rel(out.gradient, g) < 1e-12


def test_f64_single_leaf_and_duplicates(oracle):
    rng = np.random.default_rng(2)
    x = rng.uniform(0, 1, (50, 3))
    x = np.concatenate([x, x[:10]])  # exact duplicates: coincident pairs are skipped
    q = rng.uniform(-1, 1, len(x))
    fmm, out, phi, g = run_both(oracle, x, q, x, 6, 64, True)  # root is the only leaf
    assert fmm.info()["nleaves"] == 1
    assert rel(out.potential, phi) < 1e-12 and rel(out.gradient, g) < 1e-12


def test_f64_bitwise_repeatable(oracle):
    x, q = oracle.point_sets("sphere", 20000, 3)
    fmm = F.FmmBuilder(6).gradients().max_points_per_leaf(32).build(x)
    a = fmm.evaluate(q)
    b = fmm.evaluate(q)
    assert np.array_equal(a.potential, b.potential) and np.array_equal(a.gradient, b.gradient)


@pytest.mark.parametrize("kind,n,p,mk,grad", CASES)
def test_mixed_close_to_oracle(oracle, kind, n, p, mk, grad):
    x, q = oracle.point_sets(kind, n, 17)
    fmm, out, phi, g = run_both(oracle, x, q, x, p, mk, grad, precision="mixed")
    assert rel(out.potential, phi) < 2e-6
    if grad:
        assert rel(out.gradient, g) < 2e-6


def test_f64_accuracy_gate_problem(oracle):
    """The C3.2 gate on the device (fmm-exec/tests/accuracy.rs): p = 8, twice 1.08e-5."""
    from tests.test_oracle import gate_problem

    x, sample, q = gate_problem(vectors=4)
    fmm = F.FmmBuilder(8).vectors(4).max_points_per_leaf(64).build(x)
    out = fmm.evaluate(q)
    errs = []
    for k in range(4):
        d, _ = oracle.direct_sum(x, q[:, k], x[sample], gradients=False)
        errs.append(rel(out.potential[k][sample], d / (4 * np.pi)))
    assert np.sqrt(np.mean(np.square(errs))) < 2 * 1.08e-5


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("mixed", 1e-6)])
def test_near_and_far_fields_separately(oracle, precision, tol):
    """Near field (P2P) alone and far field alone against the oracle's same split."""
    x, q = oracle.point_sets("sphere", 30000, 17)
    fmm = F.FmmBuilder(8).gradients().max_points_per_leaf(64).precision(precision).build(x)
    errs = {}
    for kinds, name in ((1, "near"), (2, "far")):
        fmm.set_kinds(kinds)
        out = fmm.evaluate(q)
        phi, g = oracle.fmm(x, q, x, 8, 64, gradients=True, threads=8, kinds=kinds)
        errs[name] = (rel(out.potential, phi), rel(out.gradient, g))
    print(precision, errs)
    for name, (ep, eg) in errs.items():
        assert ep < tol and eg < tol, (name, ep, eg)


@pytest.mark.parametrize("p,mk", [(3, 32), (6, 32), (8, 64)])
def test_mixed_tensor_core_m2l_matches_simt_and_oracle(oracle, p, mk):
    """The tcgen05 (3xTF32) M2L against the f32 SIMT M2L and the f64 oracle."""
    x, q = oracle.point_sets("sphere", 30000, 5)
    fmm = F.FmmBuilder(p).gradients().max_points_per_leaf(mk).precision("mixed").build(x)
    fmm.set_kinds(2)  # far field only: M2L dominates it
    fmm.set_m2l_path(0)
    simt = fmm.evaluate(q)
    fmm.set_m2l_path(1)
    tc = fmm.evaluate(q)
    phi, g = oracle.fmm(x, q, x, p, mk, gradients=True, threads=8, kinds=2)
    d_simt = rel(tc.potential, simt.potential)
    e_tc, e_simt = rel(tc.potential, phi), rel(simt.potential, phi)
    print(f"p={p}: tc vs simt {d_simt:.2e}, tc vs oracle {e_tc:.2e}, simt vs oracle {e_simt:.2e}, "
          f"grad tc {rel(tc.gradient, g):.2e}")
    assert d_simt < 2e-6
    assert e_tc < 2e-6 and rel(tc.gradient, g) < 2e-6
