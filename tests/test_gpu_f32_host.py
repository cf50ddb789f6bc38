"""The f32 host call (fmmgpu_fmm_evaluate_f32, the reference's Fmm<f32>::evaluate_into,
fmm-exec/src/fmm.rs:3719): each potential and gradient is the f64 call's result on the
widened charges, rounded to the nearest f32, with and without the graph, for one and
several vectors; and the rounded result stays within the mixed tolerance of the oracle."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,m,grad", [("mixed", 1, True), ("mixed", 3, True), ("f64", 1, True),
                                              ("mixed", 1, False)])
def test_f32_call_is_the_f64_call_rounded(oracle, precision, m, grad):
    x, q = oracle.point_sets("sphere", 20000, 5)
    q = np.stack([q * (v + 1) for v in range(m)], axis=1).astype(np.float32)
    fmm = F.FmmBuilder(6).gradients(grad).vectors(m).max_points_per_leaf(32).precision(precision).build(x)
    want = fmm.evaluate(q.astype(np.float64))
    for graph in (False, True, True):  # direct launches, capture, replay
        fmm.set_graph(graph)
        got = fmm.evaluate(q)
        assert got.potential.dtype == np.float32
        assert np.array_equal(got.potential, want.potential.astype(np.float32))
        if grad:
            assert got.gradient.dtype == np.float32
            assert np.array_equal(got.gradient, want.gradient.astype(np.float32))
        else:
            assert got.gradient is None


def test_f32_call_against_the_oracle(oracle):
    x, q = oracle.point_sets("cube", 12000, 9)
    q32 = q.astype(np.float32)
    fmm = F.FmmBuilder(6).gradients().max_points_per_leaf(32).precision("mixed").build(x)
    got = fmm.evaluate(q32)
    phi, g = oracle.fmm(x, q32.astype(np.float64), x, 6, 32, gradients=True, threads=8)
    rel = np.linalg.norm(got.potential - phi) / np.linalg.norm(phi)
    assert rel <= 2e-6
    relg = np.linalg.norm(got.gradient - g) / np.linalg.norm(g)
    assert relg <= 2e-6
