"""The operator ABI (fmmgpu_op_*): an evaluation driven level by level, in the reference
evaluator's schedule (fmm-plan/src/evaluator.rs:368-440), gives the same floats as the
fused evaluation (fmmgpu_fmm_evaluate) and so matches the oracle like it."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("precision,p,mk,grad,m", [
    ("f64", 6, 32, True, 1),
    ("f64", 3, 16, False, 2),
    ("mixed", 8, 64, True, 1),
    ("mixed", 6, 32, True, 2),
])
def test_level_calls_equal_fused_evaluation(oracle, precision, p, mk, grad, m):
    x, q = oracle.point_sets("sphere", 20000, 11)
    q = np.stack([q * (v + 1) for v in range(m)], axis=1)
    fmm = F.FmmBuilder(p).gradients(grad).vectors(m).max_points_per_leaf(mk).precision(precision).build(x)
    fused = fmm.evaluate(q)
    levels = fmm.evaluate_levels(q)
    assert np.array_equal(levels.potential, fused.potential)
    if grad:
        assert np.array_equal(levels.gradient, fused.gradient)
    if m == 1:
        phi, _ = oracle.fmm(x, q[:, 0], x, p, mk, gradients=False, threads=8)
        assert rel(levels.potential[0], phi) < (1e-12 if precision == "f64" else 2e-6)


def test_level_calls_simt_m2l_path(oracle):
    x, q = oracle.point_sets("cube", 20000, 4)
    fmm = F.FmmBuilder(8).gradients().max_points_per_leaf(64).precision("mixed").build(x)
    fmm.set_m2l_path(0)
    assert np.array_equal(fmm.evaluate_levels(q).potential, fmm.evaluate(q).potential)


def test_level_call_errors(oracle):
    x, q = oracle.point_sets("cube", 4000, 1)
    fmm = F.FmmBuilder(3).max_points_per_leaf(32).build(x)
    lib = F.lib()
    assert lib.fmmgpu_op_p2m(fmm._h, 0) == 1  # before begin_evaluation
    assert b"no evaluation begun" in lib.fmmgpu_last_error()
    nl = fmm.info()["nlevels"]
    qq = np.ascontiguousarray(q, dtype=np.float64)
    assert lib.fmmgpu_op_begin_evaluation(fmm._h, qq.ctypes.data) == 0
    assert lib.fmmgpu_op_m2l(fmm._h, nl) == 1 and lib.fmmgpu_op_p2p(fmm._h, -1) == 1
    assert lib.fmmgpu_op_host_data(fmm._h, 3) == 0
    # a second evaluation through the level calls repeats the first exactly
    a = fmm.evaluate_levels(q)
    b = fmm.evaluate_levels(q)
    assert np.array_equal(a.potential, b.potential)
