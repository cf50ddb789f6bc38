"""Whole-sweep CUDA graph (fmmgpu_fmm_set_graph): replays give the floats of the direct
launches, follow new charges in the same buffers, and re-capture for new buffers."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_graph_replay_equals_direct_launches(oracle, precision):
    x, q = oracle.point_sets("sphere", 20000, 3)
    fmm = F.FmmBuilder(6).gradients().max_points_per_leaf(32).precision(precision).build(x)
    direct = [fmm.evaluate(q * s) for s in (1.0, -2.0)]
    fmm.set_graph(True)
    for _ in range(2):  # capture, then replay, with new charges each time
        for s, want in zip((1.0, -2.0), direct):
            got = fmm.evaluate(q * s)
            assert np.array_equal(got.potential, want.potential)
            assert np.array_equal(got.gradient, want.gradient)
    assert fmm.info()["launches"] > 10


def test_graph_device_buffers_recapture(oracle):
    import torch

    x, q = oracle.point_sets("cube", 20000, 8)
    fmm = F.FmmBuilder(6).gradients().max_points_per_leaf(64).precision("mixed").build(x)
    want = fmm.evaluate(q)
    fmm.set_graph(True)
    dq = torch.from_numpy(q).cuda()
    n = len(x)
    for _ in range(2):  # a fresh set of output buffers each round: re-captured
        dphi = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        dg = torch.full((n * 3,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        fmm.evaluate_device(dq.data_ptr(), dphi.data_ptr(), dg.data_ptr())
        fmm.synchronize()
        assert np.array_equal(dphi.cpu().numpy(), want.potential[0])
        assert np.array_equal(dg.cpu().numpy().reshape(n, 3), want.gradient[0])


@pytest.mark.parametrize("precision,m", [("f64", 1), ("mixed", 1), ("mixed", 2)])
def test_overlapped_near_field_equals_one_stream(oracle, precision, m):
    """P2P on its own stream beside the far field gives the floats of the one-stream order."""
    x, q = oracle.point_sets("sphere", 30000, 6)
    q = np.stack([q * (v + 1) for v in range(m)], axis=1)
    fmm = F.FmmBuilder(8).gradients().vectors(m).max_points_per_leaf(64).precision(precision).build(x)
    fmm.set_overlap(True)
    a = fmm.evaluate(q)  # overlapped
    fmm.set_overlap(False)
    b = fmm.evaluate(q)
    assert np.array_equal(a.potential, b.potential) and np.array_equal(a.gradient, b.gradient)
    fmm.set_overlap(True)
    fmm.set_graph(True)
    for _ in range(2):
        c = fmm.evaluate(q)
        assert np.array_equal(c.potential, b.potential) and np.array_equal(c.gradient, b.gradient)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_launch_shapes_change_speed_only(oracle, precision):
    """Every launch shape the autotuner may pick (P2P warps a block, L2P / M2P threads a
    block) gives the same bits, and so do the tuned handle and a handle tuned at build."""
    x, q = oracle.point_sets("sphere", 30000, 4)
    builder = F.FmmBuilder(6).gradients().max_points_per_leaf(32).precision(precision)
    fmm = builder.build(x)
    want = fmm.evaluate(q)
    assert (fmm.info()["p2p_warps"], fmm.info()["leaf_block"]) == (4, 64)
    for w in (1, 2, 4):
        for b in (32, 64, 128):
            fmm.set_launch_shapes(w, b)
            got = fmm.evaluate(q)
            assert np.array_equal(got.potential, want.potential), (w, b)
            assert np.array_equal(got.gradient, want.gradient), (w, b)
    with pytest.raises(F.FmmError):
        fmm.set_launch_shapes(3, 64)
    # the tensor-core M2L tile (mixed): the alternative column count gives the same bits
    if precision == "mixed":
        assert fmm.info()["m2l_tile_columns"] == 128
        fmm.set_m2l_tile(1)
        assert fmm.info()["m2l_tile_columns"] == 64
        got = fmm.evaluate(q)
        assert np.array_equal(got.potential, want.potential) and np.array_equal(got.gradient, want.gradient)
        fmm.set_m2l_tile(0)
    else:
        assert fmm.info()["m2l_tile_columns"] == 0
        with pytest.raises(F.FmmError):
            fmm.set_m2l_tile(1)
    with pytest.raises(F.FmmError):
        fmm.set_m2l_tile(2)
    choice = fmm.autotune(q)
    assert choice["p2p_warps"] in (1, 2, 4) and choice["leaf_block"] in (32, 64, 128)
    assert (fmm.info()["p2p_warps"], fmm.info()["leaf_block"]) == (choice["p2p_warps"], choice["leaf_block"])
    fmm.set_graph(True)
    for _ in range(2):
        got = fmm.evaluate(q)
        assert np.array_equal(got.potential, want.potential) and np.array_equal(got.gradient, want.gradient)
    tuned = builder.autotune().build(x)
    got = tuned.evaluate(q)
    assert np.array_equal(got.potential, want.potential) and np.array_equal(got.gradient, want.gradient)
    fmm.close()
    tuned.close()
