"""The point stages of the plan build on the device (Morton keys, the distinct sorted
keys, each point's leaf and the order by leaf; plan_gpu.cu) give the host build's plan
exactly: the same boxes, leaves, point order and lists (needs a B200: -m gpu)."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert np.allclose(a[k], b[k], rtol=0, atol=0), k


@pytest.mark.parametrize("case", ["sphere", "cube_distinct_targets", "clumps_and_duplicates"])
def test_device_point_stages_give_the_host_plan(oracle, case):
    rng = np.random.default_rng(21)
    if case == "sphere":
        src, _ = oracle.point_sets("sphere", 300000, 4)
        tgt = None
    elif case == "cube_distinct_targets":
        src = rng.uniform(0, 1, (120000, 3))
        tgt = rng.normal(0.5, 0.15, (70000, 3))
    else:
        base = rng.uniform(-1, 1, (60000, 3))
        clump = 0.3 + 1e-6 * rng.uniform(size=(5000, 3))
        src = np.concatenate([base, clump, base[:3000]])  # a clump below leaf size and exact duplicates
        tgt = None
    dev = F.FmmBuilder(4).max_points_per_leaf(40).build(src, tgt)
    host = F.FmmBuilder(4).max_points_per_leaf(40).plan(src, tgt)
    same(dev.plan_arrays(), host.plan_arrays())
    dev.close()
