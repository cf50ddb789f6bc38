"""Multi-cloud batches (fmmgpu_batch_*): the forest plan is every cloud's own plan, merged
level by level (boxes, leaves, lists and their accumulation order), without a GPU."""
import numpy as np

import fmm_b200 as F


def clouds():
    rng = np.random.default_rng(21)
    a = rng.uniform(0, 1, (3000, 3))
    g = rng.normal(size=(2500, 3))
    b = 2.0 + g / np.linalg.norm(g, axis=1, keepdims=True)  # a sphere elsewhere in space
    c = rng.normal(0.3, 0.05, (1200, 3))
    return [a, b, c]


def level_of(keys):
    return (keys & np.uint64(0x7FFF)).astype(np.int64)


def test_forest_boxes_are_the_clouds_boxes_level_by_level():
    cs = clouds()
    builder = F.FmmBuilder(6).max_points_per_leaf(32)
    forest = builder.plan_batch(cs)
    singles = [builder.plan(c) for c in cs]
    fk, fl = forest.boxes()
    info = forest.info()
    assert info["nboxes"] == sum(s.info()["nboxes"] for s in singles)
    assert info["near_pairs"] == sum(s.info()["near_pairs"] for s in singles)
    assert info["v_pairs"] == sum(s.info()["v_pairs"] for s in singles)
    nl = max(s.info()["nlevels"] for s in singles)
    assert info["nlevels"] == nl
    pos = 0
    for lev in range(nl):
        for s in singles:
            k, leaf = s.boxes()
            sel = level_of(k) == lev
            n = int(sel.sum())
            assert np.array_equal(fk[pos:pos + n], k[sel]) and np.array_equal(fl[pos:pos + n], leaf[sel])
            pos += n
    assert pos == len(fk)


def test_forest_lists_are_the_clouds_lists():
    cs = clouds()
    builder = F.FmmBuilder(6).max_points_per_leaf(32)
    forest = builder.plan_batch(cs)
    singles = [builder.plan(c) for c in cs]
    # box rows (V and X lists) in forest order: level by level, cloud by cloud
    nl = forest.info()["nlevels"]
    row = 0
    for lev in range(nl):
        for s in singles:
            k, _ = s.boxes()
            for b in np.nonzero(level_of(k) == lev)[0]:
                for kind in (1, 3):  # V, X
                    assert np.array_equal(forest.list(kind, row), s.list(kind, int(b))), (lev, kind)
                row += 1


def test_batch_errors_name_the_cloud():
    cs = clouds()
    cs[1] = np.full((5, 3), np.nan)
    try:
        F.FmmBuilder(3).plan_batch(cs)
    except F.FmmError as e:
        assert "cloud 1" in str(e)
    else:
        raise AssertionError("a non-finite cloud must be rejected")
