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



def test_large_forest_on_host_threads():
    """A batch large enough for the merge to run on several host threads (more than 65,536
    boxes, leaves and points): the forest's boxes are the clouds' boxes level by level, its
    pair counts are their sums, and list rows spread over the whole forest (so over every
    thread's chunk) are the clouds' rows."""
    rng = np.random.default_rng(8)
    cs = [rng.uniform(0, 1, (150000, 3)), rng.normal(0, 1, (120000, 3))]
    b = F.FmmBuilder(4).max_points_per_leaf(4)
    forest = b.plan_batch(cs)
    singles = [b.plan(c) for c in cs]
    info = forest.info()
    assert info["nboxes"] > 65536 and info["nleaves"] > 65536 and info["nsources"] > 65536
    for k in ("nboxes", "nleaves", "near_pairs", "v_pairs", "w_pairs", "x_pairs"):
        assert info[k] == sum(s.info()[k] for s in singles), k
    fk, fl = forest.boxes()
    box_of, leaf_of = [], []  # forest box / leaf -> (cloud, local box / leaf), level by level
    local = [s.boxes() for s in singles]
    for lev in range(info["nlevels"]):
        for c, (k, leaf) in enumerate(local):
            for bx in np.nonzero(level_of(k) == lev)[0]:
                box_of.append((c, int(bx)))
    for n, (c, bx) in enumerate(box_of):
        assert fk[n] == local[c][0][bx] and fl[n] == local[c][1][bx]
    leaf_index = [np.cumsum(leaf) - 1 for _, leaf in local]
    leaf_of = [(c, int(leaf_index[c][bx])) for c, bx in box_of if local[c][1][bx]]
    for kind, rows in ((1, box_of), (3, box_of), (0, leaf_of), (2, leaf_of)):
        for r in np.linspace(0, len(rows) - 1, 1500).astype(np.int64):
            c, lr = rows[r]
            assert np.array_equal(forest.list(kind, int(r)), singles[c].list(kind, lr)), (kind, int(r))
