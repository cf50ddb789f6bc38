"""The product's host plan (tree, lists, tables) against the oracle (no GPU).

The tree must equal the oracle's restatement of the reference's refinement and 2:1
balance key for key; every list row must equal the oracle's brute-force list rule
(fmm-plan/src/interaction_manager.rs:15-27) with boxes that hold no source removed
(their contributions are exact zeros), in the accumulation order of
fmm-plan/src/operator.rs:34-45; the f64 tables must equal the oracle's tables.
"""
import numpy as np
import pytest

import fmm_b200 as F

LEVEL_MASK = np.uint64(0x7FFF)


def _occupied(keys, pts_keys):
    """Boxes (keys) with at least one level-16 point key below them."""
    lv = (keys & LEVEL_MASK).astype(np.int64)
    occ = np.zeros(len(keys), dtype=bool)
    pk = np.sort(pts_keys)
    for i, (k, l) in enumerate(zip(keys, lv)):
        shift = np.uint64(15 + 3 * (16 - l))
        lo = (k >> shift) << shift
        hi = lo + (np.uint64(1) << shift)
        a = np.searchsorted(pk, lo)
        occ[i] = a < len(pk) and pk[a] < hi
    return occ


def _point_keys(oracle, x):
    tr = oracle.Tree(x, x, 16, 1 << 30)  # for the domain only
    del tr
    lo = x.min(0)
    hi = x.max(0)
    diam = hi - lo
    mean = lo + 0.5 * diam
    md = diam.max() * (1.0 + 1.0 / 65536)
    b0 = mean - 0.5 * md
    b1 = mean + 0.5 * md
    keys = np.zeros(len(x), dtype=np.uint64)
    for i, p in enumerate(x):
        idx = np.minimum(np.floor((p - b0) / (b1 - b0) * 65536).clip(0), 65535).astype(np.uint32)
        keys[i] = oracle.lib().orc_key_from_index(np.ascontiguousarray(idx), 16)
    return keys


@pytest.mark.parametrize("kind,n,mk", [("cube", 3000, 16), ("sphere", 6000, 24), ("cube", 40000, 64)])
def test_tree_equals_oracle(oracle, kind, n, mk):
    x, _ = oracle.point_sets(kind, n, 11)
    plan = F.FmmBuilder(4).max_points_per_leaf(mk).plan(x)
    keys, leaf = plan.boxes()
    tr = oracle.Tree(x, x, 16, mk)
    assert np.array_equal(keys, tr.keys)
    assert np.array_equal(leaf, tr.is_leaf)


def test_large_plan_on_host_threads(oracle):
    """Above 65,536 points the host point stages (keys, distinct sort, each point's leaf, the
    stable order by leaf) run on several threads: the tree is still the oracle's, the points
    of a leaf keep their index order, the plan passes every check of an uploaded plan, and
    targets given as a separate array of the same values give the same plan as targets
    that are the sources."""
    x, _ = oracle.point_sets("cube", 200000, 17)
    mk = 64
    a = F.FmmBuilder(4).max_points_per_leaf(mk).plan(x)
    b = F.FmmBuilder(4).max_points_per_leaf(mk).plan(x, x.copy())
    keys, leaf = a.boxes()
    tr = oracle.Tree(x, x, 16, mk)
    assert np.array_equal(keys, tr.keys) and np.array_equal(leaf, tr.is_leaf)
    pa, pb = a.plan_arrays(), b.plan_arrays()
    for name in F.PlanArrays.ARRAYS:
        assert np.array_equal(pa[name], pb[name]), name
    for s in ("source", "target"):
        off, order = pa[f"{s}_offsets"], pa[f"{s}_order"]
        assert off[0] == 0 and off[-1] == len(x) and np.array_equal(np.sort(order), np.arange(len(x)))
        step = np.diff(order)
        inside = np.ones(len(step), dtype=bool)
        inside[off[1:-1] - 1] = False  # the last point of a leaf and the first of the next
        assert np.all(step[inside] > 0)
    F.FmmBuilder(4).max_points_per_leaf(mk).plan_from(pa, x).close()
    a.close()
    b.close()
    # more than 65,536 leaves: the leaf-scaled coordinates are formed on host threads too,
    # and the upload's check puts every point inside its own leaf
    small = F.FmmBuilder(4).max_points_per_leaf(2).plan(x)
    assert small.info()["nleaves"] > 65536
    F.FmmBuilder(4).max_points_per_leaf(2).plan_from(small.plan_arrays(), x).close()
    small.close()


def test_tree_with_distinct_targets(oracle):
    rng = np.random.default_rng(3)
    src = rng.uniform(0, 1, (2500, 3))
    tgt = rng.normal(0.5, 0.1, (1500, 3))
    plan = F.FmmBuilder(4).max_points_per_leaf(10).plan(src, tgt)
    keys, leaf = plan.boxes()
    tr = oracle.Tree(src, tgt, 16, 10)
    assert np.array_equal(keys, tr.keys) and np.array_equal(leaf, tr.is_leaf)


def test_lists_equal_brute_force_rule(oracle):
    x, _ = oracle.point_sets("sphere", 5000, 5)
    assert _check_lists(oracle, x, 20) > 1000


@pytest.mark.parametrize("name", ["clumps", "planar", "duplicates"])
def test_lists_equal_brute_force_rule_on_edge_cases(oracle, name):
    """Ragged depth (clumps 1e-6 wide beside a uniform cloud), a planar cloud and coincident
    points: every list row equals the brute-force rule in accumulation order."""
    _check_lists(oracle, _edge_sets()[name], 8)  # duplicates: few sites, no V pair at all


def _check_lists(oracle, x, mk):
    plan = F.FmmBuilder(4).max_points_per_leaf(mk).plan(x)
    keys, leaf = plan.boxes()
    tr = oracle.Tree(x, x, 16, mk)
    occ = _occupied(keys, _point_keys(oracle, x))
    occ_of = dict(zip(keys.tolist(), occ.tolist()))
    leaf_ids = np.flatnonzero(leaf)
    offsets_checked = 0
    for b in range(len(keys)):
        is_leaf = bool(leaf[b])
        # V (kind 1) and X (kind 3) rows by box; near (0) and W (2) rows by leaf index
        for kind, okind in ((1, 1), (3, 3)):
            got = plan.list(kind, b)
            want = [k for k in tr.list(b, okind).tolist() if occ_of[k]] if occ[b] else []
            if kind == 1:
                # V rows are ordered by offset index; compare as sets, then check the order
                assert sorted(got.tolist()) == sorted(want)
                offs = []
                for k in got.tolist():
                    s = keys.tolist().index(k)
                    d = _index(keys[b]) - _index(keys[s])
                    offs.append(oracle.lib().orc_offset_index(*[int(t) for t in d]))
                assert offs == sorted(offs) and min(offs, default=0) >= 0
                offsets_checked += len(offs)
            else:
                assert got.tolist() == sorted(want, key=lambda k: keys.tolist().index(k))
        if is_leaf:
            j = int(np.searchsorted(leaf_ids, b))
            near = plan.list(0, j).tolist()
            want_u = [k for k in tr.list(b, 0).tolist() if occ_of[k]] if occ[b] else []
            if occ[b]:
                want_u = want_u + [int(keys[b])]
            pos = {k: i for i, k in enumerate(keys.tolist())}
            assert near == sorted(want_u, key=lambda k: pos[k])
            w = plan.list(2, j).tolist()
            want_w = [k for k in tr.list(b, 2).tolist() if occ_of[k]] if occ[b] else []
            assert w == sorted(want_w, key=lambda k: pos[k])
    return offsets_checked


def _index(key):
    key = int(key)
    level = key & 0x7FFF
    m = key >> 15
    v = [0, 0, 0]
    for bit in range(16):
        v[0] |= ((m >> (3 * bit + 2)) & 1) << bit
        v[1] |= ((m >> (3 * bit + 1)) & 1) << bit
        v[2] |= ((m >> (3 * bit)) & 1) << bit
    return np.array([c >> (16 - level) for c in v], dtype=np.int64)


@pytest.mark.parametrize("p", [3, 6])
def test_tables_equal_oracle(oracle, p):
    x, _ = oracle.point_sets("cube", 200, 1)
    plan = F.FmmBuilder(p).plan(x)
    m2l, m2m, l2l = plan.tables()
    om2l, om2m, ol2l = oracle.tables(p)
    for a, b in ((m2l, om2l), (m2m, om2m), (l2l, ol2l)):
        assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()


def test_uniform_cube_counts(oracle):
    # the reference's N = 1e5 uniform cube at 64 keys per leaf: a uniform level-4 tree,
    # 640,584 V pairs and 58.1e6 near pairs (fmm-bench/results/phase4s-gh200.md:69-72,346,397)
    x, _ = oracle.point_sets("cube", 100000, 0xBE9C06)
    info = F.FmmBuilder(6).max_points_per_leaf(64).plan(x).info()
    assert info["nleaves"] == 4096 and info["nlevels"] == 5
    assert info["v_pairs"] == 640584
    assert abs(info["near_pairs"] - 58.1e6) < 0.1e6


def test_settings_errors():
    x = np.random.default_rng(0).uniform(size=(10, 3))
    with pytest.raises(F.FmmError):
        F.FmmBuilder(4).max_points_per_leaf(0).plan(x)
    with pytest.raises(F.FmmError):
        F.FmmBuilder(4).plan(np.zeros((5, 3)))  # spans no volume
    bad = x.copy()
    bad[3, 1] = np.nan
    with pytest.raises(F.FmmError):
        F.FmmBuilder(4).plan(bad)


def test_a_reused_builder_leaves_earlier_handles_alone(tmp_path):
    """Output buffers are sized from the handle's own settings: changing the builder after a
    build (more vectors, no gradients) must not change what the earlier handle expects."""
    x = np.random.default_rng(2).uniform(size=(300, 3))
    b = F.FmmBuilder(4).vectors(3).gradients().table_cache(tmp_path)
    first = b.plan(x)
    second = b.vectors(1).gradients(False).max_points_per_leaf(16).plan(x)
    assert (first.settings.vectors, first.settings.gradients) == (3, 1)
    assert (second.settings.vectors, second.settings.gradients) == (1, 0)
    assert first.settings.table_cache is None and second.settings.table_cache is None
    first.close()
    second.close()


def _edge_sets():
    rng = np.random.default_rng(31)
    line = np.zeros((700, 3))
    line[:, 0] = rng.uniform(-1, 1, 700)  # collinear
    plane = np.column_stack([rng.uniform(0, 1, 900), rng.uniform(0, 1, 900), np.full(900, 0.25)])
    dup = np.repeat(rng.uniform(0, 1, (7, 3)), 150, axis=0)  # 7 sites of 150 coincident points
    tiny = rng.uniform(0, 1e-9, (500, 3)) + 3.0  # a cloud of width 1e-9 far from the origin
    huge = rng.uniform(-1e9, 1e9, (500, 3))
    clumps = np.concatenate([rng.normal(0, 1e-6, (400, 3)), rng.uniform(-1, 1, (400, 3))])  # ragged depth
    return {"two points": np.array([[0.0, 0, 0], [1.0, 1, 1]]),
            "collinear": line, "planar": plane, "duplicates": dup, "tiny": tiny, "huge": huge,
            "clumps": clumps}


def test_degenerate_domain_is_an_error():
    """A domain of no volume (one point, or every point coincident) is refused at build, as
    the reference's compute_global_bounding_box refuses it (octree/src/lib.rs:67-68)."""
    for x in (np.array([[0.3, 0.2, 0.1]]), np.repeat([[1.0, 2.0, 3.0]], 50, axis=0)):
        with pytest.raises(F.FmmError, match="no volume"):
            F.FmmBuilder(3).plan(x)


@pytest.mark.parametrize("name", list(_edge_sets()))
def test_tree_equals_oracle_on_edge_cases(oracle, name):
    """Degenerate point sets (two points, collinear and planar clouds, coincident points
    beyond the leaf limit, extreme scales, deep clumps beside a uniform cloud): the tree
    equals the oracle's restatement key for key."""
    x = _edge_sets()[name]
    for mk in (1, 16):
        plan = F.FmmBuilder(3).max_points_per_leaf(mk).plan(x)
        keys, leaf = plan.boxes()
        tr = oracle.Tree(x, x, 16, mk)
        assert np.array_equal(keys, tr.keys), (name, mk)
        assert np.array_equal(leaf, tr.is_leaf), (name, mk)
        info = plan.info()
        assert info["nsources"] == len(x) and info["nleaves"] == int(leaf.sum())
        plan.close()


@pytest.mark.parametrize("n", [20000, 150000])  # one host thread (sweep) and several
def test_plan_is_invariant_to_the_point_order(oracle, n):
    """Permuting the input points leaves the boxes and every list unchanged, and each leaf
    holds the same points (its order is the caller order, so the permuted indices sorted)."""
    x, _ = oracle.point_sets("sphere", n, 29)
    perm = np.random.default_rng(n).permutation(n)
    b = F.FmmBuilder(4).max_points_per_leaf(32)
    pa, pb = b.plan(x).plan_arrays(), b.plan(x[perm]).plan_arrays()
    for name in ("keys", "is_leaf", "level_start", "source_offsets", "near_rows", "near", "w_rows", "w",
                 "x_rows", "x", "v_rows", "v", "v_offsets"):
        assert np.array_equal(pa[name], pb[name]), name
    off = pa["source_offsets"]
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)  # original index -> index in the permuted input
    for j in np.linspace(0, len(off) - 2, 400).astype(np.int64):
        want = np.sort(inv[pa["source_order"][off[j]:off[j + 1]]])
        assert np.array_equal(pb["source_order"][off[j]:off[j + 1]], want), j
