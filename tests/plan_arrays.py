"""Plans in the reference's flattened layout (fmmgpu_plan_arrays) made from the oracle's
restated octree and brute-force list rule, for the plan-upload tests (test
infrastructure: reads the oracle)."""
import ctypes as C

import numpy as np

LEVEL_MASK = 0x7FFF


def _index(key):
    key = int(key)
    level = key & LEVEL_MASK
    m = key >> 15
    v = [0, 0, 0]
    for bit in range(16):
        v[0] |= ((m >> (3 * bit + 2)) & 1) << bit
        v[1] |= ((m >> (3 * bit + 1)) & 1) << bit
        v[2] |= ((m >> (3 * bit)) & 1) << bit
    return [c >> (16 - level) for c in v]


def oracle_plan(oracle, src, tgt, max_keys):
    """The oracle's tree (octree refine + 2:1 balance) and lists (fmm-plan's rule, boxes
    without sources kept) as a plan dict; points in leaf order, caller order within a leaf."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    L = oracle.lib()
    tr = oracle.Tree(src, tgt, 16, max_keys)
    keys = tr.keys
    levels = (keys & np.uint64(LEVEL_MASK)).astype(np.int64)
    nlev = int(levels.max()) + 1
    level_start = np.searchsorted(levels, np.arange(nlev + 1)).astype(np.int64)
    leaves = np.flatnonzero(tr.is_leaf)
    leaf_of_box = {int(b): j for j, b in enumerate(leaves)}
    box_of_key = {int(k): b for b, k in enumerate(keys)}
    lower, side = np.zeros(3), C.c_double()
    L.orc_tree_domain(tr._t, lower, C.byref(side))
    box6, lw, sd = np.zeros(6), np.zeros(3), C.c_double()
    L.orc_domain(len(src), src, len(tgt), tgt, lw, C.byref(sd), box6)

    def leaf_index(pts):
        out = np.empty(len(pts), dtype=np.int64)
        for i, x in enumerate(pts):
            fine = int(L.orc_point_key(np.ascontiguousarray(x), box6, 16))
            for lev in range(nlev - 1, -1, -1):
                shift = 15 + 3 * (16 - lev)
                k = ((fine >> shift) << shift) | lev
                b = box_of_key.get(k)
                if b is not None and tr.is_leaf[b]:
                    out[i] = leaf_of_box[b]
                    break
        return out

    plan = {"nlevels": nlev, "level_start": level_start, "keys": keys, "is_leaf": tr.is_leaf.astype(np.uint8),
            "lower": lower, "side": side.value}
    for name, pts in (("source", src), ("target", tgt)):
        lf = leaf_index(pts)
        order = np.argsort(lf, kind="stable")
        plan[f"{name}_order"] = order.astype(np.int64)
        plan[f"{name}_offsets"] = np.concatenate([[0], np.cumsum(np.bincount(lf, minlength=len(leaves)))]).astype(np.int64)

    def csr(rows):
        r = np.concatenate([[0], np.cumsum([len(x) for x in rows])]).astype(np.int64)
        c = np.array([v for x in rows for v in x], dtype=np.int32)
        return r, c

    near, w = [], []
    for j, b in enumerate(leaves):
        near.append(sorted([leaf_of_box[box_of_key[int(k)]] for k in tr.list(int(b), 0)] + [j]))
        w.append(sorted(box_of_key[int(k)] for k in tr.list(int(b), 2)))
    x, v, voff = [], [], []
    for b in range(len(keys)):
        x.append(sorted(leaf_of_box[box_of_key[int(k)]] for k in tr.list(b, 3)))
        row = []
        tb = _index(keys[b])
        for k in tr.list(b, 1):
            s = box_of_key[int(k)]
            sb = _index(keys[s])
            d = L.orc_offset_index(tb[0] - sb[0], tb[1] - sb[1], tb[2] - sb[2])
            row.append((d, s))
        row.sort()
        v.append([s for _, s in row])
        voff.append([d for d, _ in row])
    plan["near_rows"], plan["near"] = csr(near)
    plan["w_rows"], plan["w"] = csr(w)
    plan["x_rows"], plan["x"] = csr(x)
    plan["v_rows"], plan["v"] = csr(v)
    plan["v_offsets"] = csr(voff)[1]
    return plan
