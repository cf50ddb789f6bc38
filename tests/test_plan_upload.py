"""Plans from outside the library (fmmgpu_plan_from_arrays, the host half of
fmmgpu_upload_plan): the reference's flattened layout round-trips, the oracle's plan is
accepted, and each check refuses a broken plan with a message (no GPU needed)."""
import numpy as np
import pytest

import fmm_b200 as F
from tests.plan_arrays import oracle_plan


def same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert np.allclose(a[k], b[k]), k


def test_library_plan_round_trips():
    x = np.random.default_rng(1).uniform(size=(4000, 3))
    plan = F.FmmBuilder(4).max_points_per_leaf(16).plan(x)
    arrays = plan.plan_arrays()
    again = F.FmmBuilder(4).plan_from(arrays, x)
    same(arrays, again.plan_arrays())
    keys, leaf = plan.boxes()
    k2, l2 = again.boxes()
    assert np.array_equal(keys, k2) and np.array_equal(leaf, l2)
    assert again.info()["near_pairs"] == plan.info()["near_pairs"]


@pytest.mark.parametrize("kind,n,mk", [("cube", 1500, 16), ("sphere", 2000, 12)])
def test_oracle_plan_is_accepted_and_round_trips(oracle, kind, n, mk):
    x, _ = oracle.point_sets(kind, n, 7)
    arrays = oracle_plan(oracle, x, x, mk)
    got = F.FmmBuilder(4).plan_from(arrays, x)
    same(arrays, got.plan_arrays())
    own = F.FmmBuilder(4).max_points_per_leaf(mk).plan(x)
    keys, leaf = own.boxes()
    assert np.array_equal(keys, arrays["keys"]) and np.array_equal(leaf, arrays["is_leaf"])


def _broken(arrays, **changes):
    a = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in arrays.items()}
    for k, f in changes.items():
        f(a[k]) if callable(f) else a.__setitem__(k, f)
    return a


@pytest.mark.parametrize("what,change", [
    ("near entry out of range", {"near": lambda a: a.__setitem__(0, 10**6)}),
    ("not ascending", {"near": lambda a: a.__setitem__(slice(0, 2), a[:2][::-1].copy())}),
    ("V offset", {"v_offsets": lambda a: a.__setitem__(0, (a[0] + 1) % 316)}),
    ("not a permutation", {"source_order": lambda a: a.__setitem__(0, a[1])}),
    ("keys of level", {"keys": lambda a: a.__setitem__(slice(1, 3), a[1:3][::-1].copy())}),
    ("outside its leaf", {"source_order": lambda a: a.__setitem__(slice(None), a[::-1].copy())}),
])
def test_broken_plans_are_refused(what, change):
    x = np.random.default_rng(2).uniform(size=(3000, 3))
    arrays = F.FmmBuilder(4).max_points_per_leaf(16).plan(x).plan_arrays()
    assert arrays["v"].size and arrays["near_rows"][1] >= 2
    with pytest.raises(F.FmmError) as e:
        F.FmmBuilder(4).plan_from(_broken(arrays, **change), x)
    assert e.value.status == 1 and what in str(e.value), str(e.value)
