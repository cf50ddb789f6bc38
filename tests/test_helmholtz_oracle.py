"""The Helmholtz oracle (e^{ikr}/r, fmm-ref/src/helmholtz/p2p.rs restated) pinned to FMM3D
v2.1.0's direct sums (tests/golden/helmholtz_fmm3d.json, from the reference's fixture)."""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "helmholtz_fmm3d.json"
FOUR_PI = 4.0 * np.pi


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def golden():
    d = json.loads(GOLDEN.read_text())
    src = np.array(d["sources"], dtype=np.float64)
    tgt = np.array(d["targets"], dtype=np.float64)
    charges = {name: np.array([complex(float(a), float(b)) for a, b in v]) for name, v in d["charges"].items()}
    points = np.concatenate([src, tgt])
    cases = []
    for c in d["cases"]:
        k = complex(float(c["k"][0]), float(c["k"][1]))
        pot = np.array([complex(float(a), float(b)) for a, b in c["potential"]])
        g = np.array([[complex(float(r[2 * j]), float(r[2 * j + 1])) for j in range(3)] for r in c["gradient"]])
        cases.append((c["label"], k, charges[c["charges"]], np.array(c["points"]), pot, g))
    return src, points, cases


@pytest.mark.parametrize("i", range(7))
def test_direct_sum_matches_fmm3d(oracle, i):
    src, points, cases = golden()
    label, k, q, idx, pot, g = cases[i]
    phi, grad = oracle.helmholtz_direct_sum(k, src, q, points[idx])
    assert rel(phi / FOUR_PI, pot) < 1e-13, label
    assert rel(grad / FOUR_PI, g) < 1e-13, label


def test_doc_example(oracle):
    """fmm-ref/src/helmholtz/p2p.rs module example: e^{ikr}/r at k r = 1."""
    phi, _ = oracle.helmholtz_direct_sum(0.5, np.zeros((1, 3)), np.array([1.0 + 0j]), np.array([[0.0, 0.0, 2.0]]),
                                         gradients=False)
    assert abs(phi[0].real - np.cos(1.0) / 2) < 1e-16 and abs(phi[0].imag - np.sin(1.0) / 2) < 1e-16


def test_p2p_equals_direct_sum_and_laplace_at_k0(oracle):
    rng = np.random.default_rng(3)
    src = rng.uniform(size=(300, 3))
    tgt = np.concatenate([rng.uniform(size=(50, 3)), src[:5]])  # coincident pairs skipped
    q = rng.normal(size=300) + 1j * rng.normal(size=300)
    a, ga = oracle.helmholtz_p2p(3.0 + 0.5j, src, q, tgt)
    b, gb = oracle.helmholtz_direct_sum(3.0 + 0.5j, src, q, tgt)
    assert rel(a, b) < 1e-14 and rel(ga, gb) < 1e-14
    lap, _ = oracle.p2p(src, q.real, tgt, gradients=False)
    h0, _ = oracle.helmholtz_p2p(0.0, src, q.real.astype(np.complex128), tgt, gradients=False)
    assert np.array_equal(h0.real, lap) and not h0.imag.any()


def test_near_field_of_a_single_leaf_is_the_direct_sum(oracle):
    rng = np.random.default_rng(4)
    x = rng.uniform(size=(200, 3))
    q = rng.normal(size=200) + 1j * rng.normal(size=200)
    phi, g = oracle.helmholtz_near(x, q, x, 7.0 + 1.0j, 256, gradients=True)
    d, dg = oracle.helmholtz_direct_sum(7.0 + 1.0j, x, q, x)
    assert rel(phi[0], d / FOUR_PI) < 1e-13 and rel(g[0], dg / FOUR_PI) < 1e-13
