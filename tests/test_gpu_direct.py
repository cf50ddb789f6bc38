"""The GPU f64 direct sum (the error reference of every bench leg) against the oracle's
Neumaier direct sum (fmm-ref/src/p2p.rs:147-186), coincident points included (needs a
B200: -m gpu).  The GPU sums each target's sources in chunks with Neumaier compensation
and combines the chunks compensated, so it agrees with the serial sum to the last bits
(relative 1e-15), not bit for bit."""
import numpy as np
import pytest

import fmm_b200 as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("ns,nt", [(1, 1), (1000, 257), (70_000, 3000)])
def test_direct_sum_matches_oracle(oracle, ns, nt):
    rng = np.random.default_rng(ns + nt)
    src = rng.uniform(-1, 1, (ns, 3))
    tgt = np.concatenate([rng.normal(0.0, 0.5, (nt, 3)), src[: min(ns, 50)]])  # some coincide
    q = rng.standard_normal(ns)
    phi, g = F.direct_sum(src, q, tgt, gradients=True)
    ophi, og = oracle.direct_sum(src, q, tgt, gradients=True)
    ophi, og = ophi / (4 * np.pi), og / (4 * np.pi)
    assert np.all(np.isfinite(phi)) and np.all(np.isfinite(g))
    assert rel(phi, ophi) < 1e-15 and rel(g, og) < 1e-15, (rel(phi, ophi), rel(g, og))


def test_direct_sum_exact_answer():
    """fmm-ref/src/p2p.rs:48-64: charges 2 and -1 at the origin and (3, 4, 0)."""
    pts = np.array([[0.0, 0.0, 0.0], [3.0, 4.0, 0.0]])
    phi, g = F.direct_sum(pts, np.array([2.0, -1.0]), pts, gradients=True)
    four_pi = 4 * np.pi
    assert np.allclose(phi * four_pi, [-1.0 / 5.0, 2.0 / 5.0], rtol=1e-15, atol=0)
    # grad at the origin of -1/|x - y|, y = (3, 4, 0): -(x - y)/|x - y|^3 times -1
    assert np.allclose(g[0] * four_pi, [-3.0 / 125.0, -4.0 / 125.0, 0.0], rtol=1e-15, atol=1e-18)
