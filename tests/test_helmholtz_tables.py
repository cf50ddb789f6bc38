"""The product's dense Helmholtz M2L tables (host code, fmmgpu_helmholtz_m2l_tables; the
reference's DenseM2l layout, fmm-tables/src/helmholtz/dense.rs) against the oracle's
projection, offset by offset, and through an M2L against the direct sum.  No device."""
import numpy as np
import pytest

import fmm_b200 as F
from oracle import oracle as O

# the 316 V-list offsets in index order (max |component| 2 or 3 in [-3, 3]^3)
OFFSETS = [(x, y, z) for x in range(-3, 4) for y in range(-3, 4) for z in range(-3, 4)
           if max(abs(x), abs(y), abs(z)) >= 2]


@pytest.mark.parametrize("p,k,r", [(4, 3.0, 0.5), (6, 0.4, 0.25)])
def test_tables_equal_the_oracle_projection(p, k, r):
    T = F.helmholtz_m2l_tables(p, k, r)
    n = (p + 1) ** 2
    assert T.shape == (316, 2 * n, n) and len(OFFSETS) == 316
    for i in (0, 57, 158, 200, 315):
        ref = O.hh_m2l_dense(p, k, r, OFFSETS[i])
        assert np.abs(T[i] - ref).max() < 1e-13 * np.abs(ref).max(), OFFSETS[i]


def test_table_m2l_against_the_direct_sum():
    p, k, r = 8, 3.0, 0.5
    T = F.helmholtz_m2l_tables(p, k, r)
    i = OFFSETS.index((3, -3, 2))
    rng = np.random.default_rng(17)
    src = rng.uniform(-r, r, (10, 3))
    q = rng.standard_normal(10) + 1j * rng.standard_normal(10)
    ct = 2 * r * np.array(OFFSETS[i], dtype=float)
    tgt = ct + rng.uniform(-r, r, (6, 3))
    L = O.hh_apply_dense(T[i], O.hh_p2m(p, k, r, np.zeros(3), src, q))
    phi, _ = O.hh_eval(p, k, r, ct, L, tgt, singular=False)
    ex, _ = O.helmholtz_direct_sum(k, src, q, tgt)
    assert np.abs(phi - ex).max() / np.abs(ex).max() < 5e-5  # p = 8 at ratio 0.23: ~6e-6 measured


def test_invalid_arguments():
    for args in ((31, 1.0, 0.5), (4, 0.0, 0.5), (4, 1.0, -1.0), (4, float("inf"), 0.5)):
        with pytest.raises(F.FmmError):
            F.helmholtz_m2l_tables(*args)


def _octant_centre(o, r):
    return np.array([0.5 * r if (o >> 2) & 1 else -0.5 * r, 0.5 * r if (o >> 1) & 1 else -0.5 * r,
                     0.5 * r if o & 1 else -0.5 * r])


def test_octant_tables_equal_the_oracle_projection_and_translate():
    p, k, r = 6, 2.0, 0.5
    m2m, l2l = F.helmholtz_octant_tables(p, k, r)
    n = (p + 1) ** 2
    assert m2m.shape == (8, 2 * n, n) and l2l.shape == (8, 2 * n, n)
    rng = np.random.default_rng(18)
    for o in (0, 3, 5, 7):
        cc = _octant_centre(o, r)
        for j in (0, 7, n - 1):
            e = np.zeros(n, dtype=np.complex128)
            e[j] = 1.0
            up = O.hh_translate("m2m", p, p, k, 0.5 * r, cc, r, np.zeros(3), e)
            down = O.hh_translate("l2l", p, p, k, r, np.zeros(3), 0.5 * r, cc, e)
            assert np.abs(m2m[o][:n, j] + 1j * m2m[o][n:, j] - up).max() < 1e-12 * np.abs(up).max()
            # a local's high degrees carry the quadrature's rounding divided by jh_n(k a)
            # (fmm-ref/src/helmholtz/direct.rs:27-33): the two orders of summation differ there
            assert np.abs(l2l[o][:n, j] + 1j * l2l[o][n:, j] - down).max() < 1e-10 * np.abs(down).max()
    # a child's sources through the M2M table, seen from far away
    o = 6
    cc = _octant_centre(o, r)
    src = cc + rng.uniform(-0.5 * r, 0.5 * r, (6, 3))
    q = rng.standard_normal(6) + 1j * rng.standard_normal(6)
    Mp = O.hh_apply_dense(m2m[o], O.hh_p2m(p, k, 0.5 * r, cc, src, q))
    v = rng.standard_normal((5, 3))
    tgt = 3.0 * v / np.linalg.norm(v, axis=1)[:, None]
    phi, _ = O.hh_eval(p, k, r, np.zeros(3), Mp, tgt, singular=True)
    ex, _ = O.helmholtz_direct_sum(k, src, q, tgt)
    assert np.abs(phi - ex).max() / np.abs(ex).max() < 1e-4


def test_tables_scale_with_the_box():
    """Only k r and the geometry in units of r enter: an M2L table of boxes of half-width r
    is 1/r times the table of unit boxes at the wavenumber k r (the 4 pi i k of a
    multipole's field carries the 1/length), and the M2M/L2L tables are scale free; so a
    level's tables in leaf-scaled units (half-width 1, k_l = k r_l) serve every box size."""
    p, k, r = 5, 3.0, 0.125
    a = F.helmholtz_m2l_tables(p, k, r)
    b = F.helmholtz_m2l_tables(p, k * r, 1.0)
    assert np.abs(a - b / r).max() < 1e-11 * np.abs(a).max()
    m_a, l_a = F.helmholtz_octant_tables(p, k, r)
    m_b, l_b = F.helmholtz_octant_tables(p, k * r, 1.0)
    assert np.abs(m_a - m_b).max() < 1e-11 * np.abs(m_a).max()
    assert np.abs(l_a - l_b).max() < 1e-9 * np.abs(l_a).max()
