"""The oracle's Helmholtz expansions (real k): the reference's real orthonormal harmonics
and scaled radial functions, the leaf operators P2M / L2P / P2L / M2P and the
translations M2M / L2L / M2L by projection on a sphere (fmm-ref/src/helmholtz/leaf.rs,
direct.rs), pinned against the direct sum (itself pinned to FMM3D's values in
test_helmholtz_oracle) on the reference's own test geometry: sources in the box,
targets at 2.5 a or more (leaf.rs "Tested range"), translations between an octree pair
and between two boxes of one level.  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_harmonics_values_and_orthonormality():
    # the reference's documented values (fmm-math/src/orthonormal/harmonics.rs:19-30)
    y = O.hh_harmonics(1, [0.0, 3.0, 4.0])
    c = np.sqrt(3.0 / (4.0 * np.pi))
    assert abs(y[0] - 1.0 / np.sqrt(4.0 * np.pi)) < 1e-15
    assert abs(y[2] - 0.8 * c) < 1e-15 and abs(y[1] - 0.6 * c) < 1e-15 and abs(y[3]) < 1e-15
    # on the north pole: d_theta Y_1^1 = c and (1/sin theta) d_phi Y_1^-1 = c (harmonics.rs:93-100)
    _, dt, df = O.hh_harmonics(1, [0.0, 0.0, 1.0], derivatives=True)
    assert abs(dt[3] - c) < 1e-15 and abs(df[1] - c) < 1e-15 and abs(dt[2]) < 1e-15
    # orthonormal on the sphere (Gauss-Legendre x uniform rule, exact to degree 2p)
    p = 8
    x, w = np.polynomial.legendre.leggauss(p + 2)
    nphi = 2 * p + 2
    gram = np.zeros(((p + 1) ** 2, (p + 1) ** 2))
    for ct, wt in zip(x, w):
        st = np.sqrt(1.0 - ct * ct)
        for j in range(nphi):
            f = 2.0 * np.pi * j / nphi
            yy = O.hh_harmonics(p, [st * np.cos(f), st * np.sin(f), ct])
            gram += wt * (2.0 * np.pi / nphi) * np.outer(yy, yy)
    assert np.abs(gram - np.eye(len(gram))).max() < 1e-13


def test_angular_derivatives_against_differences():
    p, h = 6, 1e-6
    x = np.array([0.3, -0.5, 0.7])
    r = np.linalg.norm(x)
    theta, phi = np.arccos(x[2] / r), np.arctan2(x[1], x[0])

    def at(t, f):
        return O.hh_harmonics(p, [np.sin(t) * np.cos(f), np.sin(t) * np.sin(f), np.cos(t)])

    _, dt, df = O.hh_harmonics(p, x, derivatives=True)
    assert np.abs(dt - (at(theta + h, phi) - at(theta - h, phi)) / (2 * h)).max() < 1e-8
    assert np.abs(df - (at(theta, phi + h) - at(theta, phi - h)) / (2 * h) / np.sin(theta)).max() < 1e-8


@pytest.mark.parametrize("x", [1e-4, 0.3, 2.0, 15.0, 60.0, 300.0])
def test_radial_functions(x):
    p = 40
    jh, jhp, hh, hhp = O.hh_radial(p, x)
    j, y = hh.real, hh.imag
    # closed forms of orders 0 and 1, the Wronskian j_n y_{n-1} - j_{n-1} y_n = 1/x^2
    assert abs(j[0] - np.sin(x) / x) < 1e-15 and abs(y[0] + np.cos(x) / x) < 1e-15 * max(1.0, 1.0 / x)
    w = (j[1:] * y[:-1] - j[:-1] * y[1:]) * x * x
    assert np.abs(w - 1.0).max() < 1e-12
    assert np.array_equal(jh, j)  # s = 1: jh = j
    # derivatives: j_0' = -j_1, and the recurrences against a difference quotient
    assert jhp[0] == -jh[1]
    if x >= 0.1:
        d = 1e-6 * x
        jp, _, hp, _ = O.hh_radial(p, x + d)
        jm, _, hm, _ = O.hh_radial(p, x - d)
        env = np.maximum(np.abs(jh[:10]), np.abs(hh[:10]))  # j_n has zeros: relative to |h_n|
        assert np.all(np.abs(jhp[:10] - (jp[:10] - jm[:10]) / (2 * d)) < 1e-6 * env)
        assert np.all(np.abs(hhp[:10] - (hp[:10] - hm[:10]) / (2 * d)) < 1e-6 * np.abs(hhp[:10]))


def test_scaled_radial_functions():
    x, s, p = 0.05, 0.1, 12
    jh, _, hh, _ = O.hh_radial(p, x, s)
    j1, _, h1, _ = O.hh_radial(p, x, 1.0)
    n = np.arange(p + 1)
    assert np.allclose(jh, j1 / s ** n, rtol=1e-14, atol=0)
    assert np.allclose(hh, h1 * s ** n, rtol=1e-14, atol=0)


K = 2.0
CENTRE = np.zeros(3)


def _problem(seed, n=8):
    rng = np.random.default_rng(seed)
    return rng, rng.uniform(-0.5, 0.5, (n, 3)), rng.standard_normal(n) + 1j * rng.standard_normal(n)


def _shell(rng, n, radius):
    v = rng.standard_normal((n, 3))
    return radius * v / np.linalg.norm(v, axis=1)[:, None]


# Sources within sqrt(3) r = 0.87 of the centre and targets at 3 (or the reverse): the
# geometric ratio is 0.29, so the truncation error falls like 0.29^(p+1) (about 1e-6 at
# p = 10 and 5e-12 at p = 20); the tolerances leave a margin over that bound.
@pytest.mark.parametrize("p,tol", [(10, 1e-4), (20, 1e-9)])
def test_p2m_m2p(p, tol):
    rng, src, q = _problem(11)
    tgt = _shell(rng, 6, 3.0)
    M = O.hh_p2m(p, K, 0.5, CENTRE, src, q)
    phi, g = O.hh_eval(p, K, 0.5, CENTRE, M, tgt, singular=True)
    ex, eg = O.helmholtz_direct_sum(K, src, q, tgt)
    assert rel(phi, ex) < tol and rel(g, eg) < tol


@pytest.mark.parametrize("p,tol", [(10, 1e-4), (20, 1e-9)])
def test_p2l_l2p(p, tol):
    rng, tgt, q = _problem(12, 6)
    tgt[0] = 0.0  # the centre: the gradient's limit
    far = _shell(rng, 6, 3.0)
    L = O.hh_p2m(p, K, 0.5, CENTRE, far, q, singular=True)
    phi, g = O.hh_eval(p, K, 0.5, CENTRE, L, tgt, singular=False)
    ex, eg = O.helmholtz_direct_sum(K, far, q, tgt)
    assert rel(phi, ex) < tol and rel(g, eg) < tol


def test_real_charges_give_a_real_multipole():
    """For a real k and real charges the multipole is real (leaf.rs "Storage")."""
    _, src, q = _problem(13)
    M = O.hh_p2m(8, K, 0.5, CENTRE, src, q.real.astype(np.complex128))
    assert np.all(M.imag == 0.0)


def test_m2m_l2l_on_an_octree_pair():
    rng, _, q = _problem(14, 6)
    child = np.array([0.25, -0.25, 0.25])
    src = child + rng.uniform(-0.25, 0.25, (6, 3))
    tgt = _shell(rng, 5, 3.0)
    M = O.hh_translate("m2m", 16, 16, K, 0.25, child, 0.5, CENTRE, O.hh_p2m(16, K, 0.25, child, src, q))
    phi, g = O.hh_eval(16, K, 0.5, CENTRE, M, tgt, singular=True)
    ex, eg = O.helmholtz_direct_sum(K, src, q, tgt)
    assert rel(phi, ex) < 1e-8 and rel(g, eg) < 1e-8
    far = _shell(rng, 6, 3.0)
    inner = child + rng.uniform(-0.25, 0.25, (5, 3))
    L = O.hh_translate("l2l", 16, 16, K, 0.5, CENTRE, 0.25, child, O.hh_p2m(16, K, 0.5, CENTRE, far, q, singular=True))
    phi, g = O.hh_eval(16, K, 0.25, child, L, inner, singular=False)
    ex, eg = O.helmholtz_direct_sum(K, far, q, inner)
    assert rel(phi, ex) < 1e-8 and rel(g, eg) < 1e-7


@pytest.mark.parametrize("k,p,tol", [(2.0, 10, 1e-5), (2.0, 20, 1e-10), (20.0, 20, 5e-2), (20.0, 30, 1e-6)])
def test_m2l_between_boxes_of_one_level(k, p, tol):
    """Two boxes of half-width 0.5 four apart; at k = 20 (k a = 17) a box is 2.75
    wavelengths across and the expansion needs a degree well above k a."""
    rng, src, q = _problem(15)
    ct = np.array([4.0, 0.0, 0.0])
    tgt = ct + rng.uniform(-0.5, 0.5, (5, 3))
    L = O.hh_translate("m2l", p, p, k, 0.5, CENTRE, 0.5, ct, O.hh_p2m(p, k, 0.5, CENTRE, src, q))
    phi, g = O.hh_eval(p, k, 0.5, ct, L, tgt, singular=False)
    ex, eg = O.helmholtz_direct_sum(k, src, q, tgt)
    assert rel(phi, ex) < tol and rel(g, eg) < tol


def test_dense_m2l_table():
    """The dense M2L of one offset (fmm-tables/src/helmholtz/dense.rs layout: a real 2n x n
    matrix, column j the local of the unit real multipole e_j, real plane over imaginary
    plane) equals the projection M2L column by column, and applied to a complex multipole
    gives the projection's local of it."""
    p, k, r = 6, 3.0, 0.5
    n = (p + 1) ** 2
    off = (2, 1, -1)
    ct = 2 * r * np.array(off, dtype=float)
    T = O.hh_m2l_dense(p, k, r, off)
    assert T.shape == (2 * n, n)
    for j in (0, 5, n - 1):
        e = np.zeros(n, dtype=np.complex128)
        e[j] = 1.0
        col = O.hh_translate("m2l", p, p, k, r, CENTRE, r, ct, e)
        assert np.abs(T[:n, j] + 1j * T[n:, j] - col).max() < 1e-12 * np.abs(col).max()
    rng, src, q = _problem(16)
    M = O.hh_p2m(p, k, r, CENTRE, src, q)
    L = O.hh_translate("m2l", p, p, k, r, CENTRE, r, ct, M)
    assert np.abs(O.hh_apply_dense(T, M) - L).max() < 1e-12 * np.abs(L).max()


def test_helmholtz_fmm_against_the_direct_sum():
    """The oracle's Helmholtz FMM (the Laplace plan's tree and lists, these expansions,
    dense M2L tables per level and offset) on 1,200 points in the unit cube, k = 5,
    complex charges: relative L2 error against the direct sum at degree 6 (measured 9e-5
    at N = 1,500; 2.4e-6 at degree 10)."""
    rng = np.random.default_rng(5)
    x = rng.uniform(0.0, 1.0, (1200, 3))
    q = rng.standard_normal(1200) + 1j * rng.standard_normal(1200)
    phi, g = O.helmholtz_fmm(x, q, x, 5.0, 6, 64)
    ex, eg = O.helmholtz_direct_sum(5.0, x, q, x)
    assert np.linalg.norm(phi - ex) / np.linalg.norm(ex) < 5e-4
    assert np.linalg.norm(g - eg) / np.linalg.norm(eg) < 1e-3
