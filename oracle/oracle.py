"""ctypes bindings of the oracle library (oracle/_build/liboracle.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py, never by the product package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_sz = C.c_size_t


def build():
    """Compiles the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        sig = {
            "orc_rng_next": (C.c_uint64, [C.c_void_p]),
            "orc_regular": (None, [C.c_int, _dp, _dp]),
            "orc_irregular": (None, [C.c_int, _dp, _dp]),
            "orc_regular_grad": (None, [C.c_int, _dp, _dp, _dp, _dp, _dp]),
            "orc_irregular_grad": (None, [C.c_int, _dp, _dp, _dp, _dp, _dp]),
            "orc_p2m": (None, [C.c_int, _dp, C.c_double, _sz, _dp, _dp, C.c_int, _dp]),
            "orc_p2l": (None, [C.c_int, _dp, C.c_double, _sz, _dp, _dp, C.c_int, _dp]),
            "orc_l2p": (None, [C.c_int, _dp, C.c_double, _dp, C.c_int, _sz, _dp, _dp, C.c_void_p]),
            "orc_m2p": (None, [C.c_int, _dp, C.c_double, _dp, C.c_int, _sz, _dp, _dp, C.c_void_p]),
            "orc_m2m": (None, [C.c_int, _dp, C.c_double, _dp, C.c_double, _dp, _dp]),
            "orc_l2l": (None, [C.c_int, _dp, C.c_double, _dp, C.c_double, _dp, _dp]),
            "orc_m2l": (None, [C.c_int, _dp, C.c_double, _dp, C.c_double, _dp, _dp]),
            "orc_build_m2l_tables": (None, [C.c_int, _dp]),
            "orc_build_m2m_tables": (None, [C.c_int, _dp]),
            "orc_build_l2l_tables": (None, [C.c_int, _dp]),
            "orc_offset_index": (C.c_int, [C.c_int64, C.c_int64, C.c_int64]),
            "orc_p2p": (None, [_sz, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_p2p_ref": (None, [_sz, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_direct_sum": (None, [_sz, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_direct_sum_omp": (None, [_sz, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_key_from_index": (C.c_uint64, [_u32p, C.c_int]),
            "orc_tree_build": (C.c_void_p, [_sz, _dp, _sz, _dp, C.c_int, C.c_int]),
            "orc_tree_free": (None, [C.c_void_p]),
            "orc_tree_nlevels": (C.c_int, [C.c_void_p]),
            "orc_tree_nboxes": (_sz, [C.c_void_p]),
            "orc_tree_nleaves": (_sz, [C.c_void_p]),
            "orc_tree_boxes": (None, [C.c_void_p, _u64p, _u8p]),
            "orc_tree_list": (_sz, [C.c_void_p, _sz, C.c_int, _u64p, _sz]),
            "orc_tree_domain": (None, [C.c_void_p, _dp, C.POINTER(C.c_double)]),
            "orc_domain": (None, [_sz, _dp, _sz, _dp, _dp, C.POINTER(C.c_double), _dp]),
            "orc_point_key": (C.c_uint64, [_dp, _dp, C.c_int]),
            "orc_key_decode": (None, [C.c_uint64, C.POINTER(C.c_int), _u32p]),
            "orc_fmm": (C.c_int, [_sz, _dp, _dp, C.c_int, _sz, _dp, C.c_int, C.c_int, C.c_int,
                                  C.c_int, _dp, C.c_void_p]),
            "orc_fmm_kinds": (C.c_int, [_sz, _dp, _dp, C.c_int, _sz, _dp, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int, _dp, C.c_void_p]),
            "orc_fmm_last_eval_seconds": (C.c_double, []),
            "orc_fmm_new": (C.c_void_p, [_sz, _dp, _sz, _dp, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_fmm_eval": (C.c_int, [C.c_void_p, _dp, C.c_int, C.c_int, _dp, C.c_void_p]),
            "orc_fmm_free": (None, [C.c_void_p]),
            "orc_fmm_set_host_path": (None, [C.c_void_p, C.c_int]),
            "orc_hp_has_avx512": (C.c_int, []),
            "orc_hp_p2p": (None, [_sz, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_helmholtz_p2p": (None, [C.c_double, C.c_double, _sz, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_helmholtz_direct_sum": (None, [C.c_double, C.c_double, _sz, _dp, _dp, _sz, _dp, _dp,
                                                C.c_void_p]),
            "orc_helmholtz_near": (C.c_int, [_sz, _dp, _dp, C.c_int, _sz, _dp, C.c_int, C.c_double, C.c_double,
                                             C.c_int, C.c_int, _dp, C.c_void_p]),
            "orc_hh_harmonics": (None, [C.c_int, _dp, _dp, C.c_void_p, C.c_void_p]),
            "orc_hh_radial": (None, [C.c_int, C.c_double, C.c_double, _dp, C.c_void_p, C.c_void_p, C.c_void_p]),
            "orc_hh_p2m": (None, [C.c_int, C.c_double, C.c_double, _dp, _sz, _dp, _dp, _dp]),
            "orc_hh_p2l": (None, [C.c_int, C.c_double, C.c_double, _dp, _sz, _dp, _dp, _dp]),
            "orc_hh_l2p": (None, [C.c_int, C.c_double, C.c_double, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_hh_m2p": (None, [C.c_int, C.c_double, C.c_double, _dp, _dp, _sz, _dp, _dp, C.c_void_p]),
            "orc_hh_m2m": (None, [C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_double, _dp, _dp, _dp]),
            "orc_hh_l2l": (None, [C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_double, _dp, _dp, _dp]),
            "orc_hh_m2l": (None, [C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_double, _dp, _dp, _dp]),
            "orc_hh_m2l_dense": (None, [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def nc(p):
    return (p + 1) ** 2


class Rng:
    """SplitMix64 (fmm-validate/src/rng.rs:24-45)."""

    def __init__(self, seed):
        self.state = C.c_uint64(seed)

    def next_u64(self):
        return lib().orc_rng_next(C.byref(self.state))


def regular(p, x):
    out = np.zeros(nc(p))
    lib().orc_regular(p, np.ascontiguousarray(x, dtype=np.float64), out)
    return out


def irregular(p, x):
    out = np.zeros(nc(p))
    lib().orc_irregular(p, np.ascontiguousarray(x, dtype=np.float64), out)
    return out


def regular_grad(p, x):
    v, gx, gy, gz = (np.zeros(nc(p)) for _ in range(4))
    lib().orc_regular_grad(p, np.ascontiguousarray(x, dtype=np.float64), v, gx, gy, gz)
    return v, np.stack([gx, gy, gz])


def irregular_grad(p, x):
    v, gx, gy, gz = (np.zeros(nc(p)) for _ in range(4))
    lib().orc_irregular_grad(p, np.ascontiguousarray(x, dtype=np.float64), v, gx, gy, gz)
    return v, np.stack([gx, gy, gz])


def tables(p):
    n = nc(p)
    m2l = np.zeros(316 * n * n)
    m2m = np.zeros(8 * n * n)
    l2l = np.zeros(8 * n * n)
    lib().orc_build_m2l_tables(p, m2l)
    lib().orc_build_m2m_tables(p, m2m)
    lib().orc_build_l2l_tables(p, l2l)
    # column-major storage: entry (i, k) at i + k n; return A with A[t] @ x = output
    return (m2l.reshape(316, n, n).transpose(0, 2, 1), m2m.reshape(8, n, n).transpose(0, 2, 1),
            l2l.reshape(8, n, n).transpose(0, 2, 1))


def p2p(src, q, tgt, gradients=True):
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    phi = np.zeros(len(tgt))
    g = np.zeros((len(tgt), 3)) if gradients else None
    lib().orc_p2p(len(src), src, q, len(tgt), tgt, phi, _ptr(g))
    return phi, g


def host_p2p(src, q, tgt, gradients=True):
    """The AVX-512 P2P of the reference's host path (oracle/hostpath.c), no 1/(4 pi)."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    phi = np.zeros(len(tgt))
    g = np.zeros(3 * len(tgt)) if gradients else None
    lib().orc_hp_p2p(len(src), src, q, len(tgt), tgt, phi, _ptr(g))
    return phi, (g.reshape(-1, 3) if gradients else None)


def direct_sum(src, q, tgt, gradients=True, threads=True):
    """Neumaier-compensated f64 direct sum of q/|x-y| (fmm-ref/src/p2p.rs:147-186)."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    phi = np.zeros(len(tgt))
    g = np.zeros((len(tgt), 3)) if gradients else None
    f = lib().orc_direct_sum_omp if threads else lib().orc_direct_sum
    f(len(src), src, q, len(tgt), tgt, phi, _ptr(g))
    return phi, g


def _cview(a):
    return np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)


# ---- Helmholtz expansions for a real k (helmholtz_ops.c) --------------------------------
# A complex expansion of degree p is returned as a complex array of (p + 1)^2 in the layout
# n^2 + n + m (the C side's two real planes); a box is its centre and half-width r.

def hh_harmonics(p, x, derivatives=False):
    """Real orthonormal Y_n^m of x's direction (and d_theta Y, (1/sin theta) d_phi Y)."""
    n = (p + 1) ** 2
    y = np.zeros(n)
    dt = np.zeros(n) if derivatives else None
    df = np.zeros(n) if derivatives else None
    lib().orc_hh_harmonics(p, np.ascontiguousarray(x, dtype=np.float64), y, _ptr(dt), _ptr(df))
    return (y, dt, df) if derivatives else y


def hh_radial(p, z, s=1.0, singular=True):
    """Scaled jh_n, jh_n' (and hh_n, hh_n' complex) at z, n = 0..p."""
    jh, jhp = np.zeros(p + 1), np.zeros(p + 1)
    hh = np.zeros(2 * (p + 1)) if singular else None
    hhp = np.zeros(2 * (p + 1)) if singular else None
    lib().orc_hh_radial(p, float(z), float(s), jh, _ptr(jhp), _ptr(hh), _ptr(hhp))
    if not singular:
        return jh, jhp
    return jh, jhp, hh.view(np.complex128), hhp.view(np.complex128)


def _planes(e):
    e = np.asarray(e, dtype=np.complex128)
    return np.ascontiguousarray(np.concatenate([e.real, e.imag]))


def _complex(planes):
    n = len(planes) // 2
    return planes[:n] + 1j * planes[n:]


def hh_p2m(p, k, r, c, src, q, singular=False):
    """P2M (or P2L with singular=True) of complex charges about centre c."""
    out = np.zeros(2 * (p + 1) ** 2)
    f = lib().orc_hh_p2l if singular else lib().orc_hh_p2m
    f(p, float(k), float(r), np.ascontiguousarray(c, dtype=np.float64), len(src),
      np.ascontiguousarray(src, dtype=np.float64), _cview(q), out)
    return _complex(out)


def hh_eval(p, k, r, c, e, tgt, singular):
    """L2P (singular=False) or M2P: phi (nt,) and grad (nt, 3) complex."""
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    phi = np.zeros(2 * len(tgt))
    g = np.zeros(6 * len(tgt))
    f = lib().orc_hh_m2p if singular else lib().orc_hh_l2p
    f(p, float(k), float(r), np.ascontiguousarray(c, dtype=np.float64), _planes(e), len(tgt), tgt, phi, _ptr(g))
    return phi.view(np.complex128), g.view(np.complex128).reshape(len(tgt), 3)


def hh_translate(kind, p_in, p_out, k, r_in, c_in, r_out, c_out, e):
    """M2M, L2L or M2L by projection: the output expansion (complex, (p_out + 1)^2)."""
    out = np.zeros(2 * (p_out + 1) ** 2)
    f = {"m2m": lib().orc_hh_m2m, "l2l": lib().orc_hh_l2l, "m2l": lib().orc_hh_m2l}[kind]
    f(p_in, p_out, float(k), float(r_in), np.ascontiguousarray(c_in, dtype=np.float64), float(r_out),
      np.ascontiguousarray(c_out, dtype=np.float64), _planes(e), out)
    return _complex(out)


def hh_m2l_dense(p, k, r, offset):
    """The dense M2L table of one offset (fmm-tables/src/helmholtz/dense.rs layout):
    a real (2n, n) matrix whose column j is the local of the unit real multipole e_j."""
    n = (p + 1) ** 2
    t = np.zeros(2 * n * n)
    lib().orc_hh_m2l_dense(p, float(k), float(r), int(offset[0]), int(offset[1]), int(offset[2]), t)
    return t.reshape(n, 2 * n).T  # column-major storage -> (2n, n)


def hh_apply_dense(table, m):
    """A complex multipole through a dense table: (A_r + i A_i)(M_r + i M_i)."""
    n = table.shape[1]
    a = table[:n] + 1j * table[n:]
    return a @ np.asarray(m, dtype=np.complex128)


_DEEPEST = 16  # the tree's finest key level (fmm.c DEEPEST)


def _decode(key):
    lvl = C.c_int()
    idx = np.zeros(3, dtype=np.uint32)
    lib().orc_key_decode(int(key), C.byref(lvl), idx)
    return lvl.value, idx.astype(np.int64)


def helmholtz_fmm(src, q, tgt, k, p, max_keys):
    """A Helmholtz FMM for a real k on the oracle's octree and lists (the Laplace plan's
    tree, U/V/W/X lists and pass order, fmm-plan/src/evaluator.rs:368-440), with the
    expansions of helmholtz_ops.c in absolute units: P2M; M2M and L2L by projection;
    M2L from the dense tables of each level and offset (fmm-tables/src/helmholtz/dense.rs
    layout, built by projection); P2L over X lists; L2P; M2P over W lists; P2P over the
    near lists.  Degree p on every level.  Returns phi (nt,) and grad (nt, 3), complex, the
    sums of q e^{ikr}/r (no 1/(4 pi)), in caller order."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    q = np.asarray(q, dtype=np.complex128)
    T = Tree(src, tgt, _DEEPEST, max_keys)
    L = lib()
    lower, side = np.zeros(3), C.c_double()
    L.orc_tree_domain(T._t, lower, C.byref(side))
    side = side.value
    box6, lw, sd = np.zeros(6), np.zeros(3), C.c_double()
    L.orc_domain(len(src), src, len(tgt), tgt, lw, C.byref(sd), box6)
    nb = len(T.keys)
    index = {int(kk): b for b, kk in enumerate(T.keys)}
    lv = np.zeros(nb, dtype=np.int64)
    ix = np.zeros((nb, 3), dtype=np.int64)
    for b, kk in enumerate(T.keys):
        lv[b], ix[b] = _decode(kk)
    r = side / 2.0 ** (lv + 1)
    centre = lower + (2 * ix + 1) * r[:, None]

    def key(level, idx):
        return int(L.orc_key_from_index(np.ascontiguousarray(idx, dtype=np.uint32), int(level)))

    def leaf_of(x):
        _, fi = _decode(L.orc_point_key(np.ascontiguousarray(x), box6, _DEEPEST))
        for level in range(T.nlevels - 1, -1, -1):
            b = index.get(key(level, fi >> (_DEEPEST - level)))
            if b is not None and T.is_leaf[b]:
                return b
        raise RuntimeError("a point in no leaf")

    s_leaf = np.array([leaf_of(x) for x in src])
    t_leaf = np.array([leaf_of(x) for x in tgt])
    members = lambda arr, b: np.nonzero(arr == b)[0]  # noqa: E731
    boxes = lambda keys: [index[int(kk)] for kk in keys if int(kk) in index]  # noqa: E731
    n = (p + 1) ** 2
    M = np.zeros((nb, n), dtype=np.complex128)
    Lc = np.zeros((nb, n), dtype=np.complex128)
    parent = np.full(nb, -1)
    for b in range(nb):
        if lv[b] > 0:
            parent[b] = index[key(lv[b] - 1, ix[b] >> 1)]
    # upward: P2M at the leaves, M2M level by level
    for b in range(nb):
        if T.is_leaf[b]:
            sb = members(s_leaf, b)
            if len(sb):
                M[b] = hh_p2m(p, k, r[b], centre[b], src[sb], q[sb])
    for level in range(T.nlevels - 1, 0, -1):
        for b in np.nonzero(lv == level)[0]:
            if np.any(M[b]):
                P = parent[b]
                M[P] += hh_translate("m2m", p, p, k, r[b], centre[b], r[P], centre[P], M[b])
    # downward: M2L (dense tables), P2L (X lists), L2L
    tables = {}
    for level in range(2, T.nlevels):
        for b in np.nonzero(lv == level)[0]:
            for s in boxes(T.list(b, 1)):
                if not np.any(M[s]):
                    continue
                off = tuple(int(v) for v in ix[b] - ix[s])
                if (level, off) not in tables:
                    tables[(level, off)] = hh_m2l_dense(p, k, r[b], off)
                Lc[b] += hh_apply_dense(tables[(level, off)], M[s])
            for s in boxes(T.list(b, 3)):
                sb = members(s_leaf, s)
                if len(sb):
                    Lc[b] += hh_p2m(p, k, r[b], centre[b], src[sb], q[sb], singular=True)
    for level in range(1, T.nlevels):
        for b in np.nonzero(lv == level)[0]:
            P = parent[b]
            if np.any(Lc[P]):
                Lc[b] += hh_translate("l2l", p, p, k, r[P], centre[P], r[b], centre[b], Lc[P])
    # leaves: L2P, M2P (W lists), P2P (the near list and the leaf itself)
    phi = np.zeros(len(tgt), dtype=np.complex128)
    grad = np.zeros((len(tgt), 3), dtype=np.complex128)
    for b in range(nb):
        if not T.is_leaf[b]:
            continue
        tb = members(t_leaf, b)
        if not len(tb):
            continue
        x = tgt[tb]
        f, g = hh_eval(p, k, r[b], centre[b], Lc[b], x, singular=False)
        for s in boxes(T.list(b, 2)):
            if np.any(M[s]):
                f2, g2 = hh_eval(p, k, r[s], centre[s], M[s], x, singular=True)
                f, g = f + f2, g + g2
        near = set(boxes(T.list(b, 0))) | {b}
        sb = np.concatenate([members(s_leaf, s) for s in sorted(near)])
        if len(sb):
            f3, g3 = helmholtz_p2p(k, src[sb], q[sb], x)
            f, g = f + f3, g + g3
        phi[tb] = f
        grad[tb] = g
    return phi, grad


def helmholtz_p2p(k, src, q, tgt, gradients=True):
    """The reference's Helmholtz p2p (fmm-ref/src/helmholtz/p2p.rs), e^{ikr}/r without
    1/(4 pi), sources in input order: phi (nt,) complex, grad (nt, 3) complex."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    phi = np.zeros(len(tgt), dtype=np.complex128)
    g = np.zeros((len(tgt), 3), dtype=np.complex128) if gradients else None
    k = complex(k)
    lib().orc_helmholtz_p2p(k.real, k.imag, len(src), src, _cview(q), len(tgt), tgt, phi.view(np.float64),
                            None if g is None else g.view(np.float64).ctypes.data_as(C.c_void_p))
    return phi, g


def helmholtz_direct_sum(k, src, q, tgt, gradients=True):
    """The Helmholtz f64 direct sum (Neumaier per real component), without 1/(4 pi)."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    phi = np.zeros(len(tgt), dtype=np.complex128)
    g = np.zeros((len(tgt), 3), dtype=np.complex128) if gradients else None
    k = complex(k)
    lib().orc_helmholtz_direct_sum(k.real, k.imag, len(src), src, _cview(q), len(tgt), tgt, phi.view(np.float64),
                                   None if g is None else g.view(np.float64).ctypes.data_as(C.c_void_p))
    return phi, g


def helmholtz_near(src, q, tgt, k, max_keys, gradients=True, threads=0):
    """The Helmholtz near field on the restated plan, with 1/(4 pi): q (N,) or (N, m)
    complex; phi (m, Nt) complex, grad (m, Nt, 3) complex, caller order."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    q = np.asarray(q, dtype=np.complex128)
    m = 1 if q.ndim == 1 else q.shape[1]
    q = np.ascontiguousarray(q.reshape(len(src), m))
    phi = np.zeros(m * len(tgt), dtype=np.complex128)
    g = np.zeros(3 * m * len(tgt), dtype=np.complex128) if gradients else None
    k = complex(k)
    lib().orc_helmholtz_near(len(src), src, q.view(np.float64), m, len(tgt), tgt, max_keys, k.real, k.imag,
                             int(gradients), threads, phi.view(np.float64),
                             None if g is None else g.view(np.float64).ctypes.data_as(C.c_void_p))
    return phi.reshape(m, len(tgt)), (None if g is None else g.reshape(m, len(tgt), 3))


def fmm_last_eval_seconds():
    """Seconds of the last fmm() call without its plan and table builds."""
    return lib().orc_fmm_last_eval_seconds()


def fmm(src, q, tgt, p, max_keys, gradients=True, threads=0, kinds=3):
    """The restated host FMM; q is (N,) or (N, m); returns phi (m, Nt), grad (m, Nt, 3)
    in caller order with 1/(4 pi) applied.  kinds: bit 0 near field, bit 1 far field."""
    src = np.ascontiguousarray(src, dtype=np.float64)
    tgt = np.ascontiguousarray(tgt, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    m = 1 if q.ndim == 1 else q.shape[1]
    q = np.ascontiguousarray(q.reshape(len(src), m))
    phi = np.zeros(m * len(tgt))
    g = np.zeros(3 * m * len(tgt)) if gradients else None
    rc = lib().orc_fmm_kinds(len(src), src, q, m, len(tgt), tgt, p, max_keys, int(gradients), threads,
                             kinds, phi, _ptr(g))
    if rc != 0:
        raise RuntimeError(f"oracle fmm failed: {rc}")
    return phi.reshape(m, len(tgt)), (g.reshape(m, len(tgt), 3) if gradients else None)


class Fmm:
    """A built oracle FMM (plan and tables once) for repeated evaluations, as the
    reference's FmmBuilder::build then Fmm::evaluate; evaluate() returns what fmm() does."""

    def __init__(self, src, tgt, p, max_keys, gradients=True, vectors=1, host_path=False):
        """host_path: the reference's host path (lists made once, the batched M2L, the
        AVX-512 P2P of nd-fmm-simd; oracle/hostpath.c) instead of its scalar operators."""
        self.src = np.ascontiguousarray(src, dtype=np.float64)
        self.tgt = np.ascontiguousarray(tgt, dtype=np.float64)
        self.m, self.gradients = vectors, gradients
        self._h = lib().orc_fmm_new(len(self.src), self.src, len(self.tgt), self.tgt, p, max_keys, vectors,
                                    int(gradients))
        if host_path:
            lib().orc_fmm_set_host_path(self._h, 1)

    def evaluate(self, q, threads=0, kinds=3):
        q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).reshape(len(self.src), self.m))
        nt = len(self.tgt)
        phi = np.zeros(self.m * nt)
        g = np.zeros(3 * self.m * nt) if self.gradients else None
        rc = lib().orc_fmm_eval(self._h, q, threads, kinds, phi, _ptr(g))
        if rc != 0:
            raise RuntimeError(f"oracle fmm failed: {rc}")
        return phi.reshape(self.m, nt), (g.reshape(self.m, nt, 3) if self.gradients else None)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_fmm_free(self._h)
            self._h = None


class Tree:
    """The oracle's octree (refine + 2:1 balance) and its brute-force list rule."""

    def __init__(self, src, tgt, max_level, max_keys):
        src = np.ascontiguousarray(src, dtype=np.float64)
        tgt = np.ascontiguousarray(tgt, dtype=np.float64)
        self._t = lib().orc_tree_build(len(src), src, len(tgt), tgt, max_level, max_keys)
        n = lib().orc_tree_nboxes(self._t)
        self.keys = np.zeros(n, dtype=np.uint64)
        self.is_leaf = np.zeros(n, dtype=np.uint8)
        lib().orc_tree_boxes(self._t, self.keys, self.is_leaf)
        self.nlevels = lib().orc_tree_nlevels(self._t)

    def list(self, box, kind):
        out = np.zeros(4096, dtype=np.uint64)
        n = lib().orc_tree_list(self._t, box, kind, out, len(out))
        return out[:n].copy()

    def __del__(self):
        if getattr(self, "_t", None):
            lib().orc_tree_free(self._t)
            self._t = None


def point_sets(kind, n, seed):
    """Seeded inputs via the restated generators (fmm-validate/src/points.rs)."""
    L = lib()
    st = C.c_uint64(seed)
    xyz = np.zeros(3 * n)
    c = np.array([0.5, 0.5, 0.5])
    if kind == "cube":
        f = L.orc_points_cube
        f.argtypes = [C.c_void_p, _sz, _dp, C.c_double, _dp]
        f(C.byref(st), n, c, 0.5, xyz)
    elif kind == "sphere":
        f = L.orc_points_sphere_gauss
        f.argtypes = [C.c_void_p, _sz, _dp, C.c_double, _dp]
        f(C.byref(st), n, np.zeros(3), 1.0, xyz)
    else:
        raise ValueError(kind)
    q = np.zeros(n)
    L.orc_charges.argtypes = [C.c_void_p, _sz, _dp]
    L.orc_charges(C.byref(st), n, q)
    return xyz.reshape(n, 3), q


REFERENCE_BENCH_SEED = 0x00BE9C06


def bench_problem(n, sampled=1000, seed=REFERENCE_BENCH_SEED):
    """The reference's own benchmark problem (fmm-bench/src/measure.rs:34-66, Problem::new):
    from one SplitMix64 stream, N points uniform in [0, 1)^3 (points::cube about (1/2, 1/2,
    1/2) with half-width 1/2, fmm-validate/src/points.rs:28-32), then N charges U[-1, 1)
    (points.rs:138-140), then the sampled targets by a partial Fisher-Yates shuffle
    (measure.rs:49-56).  Returns (points (n, 3), charges (n,), sample (sampled,) int64)."""
    L = lib()
    st = C.c_uint64(seed)
    xyz = np.zeros(3 * n)
    f = L.orc_points_cube
    f.argtypes = [C.c_void_p, _sz, _dp, C.c_double, _dp]
    f(C.byref(st), n, np.array([0.5, 0.5, 0.5]), 0.5, xyz)
    q = np.zeros(n)
    L.orc_charges.argtypes = [C.c_void_p, _sz, _dp]
    L.orc_charges(C.byref(st), n, q)
    sampled = min(sampled, n)
    out = np.zeros(max(sampled, 1), dtype=np.uint32)
    L.orc_sample.argtypes = [C.c_void_p, _sz, _sz, _u32p]
    L.orc_sample(C.byref(st), n, sampled, out)
    return xyz.reshape(n, 3), q, out[:sampled].astype(np.int64)
