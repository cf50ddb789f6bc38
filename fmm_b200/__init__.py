"""B200 evaluator for the FMM evaluation passes of tbetcke/fmm (Laplace 1/(4 pi r)).

The Python surface mirrors nd-fmm-exec's builder API (fmm-exec/src/fmm.rs):

    fmm = (FmmBuilder(p=6).gradients().vectors(1).max_points_per_leaf(64)
           .precision("f64").build(sources, targets))
    out = fmm.evaluate(charges)        # Output: potential (m, nt), gradient (m, nt, 3)

Every call goes through the C ABI of include/fmm_b200.h in fmm_b200/libfmm_b200.so;
there is no fallback: if the library or a GPU is missing, build() raises.
"""
import ctypes as C
import os

import numpy as np

__all__ = ["FmmBuilder", "Fmm", "Output", "FmmError", "lib", "Plan", "direct_sum", "helmholtz_direct_sum"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "libfmm_b200.so")
_lib = None

PRECISIONS = {"f64": 0, "mixed": 1}


class FmmError(RuntimeError):
    """A failed call of the C ABI (status code and message)."""

    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


class Settings(C.Structure):
    _fields_ = [("p", C.c_int), ("precision", C.c_int), ("gradients", C.c_int), ("vectors", C.c_int),
                ("max_points_per_leaf", C.c_int), ("max_level", C.c_int), ("device", C.c_int),
                ("vectors_per_pass", C.c_int), ("autotune", C.c_int), ("product_bytes", C.c_int64),
                ("table_cache", C.c_char_p), ("tuning_cache", C.c_char_p)]


class Info(C.Structure):
    _fields_ = [("nlevels", C.c_int), ("nboxes", C.c_int64), ("nleaves", C.c_int64),
                ("nsources", C.c_int64), ("ntargets", C.c_int64), ("near_pairs", C.c_int64),
                ("v_pairs", C.c_int64), ("w_pairs", C.c_int64), ("x_pairs", C.c_int64),
                ("device_bytes", C.c_int64), ("close_pairs", C.c_int64), ("launches", C.c_int64),
                ("vectors_per_pass", C.c_int64), ("p2p_warps", C.c_int64), ("leaf_block", C.c_int64),
                ("product_chunks", C.c_int64), ("p2p_stream_bytes", C.c_int64), ("tables_loaded", C.c_int64),
                ("tuning_loaded", C.c_int64), ("m2l_tile_columns", C.c_int64),
                ("vjp_forward_reused", C.c_int64)]


def lib():
    """Loads libfmm_b200.so (built by fmm_b200.build); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIBPATH):
            raise FmmError(-1, f"{_LIBPATH} is missing: run `python -m fmm_b200.build`")
        L = C.CDLL(_LIBPATH)
        vp, sz, dp = C.c_void_p, C.c_size_t, C.c_void_p
        sig = {
            "fmmgpu_default_settings": (None, [C.POINTER(Settings)]),
            "fmmgpu_fmm_build": (C.c_int, [C.POINTER(Settings), sz, dp, sz, dp, C.POINTER(vp)]),
            "fmmgpu_plan_build": (C.c_int, [C.POINTER(Settings), sz, dp, sz, dp, C.POINTER(vp)]),
            "fmmgpu_batch_build": (C.c_int, [C.POINTER(Settings), sz, dp, dp, dp, dp, C.POINTER(vp)]),
            "fmmgpu_batch_plan_build": (C.c_int, [C.POINTER(Settings), sz, dp, dp, dp, dp, C.POINTER(vp)]),
            "fmmgpu_fmm_evaluate": (C.c_int, [vp, dp, dp, dp]),
            "fmmgpu_fmm_evaluate_f32": (C.c_int, [vp, dp, dp, dp]),
            "fmmgpu_fmm_evaluate_device": (C.c_int, [vp, dp, dp, dp]),
            "fmmgpu_fmm_vjp": (C.c_int, [vp, dp, dp, dp, dp, dp]),
            "fmmgpu_fmm_stream": (vp, [vp]),
            "fmmgpu_fmm_synchronize": (C.c_int, [vp]),
            "fmmgpu_fmm_info": (C.c_int, [vp, C.POINTER(Info)]),
            "fmmgpu_fmm_destroy": (None, [vp]),
            "fmmgpu_fmm_boxes": (C.c_int, [vp, dp, dp]),
            "fmmgpu_fmm_list": (C.c_int64, [vp, C.c_int, C.c_int64, dp, C.c_int64]),
            "fmmgpu_fmm_tables": (C.c_int, [vp, dp, dp, dp]),
            "fmmgpu_fmm_set_kind_timing": (C.c_int, [vp, C.c_int]),
            "fmmgpu_fmm_kind_times": (C.c_int, [vp, dp]),
            "fmmgpu_fmm_set_kinds": (C.c_int, [vp, C.c_int]),
            "fmmgpu_fmm_set_graph": (C.c_int, [vp, C.c_int]),
            "fmmgpu_fmm_set_overlap": (C.c_int, [vp, C.c_int]),
            "fmmgpu_fmm_set_m2l_path": (C.c_int, [vp, C.c_int]),
            "fmmgpu_fmm_set_p2p_path": (C.c_int, [vp, C.c_int]),
            "fmmgpu_fmm_autotune": (C.c_int, [vp, dp, dp]),
            "fmmgpu_fmm_set_launch_shapes": (C.c_int, [vp, C.c_int, C.c_int]),
            "fmmgpu_fmm_set_m2l_tile": (C.c_int, [vp, C.c_int]),
            "fmmgpu_fmm_set_vjp_store": (C.c_int, [vp, C.c_int]),
            "fmmgpu_direct_sum": (C.c_int, [sz, dp, dp, sz, dp, dp, dp, C.c_int]),
            "fmmgpu_direct_sum_noalloc": (C.c_int, [sz, dp, dp, sz, dp, dp, dp, C.c_int, vp]),
            "fmmgpu_helmholtz_direct_sum": (C.c_int, [C.c_double, C.c_double, sz, dp, dp, sz, dp, dp, dp, C.c_int]),
            "fmmgpu_helmholtz_near": (C.c_int, [vp, C.c_double, C.c_double, dp, dp, dp]),
            "fmmgpu_helmholtz_evaluate": (C.c_int, [vp, C.c_double, C.c_double, dp, dp, dp]),
            "fmmgpu_helmholtz_evaluate_f32": (C.c_int, [vp, C.c_double, C.c_double, dp, dp, dp]),
            "fmmgpu_upload_plan": (C.c_int, [C.POINTER(Settings), vp, sz, dp, sz, dp, C.POINTER(vp)]),
            "fmmgpu_plan_from_arrays": (C.c_int, [C.POINTER(Settings), vp, sz, dp, sz, dp, C.POINTER(vp)]),
            "fmmgpu_fmm_plan_arrays": (C.c_int, [vp, vp]),
            "fmmgpu_helmholtz_evaluate_device": (C.c_int, [vp, C.c_double, C.c_double, dp, dp, dp]),
            "fmmgpu_helmholtz_table_seconds": (C.c_double, [vp]),
            "fmmgpu_helmholtz_m2l_tables": (C.c_int, [C.c_int, C.c_double, C.c_double, dp]),
            "fmmgpu_helmholtz_octant_tables": (C.c_int, [C.c_int, C.c_double, C.c_double, dp, dp]),
            "fmmgpu_op_begin_evaluation": (C.c_int, [vp, dp]),
            "fmmgpu_op_p2m": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_m2m": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_l2l": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_m2l": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_p2l": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_l2p": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_m2p": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_p2p": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_host_data": (C.c_int, [vp, C.c_int]),
            "fmmgpu_op_read_output": (C.c_int, [vp, dp, dp]),
            "fmmgpu_status_string": (C.c_char_p, [C.c_int]),
            "fmmgpu_last_error": (C.c_char_p, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise FmmError(status, lib().fmmgpu_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _points(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim != 2 or x.shape[1] != 3:
        raise ValueError("points must have shape (n, 3)")
    return x


def direct_sum(sources, charges, targets, gradients=True, device=0):
    """f64 direct sum on the GPU (Neumaier per target), with 1/(4 pi): phi (nt,), grad (nt, 3)."""
    src = _points(sources)
    tgt = _points(targets)
    q = np.ascontiguousarray(charges, dtype=np.float64).reshape(len(src))
    phi = np.zeros(len(tgt))
    g = np.zeros((len(tgt), 3)) if gradients else None
    _check(lib().fmmgpu_direct_sum(len(src), _ptr(src), _ptr(q), len(tgt), _ptr(tgt), _ptr(phi), _ptr(g), device))
    return phi, g


def helmholtz_m2l_tables(p, k, half_width):
    """The dense Helmholtz M2L tables of one level (real k; fmm-tables/src/helmholtz/dense.rs
    layout): an array (316, 2n, n), offset index order, column j the local of e_j with the
    real plane over the imaginary plane.  Host only."""
    n = (p + 1) ** 2
    t = np.zeros(316 * 2 * n * n)
    _check(lib().fmmgpu_helmholtz_m2l_tables(int(p), float(k), float(half_width), _ptr(t)))
    return t.reshape(316, n, 2 * n).transpose(0, 2, 1)  # column-major storage


def helmholtz_octant_tables(p, k, half_width):
    """The Helmholtz M2M and L2L tables of a parent level (real k): two arrays (8, 2n, n),
    octant o's child at the parent centre + half_width/2 (+-1, +-1, +-1) (x from bit 2)."""
    n = (p + 1) ** 2
    a = np.zeros(8 * 2 * n * n)
    b = np.zeros(8 * 2 * n * n)
    _check(lib().fmmgpu_helmholtz_octant_tables(int(p), float(k), float(half_width), _ptr(a), _ptr(b)))
    return a.reshape(8, n, 2 * n).transpose(0, 2, 1), b.reshape(8, n, 2 * n).transpose(0, 2, 1)


def helmholtz_direct_sum(k, sources, charges, targets, gradients=True, device=0):
    """f64 Helmholtz direct sum on the GPU, e^{ikr}/(4 pi r): phi (nt,) complex, grad (nt, 3) complex."""
    src = _points(sources)
    tgt = _points(targets)
    q = np.ascontiguousarray(charges, dtype=np.complex128).reshape(len(src))
    phi = np.zeros(len(tgt), dtype=np.complex128)
    g = np.zeros((len(tgt), 3), dtype=np.complex128) if gradients else None
    k = complex(k)
    _check(lib().fmmgpu_helmholtz_direct_sum(k.real, k.imag, len(src), _ptr(src), _ptr(q), len(tgt), _ptr(tgt),
                                             _ptr(phi), _ptr(g), device))
    return phi, g


class Output:
    """Potentials (m, nt) and, with gradients, gradients (m, nt, 3), caller order."""

    def __init__(self, potential, gradient):
        self.potential = potential
        self.gradient = gradient


class PlanArrays(C.Structure):
    """fmmgpu_plan_arrays: a plan in the reference's flattened layout (include/fmm_b200.h)."""
    _fields_ = [("nlevels", C.c_int), ("level_start", C.c_void_p), ("keys", C.c_void_p), ("is_leaf", C.c_void_p),
                ("lower", C.c_double * 3), ("side", C.c_double), ("source_offsets", C.c_void_p),
                ("target_offsets", C.c_void_p), ("source_order", C.c_void_p), ("target_order", C.c_void_p),
                ("near_rows", C.c_void_p), ("near", C.c_void_p), ("w_rows", C.c_void_p), ("w", C.c_void_p),
                ("x_rows", C.c_void_p), ("x", C.c_void_p), ("v_rows", C.c_void_p), ("v", C.c_void_p),
                ("v_offsets", C.c_void_p)]

    # name -> (dtype, length key): the arrays of a plan dict
    ARRAYS = {"level_start": np.int64, "keys": np.uint64, "is_leaf": np.uint8, "source_offsets": np.int64,
              "target_offsets": np.int64, "source_order": np.int64, "target_order": np.int64,
              "near_rows": np.int64, "near": np.int32, "w_rows": np.int64, "w": np.int32, "x_rows": np.int64,
              "x": np.int32, "v_rows": np.int64, "v": np.int32, "v_offsets": np.int32}

    @classmethod
    def from_dict(cls, plan):
        """A struct pointing into contiguous copies of the dict's arrays (kept on the struct)."""
        s = cls()
        keep = {}
        for name, dt in cls.ARRAYS.items():
            a = np.ascontiguousarray(plan[name], dtype=dt)
            keep[name] = a
            setattr(s, name, a.ctypes.data if a.size else None)
        s.nlevels = int(plan["nlevels"])
        for k in range(3):
            s.lower[k] = float(plan["lower"][k])
        s.side = float(plan["side"])
        s._keep = keep
        return s

    def to_dict(self, nboxes, nleaves, ns, nt):
        """Copies of the arrays the struct points to."""
        def arr(name, n):
            ptr = getattr(self, name)
            dt = np.dtype(self.ARRAYS[name])
            if not n or not ptr:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), (n,)).copy()
        nl = self.nlevels
        out = {"nlevels": nl, "lower": list(self.lower), "side": self.side}
        out["level_start"] = arr("level_start", nl + 1)
        out["keys"] = arr("keys", nboxes)
        out["is_leaf"] = arr("is_leaf", nboxes)
        for s in ("source", "target"):
            out[f"{s}_offsets"] = arr(f"{s}_offsets", nleaves + 1)
        out["source_order"] = arr("source_order", ns)
        out["target_order"] = arr("target_order", nt)
        for name, nrows in (("near", nleaves), ("w", nleaves), ("x", nboxes), ("v", nboxes)):
            out[f"{name}_rows"] = arr(f"{name}_rows", nrows + 1)
            out[name] = arr(name, int(out[f"{name}_rows"][-1]))
        out["v_offsets"] = arr("v_offsets", int(out["v_rows"][-1]))
        return out


class FmmBuilder:
    """The settings of an FMM, as nd-fmm-exec's FmmBuilder (fmm-exec/src/fmm.rs:1228-1270)."""

    def __init__(self, p=6):
        self._s = Settings()
        lib().fmmgpu_default_settings(C.byref(self._s))
        self._s.p = p

    def gradients(self, on=True):
        self._s.gradients = int(bool(on))
        return self

    def vectors(self, m):
        self._s.vectors = int(m)
        return self

    def max_points_per_leaf(self, n):
        self._s.max_points_per_leaf = int(n)
        return self

    def vectors_per_pass(self, n):
        """Charge vectors per device pass (0: as many as fit); the results do not depend on it."""
        self._s.vectors_per_pass = int(n)
        return self

    def autotune(self, on=True):
        """Time the launch shapes at build and keep the fastest (the results are the same bits)."""
        self._s.autotune = int(bool(on))
        return self

    def product_bytes(self, n):
        """M2L product buffer bytes (0: automatic); smaller buffers run the products in
        chunks of target boxes, with the same results."""
        self._s.product_bytes = int(n)
        return self

    def table_cache(self, directory):
        """Load the operator tables from `directory` (the reference's TableCache files),
        building and storing the missing ones (FmmBuilder::table_cache); None: always build."""
        self._table_cache = None if directory is None else os.fsencode(directory)
        self._s.table_cache = self._table_cache
        return self

    def tuning_cache(self, directory):
        """Keep the autotuner's choices in `directory` and reuse them (FmmBuilder::tuning_cache)."""
        self._tuning_cache = None if directory is None else os.fsencode(directory)
        self._s.tuning_cache = self._tuning_cache
        return self

    def max_level(self, level):
        self._s.max_level = int(level)
        return self

    def precision(self, name):
        if name not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self._s.precision = PRECISIONS[name]
        return self

    def device(self, ordinal):
        self._s.device = int(ordinal)
        return self

    def build(self, sources, targets=None):
        src = _points(sources)
        tgt = src if targets is None else _points(targets)  # the same array: a symmetric FMM
        h = C.c_void_p()
        _check(lib().fmmgpu_fmm_build(C.byref(self._s), len(src), _ptr(src), len(tgt), _ptr(tgt), C.byref(h)))
        return Fmm(h, self._s, len(src), len(tgt))

    def _batch(self, fn, clouds, targets):
        srcs = [_points(c) for c in clouds]
        ns = np.array([len(c) for c in srcs], dtype=np.uint64)
        src = np.ascontiguousarray(np.concatenate(srcs) if srcs else np.zeros((0, 3)))
        if targets is None:
            nt, tgt, ntot = None, None, int(ns.sum())
        else:
            tgts = [_points(c) for c in targets]
            if len(tgts) != len(srcs):
                raise ValueError("one target set per cloud")
            nt = np.array([len(c) for c in tgts], dtype=np.uint64)
            tgt = np.ascontiguousarray(np.concatenate(tgts))
            ntot = int(nt.sum())
        h = C.c_void_p()
        _check(fn(C.byref(self._s), len(srcs), _ptr(ns), _ptr(src), _ptr(nt), _ptr(tgt), C.byref(h)))
        return h, int(ns.sum()), ntot

    def build_batch(self, clouds, targets=None):
        """Many independent clouds as one forest: one launch per pass for the whole batch.
        Charges and outputs are the clouds' arrays concatenated in cloud order."""
        h, ns, nt = self._batch(lib().fmmgpu_batch_build, clouds, targets)
        return Fmm(h, self._s, ns, nt)

    def plan_batch(self, clouds, targets=None):
        """The host half of build_batch (no GPU)."""
        h, ns, nt = self._batch(lib().fmmgpu_batch_plan_build, clouds, targets)
        return Plan(h, self._s, ns, nt)

    def upload(self, plan, sources, targets=None):
        """An FMM on a caller's plan (a dict of the fmmgpu_plan_arrays fields, the reference's
        flattened layout): checked, uploaded, then evaluated like any other (fmmgpu_upload_plan)."""
        src = _points(sources)
        tgt = src if targets is None else _points(targets)
        arrays = PlanArrays.from_dict(plan)
        h = C.c_void_p()
        _check(lib().fmmgpu_upload_plan(C.byref(self._s), C.byref(arrays), len(src), _ptr(src), len(tgt), _ptr(tgt),
                                        C.byref(h)))
        return Fmm(h, self._s, len(src), len(tgt))

    def plan_from(self, plan, sources, targets=None):
        """The host half of upload(): the checks and a plan-only handle; needs no GPU."""
        src = _points(sources)
        tgt = src if targets is None else _points(targets)
        arrays = PlanArrays.from_dict(plan)
        h = C.c_void_p()
        _check(lib().fmmgpu_plan_from_arrays(C.byref(self._s), C.byref(arrays), len(src), _ptr(src), len(tgt),
                                             _ptr(tgt), C.byref(h)))
        return Plan(h, self._s, len(src), len(tgt))

    def plan(self, sources, targets=None):
        """The host half only (tree, lists, tables); needs no GPU."""
        src = _points(sources)
        tgt = src if targets is None else _points(targets)
        h = C.c_void_p()
        _check(lib().fmmgpu_plan_build(C.byref(self._s), len(src), _ptr(src), len(tgt), _ptr(tgt), C.byref(h)))
        return Plan(h, self._s, len(src), len(tgt))


class Plan:
    """A built plan (host half of an FMM): boxes, lists and tables, for inspection."""

    def __init__(self, handle, settings, ns, nt):
        self._h = handle
        # a copy of the settings the handle was built with: the output buffers are sized from
        # it, so a builder changed and reused afterwards must not change them (the handle keeps
        # its own copy, cache directories included, so the copy's pointers are dropped)
        self.settings = Settings.from_buffer_copy(settings)
        self.settings.table_cache = None
        self.settings.tuning_cache = None
        self.nsources = ns
        self.ntargets = nt

    def info(self):
        i = Info()
        _check(lib().fmmgpu_fmm_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in Info._fields_}

    def boxes(self):
        n = self.info()["nboxes"]
        keys = np.zeros(n, dtype=np.uint64)
        leaf = np.zeros(n, dtype=np.uint8)
        _check(lib().fmmgpu_fmm_boxes(self._h, _ptr(keys), _ptr(leaf)))
        return keys, leaf

    def list(self, kind, row):
        """One row of a list (kind 0 near, 1 V, 2 W, 3 X) as box keys."""
        out = np.zeros(64, dtype=np.uint64)  # near rows fit; longer V rows take the second call
        n = lib().fmmgpu_fmm_list(self._h, kind, row, _ptr(out), len(out))
        if n < 0:
            raise IndexError(row)
        if n > len(out):  # the call returns the row's full length: fetch it whole
            out = np.zeros(n, dtype=np.uint64)
            lib().fmmgpu_fmm_list(self._h, kind, row, _ptr(out), len(out))
        return out[:n].copy()

    def plan_arrays(self):
        """The plan in the reference's flattened layout (fmmgpu_fmm_plan_arrays), as a dict of
        copies: what FmmBuilder.upload takes."""
        a = PlanArrays()
        _check(lib().fmmgpu_fmm_plan_arrays(self._h, C.byref(a)))
        info = self.info()
        return a.to_dict(info["nboxes"], info["nleaves"], self.nsources, self.ntargets)

    def tables(self):
        p = self.settings.p
        n = (p + 1) ** 2
        m2l = np.zeros(316 * n * n)
        m2m = np.zeros(8 * n * n)
        l2l = np.zeros(8 * n * n)
        _check(lib().fmmgpu_fmm_tables(self._h, _ptr(m2l), _ptr(m2m), _ptr(l2l)))
        # column-major storage: entry (i, k) at i + k n; return A with A[t] @ x = output
        return (m2l.reshape(316, n, n).transpose(0, 2, 1), m2m.reshape(8, n, n).transpose(0, 2, 1),
                l2l.reshape(8, n, n).transpose(0, 2, 1))

    def close(self):
        if self._h:
            lib().fmmgpu_fmm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Fmm(Plan):
    """A built FMM on one GPU (nd-fmm-exec's Fmm): evaluate charge vectors."""

    def evaluate(self, charges):
        """Fmm::evaluate (fmm.rs:3691): the value type follows the charges', as the reference's
        Fmm<T> does: float32 charges give float32 potentials and gradients (the f64 evaluation
        of the widened charges, rounded), anything else float64."""
        m = self.settings.vectors
        f32 = np.asarray(charges).dtype == np.float32
        dt = np.float32 if f32 else np.float64
        q = np.ascontiguousarray(charges, dtype=dt).reshape(self.nsources, m)
        phi = np.zeros((m, self.ntargets), dtype=dt)
        g = np.zeros((m, self.ntargets, 3), dtype=dt) if self.settings.gradients else None
        call = lib().fmmgpu_fmm_evaluate_f32 if f32 else lib().fmmgpu_fmm_evaluate
        _check(call(self._h, _ptr(q), _ptr(phi), _ptr(g)))
        return Output(phi, g)

    def helmholtz_near(self, k, charges):
        """The Helmholtz near field (P2P of every leaf) of e^{ikr}/(4 pi r) on this FMM's
        plan, complex charges (ns, m): Output with complex potential (m, nt) and gradient."""
        m = self.settings.vectors
        q = np.ascontiguousarray(charges, dtype=np.complex128).reshape(self.nsources, m)
        phi = np.zeros((m, self.ntargets), dtype=np.complex128)
        g = np.zeros((m, self.ntargets, 3), dtype=np.complex128) if self.settings.gradients else None
        k = complex(k)
        _check(lib().fmmgpu_helmholtz_near(self._h, k.real, k.imag, _ptr(q), _ptr(phi), _ptr(g)))
        return Output(phi, g)

    def helmholtz_evaluate(self, k, charges):
        """The whole Helmholtz FMM of e^{ikr}/(4 pi r) for a real k > 0 (near and far field)
        on this FMM's tree and lists, complex charges (ns, m): Output with complex potential
        (m, nt) and gradient (m, nt, 3).  The tables of a new k are built on the first call.
        complex64 charges give complex64 outputs (fmmgpu_helmholtz_evaluate_f32), anything
        else complex128."""
        m = self.settings.vectors
        c64 = np.asarray(charges).dtype == np.complex64
        dt = np.complex64 if c64 else np.complex128
        q = np.ascontiguousarray(charges, dtype=dt).reshape(self.nsources, m)
        phi = np.zeros((m, self.ntargets), dtype=dt)
        g = np.zeros((m, self.ntargets, 3), dtype=dt) if self.settings.gradients else None
        k = complex(k)
        call = lib().fmmgpu_helmholtz_evaluate_f32 if c64 else lib().fmmgpu_helmholtz_evaluate
        _check(call(self._h, k.real, k.imag, _ptr(q), _ptr(phi), _ptr(g)))
        return Output(phi, g)

    def helmholtz_evaluate_device(self, k, charges_ptr, potential_ptr, gradient_ptr=None):
        """The Helmholtz FMM on device buffers (pointers) on the evaluator's stream; no sync."""
        k = complex(k)
        _check(lib().fmmgpu_helmholtz_evaluate_device(self._h, k.real, k.imag, C.c_void_p(charges_ptr),
                                                      C.c_void_p(potential_ptr),
                                                      C.c_void_p(gradient_ptr) if gradient_ptr else None))

    def helmholtz_table_seconds(self):
        return float(lib().fmmgpu_helmholtz_table_seconds(self._h))

    def vjp(self, charges, cotangent):
        """Vector-Jacobian product of the potentials for the cotangent w (shape (m, nt)):
        returns (dcharges (ns, m), dsources (ns, 3), dtargets (nt, 3))."""
        m = self.settings.vectors
        q = np.ascontiguousarray(charges, dtype=np.float64).reshape(self.nsources, m)
        w = np.ascontiguousarray(cotangent, dtype=np.float64).reshape(m, self.ntargets)
        dq = np.zeros((self.nsources, m))
        dxs = np.zeros((self.nsources, 3))
        dxt = np.zeros((self.ntargets, 3))
        _check(lib().fmmgpu_fmm_vjp(self._h, _ptr(q), _ptr(w), _ptr(dq), _ptr(dxs), _ptr(dxt)))
        return dq, dxs, dxt

    def evaluate_levels(self, charges, calls=None):
        """The same evaluation driven by the level calls of the operator ABI, in the
        reference evaluator's schedule (fmm-plan/src/evaluator.rs:368-440): upward
        P2M(l), M2M(l-1) for l = L..0; downward L2L, M2L, P2L for l = 1..L; leaves L2P,
        M2P, P2P for l = 0..L.  `calls`, if given, overrides that list of
        (kind, level) pairs."""
        L = lib()
        m = self.settings.vectors
        nl = self.info()["nlevels"]
        q = np.ascontiguousarray(charges, dtype=np.float64).reshape(self.nsources, m)
        _check(L.fmmgpu_op_begin_evaluation(self._h, _ptr(q)))
        if calls is None:
            calls = []
            for lv in range(nl - 1, -1, -1):
                calls.append(("p2m", lv))
                if lv > 0:
                    calls.append(("m2m", lv - 1))
            for lv in range(1, nl):
                calls += [("l2l", lv), ("m2l", lv), ("p2l", lv)]
            for lv in range(nl):
                calls += [("l2p", lv), ("m2p", lv), ("p2p", lv)]
        for kind, lv in calls:
            _check(getattr(L, "fmmgpu_op_" + kind)(self._h, lv))
        phi = np.zeros((m, self.ntargets))
        g = np.zeros((m, self.ntargets, 3)) if self.settings.gradients else None
        _check(L.fmmgpu_op_read_output(self._h, _ptr(phi), _ptr(g)))
        return Output(phi, g)

    def evaluate_device(self, charges_ptr, potential_ptr, gradient_ptr=None):
        """Device-pointer form (no copies, no sync) on the evaluator's stream."""
        _check(lib().fmmgpu_fmm_evaluate_device(self._h, charges_ptr, potential_ptr, gradient_ptr))

    KINDS = ("load", "p2m", "m2m", "l2l", "m2l", "p2l", "l2p_m2p", "p2p")

    def set_kind_timing(self, on=True):
        _check(lib().fmmgpu_fmm_set_kind_timing(self._h, int(on)))

    def set_overlap(self, on=True):
        """Near field on a second stream beside the far field (default off)."""
        _check(lib().fmmgpu_fmm_set_overlap(self._h, int(on)))

    def set_graph(self, on=True):
        """Replay later evaluations from one captured CUDA graph of the whole sweep."""
        _check(lib().fmmgpu_fmm_set_graph(self._h, int(on)))

    def autotune(self, charges):
        """Times the launch shapes that change no result on this plan and keeps the fastest;
        returns {"p2p_warps": w, "leaf_block": b}.  Drops a captured graph."""
        m = self.settings.vectors
        q = np.ascontiguousarray(charges, dtype=np.float64).reshape(self.nsources, m)
        choice = np.zeros(2, dtype=np.int32)
        _check(lib().fmmgpu_fmm_autotune(self._h, _ptr(q), _ptr(choice)))
        return {"p2p_warps": int(choice[0]), "leaf_block": int(choice[1])}

    def set_launch_shapes(self, p2p_warps, leaf_block):
        """Sets the shapes autotune chooses (e.g. a stored choice): 1, 2 or 4 and 32, 64 or 128."""
        _check(lib().fmmgpu_fmm_set_launch_shapes(self._h, int(p2p_warps), int(leaf_block)))

    def set_vjp_store(self, on):
        """Stores each evaluation's charges and target gradients so that a VJP with the same
        charges skips its forward FMM (on), or recomputes it every time (off, the default)."""
        _check(lib().fmmgpu_fmm_set_vjp_store(self._h, 1 if on else 0))

    def set_m2l_tile(self, tile):
        """The tensor-core M2L tile: 0 its default columns, 1 the tuner's alternative (the
        same floats); info()["m2l_tile_columns"] names the columns in use."""
        _check(lib().fmmgpu_fmm_set_m2l_tile(self._h, int(tile)))

    def set_kinds(self, kinds):
        """Test hook: bit 0 near field, bit 1 far field (3, the default, is the FMM)."""
        _check(lib().fmmgpu_fmm_set_kinds(self._h, int(kinds)))

    def set_m2l_path(self, path):
        """M2L path (mixed, p <= 8): 1 tensor-core products then the reduce (the default),
        2 tensor-core M2L fused with the reduce (the same bits), 0 SIMT products."""
        _check(lib().fmmgpu_fmm_set_m2l_path(self._h, int(path)))

    def set_p2p_path(self, path):
        """Mixed P2P sources (test hook): 1 the near rows' streams mapped at build time (the
        default when built), 0 mapped per flush; the same bits."""
        _check(lib().fmmgpu_fmm_set_p2p_path(self._h, int(path)))

    def kind_times(self):
        """Milliseconds per kind of the last evaluation (after set_kind_timing(True))."""
        ms = np.zeros(8)
        _check(lib().fmmgpu_fmm_kind_times(self._h, _ptr(ms)))
        return dict(zip(self.KINDS, ms.tolist()))

    @property
    def stream(self):
        return lib().fmmgpu_fmm_stream(self._h)

    def synchronize(self):
        _check(lib().fmmgpu_fmm_synchronize(self._h))
