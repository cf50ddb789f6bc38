"""The on-disk table cache in the reference's TableCache format (fmm-tables/src/cache.rs:
a 44-byte little-endian header -- magic NDFMMTAB, format version 1, convention version 4,
kind code (1 M2M, 2 L2L, 3 M2L), p, bits per value, payload length, FNV-1a 64 checksum --
then the matrices column-major; files named <kind>-p<pp>-f64-c4-v1.bin).  Plan-only
builds, no GPU needed."""
import os
import struct

import numpy as np

import fmm_b200 as F

FNV_OFFSET, FNV_PRIME = 0xCBF29CE484222325, 0x100000001B3


def fnv1a(data):
    h = FNV_OFFSET
    for b in data:
        h = ((h ^ b) * FNV_PRIME) & 0xFFFFFFFFFFFFFFFF
    return h


def points():
    return np.random.default_rng(3).uniform(size=(3000, 3))


def storage(tables):
    """The column-major storage of tables() (which returns A with A[t] @ x = output)."""
    return np.ascontiguousarray(tables.transpose(0, 2, 1)).ravel()


def reference_file(kind_code, p, values):
    """A cache file as the reference's TableCache::store writes it."""
    payload = np.ascontiguousarray(values, dtype="<f8").tobytes()
    head = b"NDFMMTAB" + struct.pack("<IIIII", 1, 4, kind_code, p, 64) + struct.pack("<QQ", len(payload), fnv1a(payload))
    assert len(head) == 44
    return head + payload


def test_store_then_load_in_the_reference_format(tmp_path):
    d = str(tmp_path)
    a = F.FmmBuilder(3).max_points_per_leaf(32).table_cache(d).plan(points())
    assert a.info()["tables_loaded"] == 0
    names = sorted(os.listdir(d))
    assert names == ["l2l-p03-f64-c4-v1.bin", "m2l-p03-f64-c4-v1.bin", "m2m-p03-f64-c4-v1.bin"]
    m2l, m2m, l2l = a.tables()
    for name, code, t in (("m2l", 3, m2l), ("m2m", 1, m2m), ("l2l", 2, l2l)):
        raw = open(os.path.join(d, f"{name}-p03-f64-c4-v1.bin"), "rb").read()
        assert raw == reference_file(code, 3, storage(t))  # byte for byte the reference's layout
    b = F.FmmBuilder(3).max_points_per_leaf(32).table_cache(d).plan(points())
    assert b.info()["tables_loaded"] == 7
    for x, y in zip(a.tables(), b.tables()):
        assert np.array_equal(x, y)


def test_a_file_written_in_the_reference_format_is_read(tmp_path):
    """Values that only the file holds (the true M2M tables times 2, exact) reach the plan."""
    d = str(tmp_path)
    base = F.FmmBuilder(3).max_points_per_leaf(32).plan(points())
    _, m2m, _ = base.tables()
    with open(os.path.join(d, "m2m-p03-f64-c4-v1.bin"), "wb") as f:
        f.write(reference_file(1, 3, 2.0 * storage(m2m)))
    c = F.FmmBuilder(3).max_points_per_leaf(32).table_cache(d).plan(points())
    assert c.info()["tables_loaded"] == 2
    assert np.array_equal(c.tables()[1], 2.0 * m2m)


def test_rejected_files_are_rebuilt_and_replaced(tmp_path):
    d = str(tmp_path)
    F.FmmBuilder(3).max_points_per_leaf(32).table_cache(d).plan(points())
    path = os.path.join(d, "m2l-p03-f64-c4-v1.bin")
    good = open(path, "rb").read()
    bad = [
        good[:40],                                              # shorter than the header
        b"XDFMMTAB" + good[8:],                                 # magic
        good[:12] + struct.pack("<I", 3) + good[16:],           # convention version
        good[:20] + struct.pack("<I", 4) + good[24:],           # key: another p
        good[:-8],                                              # payload length
        good[:-1] + bytes([good[-1] ^ 1]),                      # checksum
    ]
    for b in bad:
        with open(path, "wb") as f:
            f.write(b)
        e = F.FmmBuilder(3).max_points_per_leaf(32).table_cache(d).plan(points())
        assert e.info()["tables_loaded"] == 6  # M2L rebuilt, M2M and L2L loaded
        assert open(path, "rb").read() == good  # the rebuilt table stored over the rejected file
    assert not [n for n in os.listdir(d) if n.endswith(".tmp")]
