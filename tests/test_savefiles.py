"""Savefile formats of the host drivers (include/owl_host.h) against the reference's own Saver
(src/Saver.cpp, compiled into oracle/_ref): each side reads what the other writes, bit for bit."""
import ctypes
import os
import zlib

import numpy as np
import pytest

from conftest import ROOT, random_words

REF = os.path.join(ROOT, "oracle", "_ref", "libref_state.so")


@pytest.fixture(scope="module")
def owl():
    from gpuowl_b200 import build
    build.build()
    import gpuowl_b200 as g
    g.load()
    return g


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref not built (make -C oracle ref)")
    lib = ctypes.CDLL(REF)
    u32, u64, P32, P64 = ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64)
    lib.ref_prp_save.argtypes = [ctypes.c_char_p, u32, u32, u32, u64, P32, u32, ctypes.c_double]
    lib.ref_prp_load.argtypes = [ctypes.c_char_p, u32, u32, P32, P32, P64, P32, P32]
    lib.ref_ll_save.argtypes = [ctypes.c_char_p, u32, u32, P32]
    lib.ref_ll_load.argtypes = [ctypes.c_char_p, u32, P32, P32]
    lib.ref_crc32.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    lib.ref_crc32.restype = u32
    return lib


E = 4989349


def test_crc32_matches_reference_and_zlib(owl, ref):
    for n in (0, 1, 7, 4096, 100003):
        b = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
        assert owl.crc32(b) == ref.ref_crc32(b, len(b)) == zlib.crc32(b)


def test_prp_savefile_ours_read_by_reference(owl, ref, tmp_path):
    check = random_words(E, 5)
    owl.prp_save(str(tmp_path), E, 123000, 1000, 0x0123456789abcdef, check, n_errors=2, elapsed=12.5)
    k, b, ne = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    r = ctypes.c_uint64()
    got = np.zeros(len(check), dtype=np.uint32)
    assert ref.ref_prp_load(str(tmp_path).encode(), E, 1000, ctypes.byref(k), ctypes.byref(b), ctypes.byref(r),
                            got.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), ctypes.byref(ne)) == 0
    assert (k.value, b.value, r.value, ne.value) == (123000, 1000, 0x0123456789abcdef, 2)
    assert np.array_equal(got, check)
    # same bytes as the reference writes for the same state
    ours = open(tmp_path / str(E) / ("%d-%09d.prp" % (E, 123000)), "rb").read()
    d2 = tmp_path / "ref"
    d2.mkdir()
    assert ref.ref_prp_save(str(d2).encode(), E, 123000, 1000, 0x0123456789abcdef,
                            check.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), 2, 12.5) == 0
    theirs = open(d2 / str(E) / ("%d-%09d.prp" % (E, 123000)), "rb").read()
    assert ours == theirs


def test_prp_savefile_reference_read_by_ours(owl, ref, tmp_path):
    check = random_words(E, 6)
    assert ref.ref_prp_save(str(tmp_path).encode(), E, 7000, 500, 0xfeedfacecafebeef,
                            check.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), 0, 3.0) == 0
    st = owl.prp_load(str(tmp_path), E)
    assert (st["k"], st["block"], st["res64"], st["n_errors"]) == (7000, 500, 0xfeedfacecafebeef, 0)
    assert np.array_equal(st["check"], check)


def test_ll_savefile_both_ways(owl, ref, tmp_path):
    data = random_words(E, 7)
    owl.ll_save(str(tmp_path), E, 30000, data)
    k = ctypes.c_uint32()
    got = np.zeros(len(data), dtype=np.uint32)
    assert ref.ref_ll_load(str(tmp_path).encode(), E, ctypes.byref(k),
                           got.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))) == 0
    assert k.value == 30000 and np.array_equal(got, data)
    d2 = tmp_path / "r"
    d2.mkdir()
    assert ref.ref_ll_save(str(d2).encode(), E, 40000, data.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))) == 0
    st = owl.ll_load(str(d2), E)
    assert st["k"] == 40000 and np.array_equal(st["data"], data)


def test_bad_crc_falls_back_to_previous_savefile(owl, tmp_path):
    a, b = random_words(E, 1), random_words(E, 2)
    owl.prp_save(str(tmp_path), E, 1000, 1000, 11, a)
    owl.prp_save(str(tmp_path), E, 2000, 1000, 22, b)
    newest = tmp_path / str(E) / ("%d-%09d.prp" % (E, 2000))
    raw = bytearray(open(newest, "rb").read())
    raw[-5] ^= 0x40                      # corrupt one data byte: CRC mismatch
    open(newest, "wb").write(bytes(raw))
    st = owl.prp_load(str(tmp_path), E)
    assert st["k"] == 1000 and st["res64"] == 11 and np.array_equal(st["check"], a)
    assert os.path.exists(str(newest) + ".bad")


def test_retention_keeps_n_savefiles(owl, tmp_path):
    w = random_words(E, 3)
    for k in range(1000, 11000, 1000):
        owl.prp_save(str(tmp_path), E, k, 1000, k, w)
    files = sorted(os.listdir(tmp_path / str(E)))
    assert len(files) == 4
    assert files[-1] == "%d-%09d.prp" % (E, 10000)
