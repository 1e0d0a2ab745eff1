"""Shared test setup.

Markers: `gpu` -- needs a CUDA device and the built libowl.so; every other test
runs on the CPU (oracle, emulator, ABI surface, host logic).
"""
import ctypes
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libowl.so")


def _oracle_lib():
    path = os.path.join(ROOT, "oracle", "liboracle.so")
    srcs = [os.path.join(ROOT, "oracle", f) for f in ("words.c", "gmp_loop.c", "ibdwt.c", "owl_oracle.h")]
    if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in srcs):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       capture_output=True)
    lib = ctypes.CDLL(path)
    u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32
    P32, P64, PI = ctypes.POINTER(u32), ctypes.POINTER(u64), ctypes.POINTER(i32)
    sig = {
        "oracle_step": ([u32, u32], u32), "oracle_extra": ([u32, u32, u32], u32),
        "oracle_is_big_word": ([u32, u32, u32], ctypes.c_int), "oracle_bitlen": ([u32, u32, u32], u32),
        "oracle_nwords": ([u32], u32),
        "oracle_compact_bits": ([PI, u32, u32, P32], ctypes.c_int),
        "oracle_expand_bits": ([P32, u32, u32, PI], ctypes.c_int),
        "oracle_buf_residue": ([PI, u32, u32], u64),
        "oracle_next_prime": ([u32], u32), "oracle_is_prime": ([u32], ctypes.c_int),
        "oracle_seeded_prime": ([u64, u32, u32], u32),
        "oracle_gmp_run": ([u32, u32, ctypes.c_int, u32, u32, P64, ctypes.c_char_p], ctypes.c_int),
        "oracle_gmp_square_words": ([u32, P32, u32, ctypes.c_int, P32], ctypes.c_int),
        "oracle_gmp_mul_words": ([u32, P32, P32, ctypes.c_int, P32], ctypes.c_int),
        "oracle_gmp_ms_per_iter": ([u32, u32], ctypes.c_double),
        "oracle_ibdwt_create": ([u32, u32, ctypes.c_int], ctypes.c_void_p),
        "oracle_ibdwt_destroy": ([ctypes.c_void_p], None),
        "oracle_ibdwt_square": ([ctypes.c_void_p, PI, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "oracle_ibdwt_mul": ([ctypes.c_void_p, PI, PI, ctypes.c_int, ctypes.POINTER(ctypes.c_double)],
                             ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


class Oracle:
    """numpy-friendly wrappers over oracle/liboracle.so (test infrastructure)."""

    def __init__(self):
        self.lib = _oracle_lib()

    def nwords(self, E):
        return (E - 1) // 32 + 1

    def gmp_square(self, E, words, n, ll=False):
        import numpy as np
        nw = self.nwords(E)
        a = np.ascontiguousarray(words, dtype=np.uint32)
        out = np.zeros(nw, dtype=np.uint32)
        self.lib.oracle_gmp_square_words(E, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n, 1 if ll else 0,
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        return out

    def gmp_mul(self, E, a, b, mul3=False):
        import numpy as np
        nw = self.nwords(E)
        aa = np.ascontiguousarray(a, dtype=np.uint32)
        bb = np.ascontiguousarray(b, dtype=np.uint32)
        out = np.zeros(nw, dtype=np.uint32)
        P = ctypes.POINTER(ctypes.c_uint32)
        self.lib.oracle_gmp_mul_words(E, aa.ctypes.data_as(P), bb.ctypes.data_as(P), 1 if mul3 else 0,
                                      out.ctypes.data_as(P))
        return out

    def gmp_res64(self, E, start, n, step, ll=False):
        cnt = n // step
        buf = (ctypes.c_uint64 * max(cnt, 1))()
        self.lib.oracle_gmp_run(E, start, 1 if ll else 0, n, step, buf, None)
        return [buf[i] for i in range(cnt)]

    def expand(self, E, N, words):
        import numpy as np
        w = np.ascontiguousarray(words, dtype=np.uint32)
        out = np.zeros(N, dtype=np.int32)
        rc = self.lib.oracle_expand_bits(w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), N, E,
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        assert rc == 0
        return out

    def compact(self, E, N, digits):
        import numpy as np
        d = np.ascontiguousarray(digits, dtype=np.int32)
        out = np.zeros(self.nwords(E), dtype=np.uint32)
        rc = self.lib.oracle_compact_bits(d.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), N, E,
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
        assert rc == 0
        return out


@pytest.fixture(scope="session")
def oracle():
    return Oracle()


def random_words(E, seed):
    """Uniform E-bit value as compact words, splitmix64 stream of `seed`."""
    import numpy as np
    mask = (1 << 64) - 1
    s = seed & mask
    nw = (E - 1) // 32 + 1
    out = np.zeros(nw, dtype=np.uint32)
    for i in range(nw):
        s = (s + 0x9E3779B97F4A7C15) & mask
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        out[i] = (z ^ (z >> 31)) & 0xFFFFFFFF
    if E % 32:
        out[-1] &= (1 << (E % 32)) - 1
    return out


def small_words(E, value):
    import numpy as np
    w = np.zeros((E - 1) // 32 + 1, dtype=np.uint32)
    w[0] = value
    return w


def res64_of(words):
    return int(words[0]) | (int(words[1]) << 32)


def load_golden(name):
    path = os.path.join(GOLDEN, name + ".json")
    if not os.path.exists(path):
        pytest.skip("golden fixture %s not generated yet (tests/golden/gen_golden.py %s)" % (name, name))
    with open(path) as f:
        return json.load(f)


def has_gpu():
    try:
        import gpuowl_b200 as g
        return g.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def owl():
    """The built engine; on a GPU test machine a missing build is an error, not a skip."""
    import gpuowl_b200 as g
    from gpuowl_b200 import build as b
    b.build()
    g.load()
    if g.device_count() == 0:
        pytest.skip("no CUDA device")
    return g
