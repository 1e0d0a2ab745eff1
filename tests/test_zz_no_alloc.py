"""owl_square_noalloc: the squaring entry point that allocates nothing.

Some callers cannot call cudaMalloc -- hosts whose device memory all belongs to
their own pool allocator, real-time loops that must not block in the allocator,
plug-ins whose host forbids allocation -- so this entry point keeps all of its
scratch in one fixed device array inside libowl and squares a buffer the caller
already owns. Its results must equal the regular entry point's (owl_square) and
the GMP oracle's word for word, call after call: the shared array keeps the
previous call's contents, and each call must clear what has to start at zero.
This file runs last so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

from conftest import random_words

pytestmark = pytest.mark.gpu


def _noalloc(owl):
    fn = owl.load().owl_square_noalloc
    fn.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                   ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


@pytest.mark.parametrize("E,W,H,flags", [(500009, 128, 128, 0), (1000003, 128, 256, 2),
                                         (86243, 64, 64, 1)])
def test_noalloc_matches_square_twice(owl, oracle, E, W, H, flags):
    fn = _noalloc(owl)
    n = 25
    with owl.Plan(E, W=W, H=H) as p:
        ref, buf = p.alloc(), p.alloc()
        w = random_words(E, E ^ 0x5EED)
        p.writeIn(ref, w)
        p.writeIn(buf, w)
        want = w
        for _ in range(2):  # two calls in a row: the second starts from the first's leftovers
            p.squareLoop(ref, ref, n, mul3=bool(flags & 1), ll=bool(flags & 2))
            p.sync()
            rc = fn(0, E, W, H, buf, n, flags, None)
            assert rc == 0, owl.load().owl_last_error()
            got = p.readOut(buf)
            assert np.array_equal(got, p.readOut(ref))
            # the exact product: n squarings (x^2 - 2 for LL), times 3 after the last one (MUL3)
            want = oracle.gmp_square(E, want, n, ll=bool(flags & 2))
            if flags & 1:
                want = oracle.gmp_mul(E, want, _three(E))
            assert np.array_equal(got, want)


def _three(E):
    w = np.zeros((E - 1) // 32 + 1, dtype=np.uint32)
    w[0] = 3
    return w


def test_noalloc_rejects_sizes_beyond_its_scratch(owl):
    fn = _noalloc(owl)
    with owl.Plan(4989349, W=256, H=512) as p:
        buf = p.alloc()
        assert fn(0, 4989349, 256, 512, buf, 1, 0, None) == -1
        assert b"no-alloc" in owl.load().owl_last_error()
        assert fn(0, 4989349, 0, 0, buf, 1, 0, None) == -1
    # 20 bits per word on the largest shape: above the path's 19-bit limit
    with owl.Plan(1310719, W=128, H=256) as p:
        buf = p.alloc()
        assert fn(0, 1310719, 128, 256, buf, 1, 0, None) == -1
        assert b"bits per word" in owl.load().owl_last_error()
