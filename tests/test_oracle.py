"""The oracle itself, on the CPU: pinned against the reference's own host code (oracle/_ref, built
from the reference's src/state.cpp, src/Primes.cpp, src/common.cpp) and against GMP known answers."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, random_words, res64_of, small_words

REF = os.path.join(ROOT, "oracle", "_ref", "libref_state.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref not built (make -C oracle ref, needs the reference sources)")
    lib = ctypes.CDLL(REF)
    u32, P32, PI = ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_int32)
    lib.ref_compact_bits.argtypes = [PI, u32, u32, P32]
    lib.ref_compact_bits.restype = ctypes.c_int
    lib.ref_expand_bits.argtypes = [P32, u32, u32, PI]
    lib.ref_bitlen.argtypes = [u32, u32, u32]
    lib.ref_bitlen.restype = u32
    lib.ref_extra.argtypes = [u32, u32, u32]
    lib.ref_extra.restype = u32
    lib.ref_next_prime.argtypes = [u32]
    lib.ref_next_prime.restype = u32
    return lib


CASES = [(86243, 8192), (216091, 16384), (4989349, 262144), (1257787, 65536), (136181029, 1 << 23)]


@pytest.mark.parametrize("E,N", CASES)
def test_word_model_matches_reference(oracle, ref, E, N):
    rng = np.random.default_rng(E)
    for k in list(range(64)) + list(rng.integers(0, N, 200)):
        k = int(k)
        assert oracle.lib.oracle_bitlen(N, E, k) == ref.ref_bitlen(N, E, k)
        assert oracle.lib.oracle_extra(N, E, k) == ref.ref_extra(N, E, k)


@pytest.mark.parametrize("E,N", CASES[:4])
def test_expand_compact_match_reference(oracle, ref, E, N):
    P32, PI = ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_int32)
    for seed in (1, 2, 3):
        w = random_words(E, seed)
        d_ref = np.zeros(N, dtype=np.int32)
        ref.ref_expand_bits(w.ctypes.data_as(P32), N, E, d_ref.ctypes.data_as(PI))
        d = oracle.expand(E, N, w)
        assert np.array_equal(d, d_ref)
        out_ref = np.zeros(oracle.nwords(E), dtype=np.uint32)
        n = ref.ref_compact_bits(d_ref.ctypes.data_as(PI), N, E, out_ref.ctypes.data_as(P32))
        assert n == oracle.nwords(E)
        assert np.array_equal(oracle.compact(E, N, d), out_ref)
        assert np.array_equal(out_ref, w)
    # sloppy digits (one word outside the balanced range, as carries leave them) compact the same way
    d = oracle.expand(E, N, random_words(E, 9))
    d[5] += 1 << (oracle.lib.oracle_bitlen(N, E, 5) - 1)
    d[4] -= 1
    out_ref = np.zeros(oracle.nwords(E), dtype=np.uint32)
    ref.ref_compact_bits(d.ctypes.data_as(PI), N, E, out_ref.ctypes.data_as(P32))
    assert np.array_equal(oracle.compact(E, N, d), out_ref)


def test_next_prime_and_seeded_exponents_match_reference(oracle, ref):
    for n in (4_800_000, 136_000_000, 330_000_000, 1_000_003, 19_999_999, 86242):
        assert oracle.lib.oracle_next_prime(n) == ref.ref_next_prime(n)
    # the exponents of the workloads: splitmix64(seed + cfg) into the range, then nextPrime
    import sys
    sys.path.insert(0, GOLDEN)
    import gen_golden
    for name, w in gen_golden.WORKLOADS.items():
        E = gen_golden.seeded_prime(w["cfg"], w["lo"], w["hi"])
        assert w["lo"] <= E and oracle.lib.oracle_is_prime(E)
    assert gen_golden.seeded_prime(2, 136_000_000, 139_000_000) == 136181029


@pytest.mark.parametrize("E,N", CASES[:3])
def test_buf_residue_matches_compact(oracle, E, N):
    """bufResidue's wrap-window rule (src/Gpu.cpp:955-975) gives the low 64 bits of compactBits."""
    for seed in range(5):
        d = oracle.expand(E, N, random_words(E, 100 + seed))
        win = np.array([d[(N - 32 + i) % N] for i in range(64)], dtype=np.int32)
        r = oracle.lib.oracle_buf_residue(win.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), N, E)
        assert r == res64_of(oracle.compact(E, N, d))


@pytest.mark.parametrize("E,ll,want", [(521, True, 0), (607, False, 9), (1279, True, 0), (2203, False, 9)])
def test_gmp_known_mersenne_primes(oracle, E, ll, want):
    n = E - 2 if ll else E
    w = oracle.gmp_square(E, small_words(E, 4 if ll else 3), n, ll=ll)
    assert int(w[0]) == want and not w[1:].any()


def test_gmp_composite_is_not_9(oracle):
    E = 523  # M523 is composite
    w = oracle.gmp_square(E, small_words(E, 3), E)
    assert not (int(w[0]) == 9 and not w[1:].any())


@pytest.mark.parametrize("E,N,mul3,ll", [(216091, 16384, 0, 0), (110503, 8192, 1, 0), (86243, 8192, 0, 1)])
def test_ibdwt_restatement_matches_gmp(oracle, E, N, mul3, ll):
    lib = oracle.lib
    p = lib.oracle_ibdwt_create(E, N, 2)
    try:
        w = random_words(E, 7)
        d = oracle.expand(E, N, w)
        roe = ctypes.c_double()
        PI = ctypes.POINTER(ctypes.c_int32)
        for i in range(6):
            assert lib.oracle_ibdwt_square(p, d.ctypes.data_as(PI), mul3 if i == 5 else 0, ll,
                                           ctypes.byref(roe)) == 0
        want = oracle.gmp_square(E, w, 6, ll=bool(ll))
        if mul3:
            want = oracle.gmp_mul(E, want, small_words(E, 3))
        assert np.array_equal(oracle.compact(E, N, d), want)
        assert roe.value < 0.1
    finally:
        lib.oracle_ibdwt_destroy(p)


def test_golden_fixtures_are_well_formed():
    for name in ("prp_256k", "small", "prp_8m", "ll_8m", "prp_20m"):
        path = os.path.join(GOLDEN, name + ".json")
        if not os.path.exists(path):
            continue
        g = json.load(open(path))
        items = g.get("items", [g])
        for it in items:
            assert it["iters"] // it["step"] == len(it["res64"])
            assert all(len(r) == 16 for r in it["res64"])


def test_golden_256k_prefix_recomputes(oracle):
    """The first checkpoint of the stored 256K table recomputes with GMP (cheap spot check)."""
    path = os.path.join(GOLDEN, "prp_256k.json")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    g = json.load(open(path))
    r = oracle.gmp_res64(g["E"], 3, g["step"], g["step"])
    assert "%016x" % r[0] == g["res64"][0]
