"""PRP proofs exchanged with the reference's own proof code (src/Proof.cpp with src/sha3.cpp and
src/md5.cpp, compiled from its sources into oracle/_ref/libref_proof.so; its Gpu is replaced by the
GMP oracle, oracle/ref_stub/Gpu.h).

CPU: the proof points and the residue hash agree with the reference's, and the reference's
computeProof / verify pair accepts its own proof built from GMP residues (the stand-in works).
GPU: a proof that owl_prp_run writes verifies with the reference's Proof::verify; the reference's
ProofSet::computeProof, run on the residue files owl_prp_run saved, writes the same proof file byte
for byte; a proof the reference computes from GMP residues passes owl_proof_verify.
"""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_proof.so")
P32 = ctypes.POINTER(ctypes.c_uint32)


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref not built (make -C oracle ref, needs the reference sources)")
    lib = ctypes.CDLL(REF)
    lib.ref_proof_verify.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    lib.ref_proof_verify.restype = ctypes.c_int
    lib.ref_proof_hash_words.argtypes = [ctypes.c_uint32, P32, ctypes.POINTER(ctypes.c_uint64)]
    lib.ref_proof_hash_words.restype = None
    lib.ref_proofset_save.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, P32]
    lib.ref_proofset_save.restype = ctypes.c_int
    lib.ref_proof_compute_and_save.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32,
                                               ctypes.c_char_p, ctypes.c_size_t]
    lib.ref_proof_compute_and_save.restype = ctypes.c_int
    lib.ref_proof_points.argtypes = [ctypes.c_uint32, ctypes.c_uint32, P32, ctypes.c_uint32]
    lib.ref_proof_points.restype = ctypes.c_int
    return lib


@pytest.fixture(scope="module")
def owlcpu():
    import gpuowl_b200 as g
    from gpuowl_b200 import build as b
    b.build()
    g.load()
    return g


def ref_verify(ref, path):
    prime = ctypes.c_int(-1)
    rc = ref.ref_proof_verify(str(path).encode(), ctypes.byref(prime))
    return rc, bool(prime.value)


def ref_compute(ref, d, E, power):
    out = ctypes.create_string_buffer(4096)
    assert ref.ref_proof_compute_and_save(str(d).encode(), E, power, out, 4096) == 0
    return out.value.decode()


def gmp_residues(oracle, ref, d, E, power):
    """3^(2^k) mod 2^E - 1 at every proof point k, saved with the reference's ProofSet::save."""
    pts = (ctypes.c_uint32 * (1 << power))()
    n = ref.ref_proof_points(E, power, pts, 1 << power)
    assert n == 1 << power
    x = np.zeros((E - 1) // 32 + 1, dtype=np.uint32)
    x[0] = 3
    k = 0
    for p in list(pts)[:n]:
        x = oracle.gmp_square(E, x, p - k)
        k = p
        assert ref.ref_proofset_save(str(d).encode(), E, power, p, x.ctypes.data_as(P32)) == 0
    return x


@pytest.mark.parametrize("E,power", [(86243, 3), (216091, 5), (3021377, 8)])
def test_proof_points_match_reference(owlcpu, ref, E, power):
    pts = (ctypes.c_uint32 * (1 << power))()
    n = ref.ref_proof_points(E, power, pts, 1 << power)
    assert owlcpu.proof_points(E, power) == list(pts)[:n]


@pytest.mark.parametrize("E", [86243, 216091])
def test_residue_hash_matches_reference(owlcpu, ref, E):
    from conftest import random_words
    w = random_words(E, E)
    h = (ctypes.c_uint64 * 4)()
    ref.ref_proof_hash_words(E, w.ctypes.data_as(P32), h)
    nb = (E - 1) // 8 + 1
    assert owlcpu.sha3_256(w.tobytes()[:nb]) == b"".join(int(x).to_bytes(8, "little") for x in h)


@pytest.mark.parametrize("E,prime", [(86243, True), (86249, False)])
def test_reference_proof_of_gmp_residues_verifies_in_reference(oracle, ref, tmp_path, E, prime):
    gmp_residues(oracle, ref, tmp_path, E, 3)
    path = ref_compute(ref, tmp_path, E, 3)
    assert ref_verify(ref, path) == (1, prime)


@pytest.mark.gpu
@pytest.mark.parametrize("E,prime", [(86243, True), (86249, False)])
def test_proofs_exchange_with_reference(owl, ref, tmp_path, E, prime):
    r = owl.prp_run(E, W=64, H=64, block=500, save_dir=str(tmp_path), proof_power=3)
    assert r["finished"] and r["is_prime"] == prime and r["proof_power"] == 3
    ours = open(r["proof_file"], "rb").read()
    # ours, through the reference's Proof::load + Proof::verify
    assert ref_verify(ref, r["proof_file"]) == (1, prime)
    # the reference's computeProof on the residue files our PRP loop saved: the same file
    theirs_path = ref_compute(ref, tmp_path, E, 3)
    assert open(theirs_path, "rb").read() == ours


@pytest.mark.gpu
@pytest.mark.parametrize("E,prime", [(86243, True), (86249, False)])
def test_reference_proof_verifies_here(owl, oracle, ref, tmp_path, E, prime):
    gmp_residues(oracle, ref, tmp_path, E, 4)
    path = ref_compute(ref, tmp_path, E, 4)
    assert owl.proof_verify(path) == (True, prime)
    # a flipped bit in the last middle residue is rejected by both
    data = bytearray(open(path, "rb").read())
    data[-100] ^= 0x04
    bad = tmp_path / "bad.proof"
    bad.write_bytes(bytes(data))
    assert owl.proof_verify(str(bad))[0] is False
    assert ref_verify(ref, bad)[0] == 0
