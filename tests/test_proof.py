"""PRP proofs (reference src/Proof.cpp, src/Proof.h): SHA3-256, the proof points, A^h * B on the
engine, generation inside the PRP loop and verification.

CPU tests: the hash against Python's hashlib and the point set against a restatement of
ProofSet's construction. GPU tests: expMul against Python integers, proofs of a Mersenne prime and
of a composite, a corrupted proof, and a proof continued after a stop.
"""
import hashlib
import os
import random

import numpy as np
import pytest

from conftest import random_words


@pytest.fixture(scope="module")
def owlcpu():
    """The library for host-only calls (no device needed)."""
    import gpuowl_b200 as g
    from gpuowl_b200 import build as b
    b.build()
    g.load()
    return g


def _points(E, power):
    pts = [0]
    span = (E + 1) // 2
    for _ in range(power):
        pts += [p + span for p in pts]
        span = (span + 1) // 2
    pts[0] = E
    return sorted(pts)


def test_sha3_256_matches_hashlib(owlcpu):
    owl = owlcpu
    rng = random.Random(5)
    for n in [0, 1, 31, 32, 135, 136, 137, 271, 272, 273, 4096, 86243 // 8 + 1]:
        data = bytes(rng.getrandbits(8) for _ in range(n))
        assert owl.sha3_256(data) == hashlib.sha3_256(data).digest(), n


@pytest.mark.parametrize("E,power", [(86243, 1), (86243, 5), (216091, 8), (332999993, 8), (136181029, 10)])
def test_proof_points(owlcpu, E, power):
    owl = owlcpu
    pts = owl.proof_points(E, power)
    assert pts == _points(E, power)
    assert len(pts) == 1 << power and pts[-1] == E and pts == sorted(set(pts))


def _int(words):
    return int.from_bytes(np.asarray(words, dtype=np.uint32).tobytes(), "little")


def _words(x, E):
    nw = (E - 1) // 32 + 1
    return np.frombuffer(x.to_bytes(4 * nw, "little"), dtype=np.uint32).copy()


@pytest.mark.gpu
@pytest.mark.parametrize("h", [0, 1, 2, 3, 0xFFFFFFFFFFFFFFFF, 0x9E3779B97F4A7C15])
def test_exp_mul_vs_python(owl, h):
    E = 86243
    M = (1 << E) - 1
    a, b = random_words(E, 41), random_words(E, 42)
    with owl.Plan(E, W=64, H=64) as p:
        ba, bb = p.alloc(), p.alloc()
        p.writeIn(ba, a)
        p.writeIn(bb, b)
        p.expMul(ba, h, bb)
        got = _int(p.readOut(ba)) % M
    assert got == pow(_int(a), h, M) * _int(b) % M


def _proof_bytes(path):
    with open(path, "rb") as f:
        return f.read()


@pytest.mark.gpu
@pytest.mark.parametrize("E,prime", [(86243, True), (86249, False)])
def test_prp_proof_generated_and_verified(owl, tmp_path, E, prime):
    r = owl.prp_run(E, W=64, H=64, block=500, save_dir=str(tmp_path), proof_power=5)
    assert r["finished"] and r["is_prime"] == prime and r["n_errors"] == 0
    assert r["proof_power"] == 5 and r["proof_file"].endswith("%d-5.proof" % E)
    data = _proof_bytes(r["proof_file"])
    header = b"PRP PROOF\nVERSION=2\nHASHSIZE=64\nPOWER=5\nNUMBER=M%d\n" % E
    nb = (E - 1) // 8 + 1
    assert data.startswith(header) and len(data) == len(header) + 6 * nb
    assert (data[len(header):len(header) + nb] == (9).to_bytes(nb, "little")) == prime
    assert owl.proof_verify(r["proof_file"]) == (True, prime)
    # one flipped bit in a middle residue must fail verification
    bad = bytearray(data)
    bad[len(header) + 2 * nb + 100] ^= 0x10
    bad_path = tmp_path / "bad.proof"
    bad_path.write_bytes(bytes(bad))
    assert owl.proof_verify(str(bad_path))[0] is False


@pytest.mark.gpu
def test_prp_proof_after_stop_and_resume(owl, tmp_path):
    """Stop in the middle, resume from the savefile: the residues saved before the stop are reused."""
    E = 86243
    r1 = owl.prp_run(E, W=64, H=64, block=500, save_dir=str(tmp_path), proof_power=4, stop_after=40000)
    assert not r1["finished"] and r1["k"] >= 40000
    saved = sorted(int(f) for f in os.listdir(tmp_path / str(E) / "proof") if f.isdigit())
    assert saved and all(k <= r1["k"] for k in saved)
    r2 = owl.prp_run(E, W=64, H=64, block=500, save_dir=str(tmp_path), proof_power=4)
    assert r2["finished"] and r2["is_prime"] and r2["proof_power"] == 4
    assert owl.proof_verify(r2["proof_file"]) == (True, True)


@pytest.mark.gpu
def test_prp_of_m3021377_proves_prime_with_power_8(owl, tmp_path):
    """A full PRP test of the Mersenne prime M3021377 (3.02 M iterations at the 256K FFT, Gerbicz
    every 1,000) through the C++ driver, with a power-8 proof that then verifies."""
    E = 3021377
    r = owl.prp_run(E, save_dir=str(tmp_path), proof_power=8)
    assert r["finished"] and r["is_prime"] and r["n_errors"] == 0
    assert r["res64"] == 1                      # type-1 residue 3^(2^E) / 9 of a prime
    assert r["proof_power"] == 8
    assert owl.proof_verify(r["proof_file"]) == (True, True)
