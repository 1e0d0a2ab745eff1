"""The large configuration: PRP-3 at the 20M FFT (N = 5 * 2^22 = 4096 x 2560, a radix-5 stage in the
column FFT), E the seeded prime in [330M, 335M], Gerbicz every 1,000 iterations, proof power 8 enabled,
res64 at every 1,000 iterations against the GMP golden table; then the first proof residue point of
power 8 (at about E / 2, far beyond the golden table) is reached from a savefile moved to just below
it, and the residue saved there is read back by the reference's own ProofSet::load.
"""
import ctypes
import os

import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_prp_20m_golden_with_proof_power_8(owl, tmp_path):
    g = load_golden("prp_20m")
    if g is None:
        pytest.skip("golden table not generated")
    E = g["E"]
    assert owl.fft_choose(E) == (5 << 22, 4096, 2560)
    r = owl.prp_run(E, W=4096, H=2560, block=1000, log_step=1000, stop_after=g["iters"], save_dir=str(tmp_path),
                    proof_power=8)
    assert r["n_errors"] == 0 and not r["finished"] and r["k"] == g["iters"]
    got = ["%016x" % res for (k, res) in r["checkpoints"] if k % g["step"] == 0]
    assert got == g["res64"]
    pts = owl.proof_points(E, 8)
    assert pts[0] > g["iters"] and os.path.isdir(tmp_path / str(E) / "proof")


def test_prp_20m_proof_residue_point(owl, tmp_path):
    """The proof residue at the first power-8 point of the 20M exponent. A PRP savefile holds the
    Gerbicz check value, from which the loop rebuilds its data; a savefile of 2,000 iterations is
    re-saved with its iteration count moved to the last block boundary before the point, so that the
    next 2,000 iterations cross it. The residue file must then exist in the reference's format
    (CRC-checked by its ProofSet::load, when oracle/_ref is built) and the Gerbicz checks on either
    side must pass."""
    g = load_golden("prp_20m")
    if g is None:
        pytest.skip("golden table not generated")
    E = g["E"]
    r = owl.prp_run(E, W=4096, H=2560, block=1000, stop_after=2000, save_dir=str(tmp_path))
    assert r["n_errors"] == 0 and r["k"] == 2000
    st = owl.prp_load(str(tmp_path), E)
    p1 = owl.proof_points(E, 8)[0]
    k0 = (p1 // 1000 - 1) * 1000
    owl.prp_save(str(tmp_path), E, k0, 1000, st["res64"], st["check"])
    r = owl.prp_run(E, W=4096, H=2560, block=1000, stop_after=2000, save_dir=str(tmp_path), proof_power=8)
    # (proof_power reports the power of a proof written at the end; this run stops before the end)
    assert r["n_errors"] == 0 and k0 + 2000 <= r["k"] < k0 + 3000 and r["k"] > p1
    path = tmp_path / str(E) / "proof" / str(p1)
    assert path.stat().st_size == ((E // 32) + 2) * 4  # CRC word + E/32+1 words (ProofSet::fileExists)
    ref = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libref_proof.so")
    if os.path.exists(ref):
        lib = ctypes.CDLL(ref)
        lib.ref_proofset_load.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_uint32)]
        import numpy as np
        words = np.zeros((E - 1) // 32 + 1, dtype=np.uint32)
        assert lib.ref_proofset_load(str(tmp_path).encode(), E, 8, p1,
                                     words.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))) == 0
        assert words.any()
