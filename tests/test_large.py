"""The large configuration: PRP-3 at the 20M FFT (N = 5 * 2^22 = 4096 x 2560, a radix-5 stage in the
column FFT), E the seeded prime in [330M, 335M], Gerbicz every 1,000 iterations, proof power 8 enabled
(its first residue point lies beyond the 5,000 iterations run here, so only the set-up and the
bookkeeping of the proof machinery run), res64 at every 1,000 iterations against the GMP golden table.
"""
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
