"""The host drivers (include/owl_host.h): the reference's PRP and LL loops on the GPU engine,
with Gerbicz checks, savefiles, resume, and a host-injected fault."""
import os

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("E", [86243, 110503])
def test_prp_of_mersenne_prime(owl, E):
    """M_E prime: isPrime, type-1 residue 3^(2^E)/9 = 1 (src/Gpu.cpp:1495-1504)."""
    r = owl.prp_run(E)
    assert r["finished"] and r["is_prime"]
    assert r["res64"] == 1
    assert r["res2048"] == "0" * 511 + "1"
    assert r["n_errors"] == 0


def test_prp_of_composite(owl):
    E = 86249  # prime exponent, composite Mersenne number
    r = owl.prp_run(E)
    assert r["finished"] and not r["is_prime"]


@pytest.mark.parametrize("E", [86243, 132049, 3021377])
def test_ll_of_mersenne_prime(owl, E):
    """LL to the end: the final value of a Mersenne prime is 0 (M3021377: 3.02 M iterations at
    the 256K FFT)."""
    r = owl.ll_run(E)
    assert r["finished"] and r["is_prime"] and r["res64"] == 0


def test_prp_golden_checkpoints_save_and_resume(owl, tmp_path):
    """res64 at every 1,000 iterations equals the GMP table; stopping at 10,000 and resuming
    from the savefile reaches the same res64 at 20,000."""
    g = load_golden("prp_256k")
    E = g["E"]
    r1 = owl.prp_run(E, log_step=1000, stop_after=10000, save_dir=str(tmp_path))
    assert not r1["finished"] and r1["k"] == 10000
    got = ["%016x" % res for (k, res) in r1["checkpoints"]]
    assert got == g["res64"][:10]
    assert os.path.exists(tmp_path / str(E) / ("%d-%09d.prp" % (E, 10000)))
    r2 = owl.prp_run(E, log_step=1000, stop_after=10000, save_dir=str(tmp_path))
    assert r2["k"] == 20000
    # resumed run: first checkpoint is the on-load state's successor
    ks = [k for (k, _) in r2["checkpoints"]]
    assert ks[0] == 11000 and ks[-1] == 20000
    assert ["%016x" % res for (_, res) in r2["checkpoints"]] == g["res64"][10:20]


def test_gerbicz_catches_injected_fault_and_recovers(owl, tmp_path):
    """A word flipped on the host after iteration 5,000 makes the next Gerbicz check fail; the
    driver reloads the last verified savefile, recomputes, and still proves M86243 prime."""
    E = 86243
    r = owl.prp_run(E, save_dir=str(tmp_path), inject_fault_k=5000, check_step=10000)
    assert r["finished"] and r["is_prime"] and r["res64"] == 1
    assert r["n_errors"] >= 1


@pytest.mark.parametrize("E,W,H", [(33000001, 1024, 1024), (66000001, 1024, 2048)])
def test_large_shape_short_blocks_repeat(owl, oracle, E, W, H):
    """Short blocks at the largest grids, repeated: the cross-CTA carry chain must give the
    same (GMP) answer every time."""
    from conftest import random_words
    w = random_words(E, 31337)
    want = {n: oracle.gmp_square(E, w, n) for n in (2, 3, 5)}
    with owl.Plan(E, W=W, H=H) as p:
        a = p.alloc()
        for rep in range(3):
            for n in (2, 3, 5):
                p.writeIn(a, w)
                p.squareLoop(a, a, n)
                assert np.array_equal(p.readOut(a), want[n]), (rep, n)


def test_prp_roe_statistics_and_danger_warning(owl, oracle):
    """Round-off statistics of the PRP loop (src/Gpu.cpp:1011-1025): sampled blocks give a Gumbel
    Z per log step. At 16 bits per word on the 8K FFT the 0.5 failure point is far off (Z well
    above 20, no warning); at 20.75 bits per word the same FFT runs close to it, Z drops and
    every log step whose Z is below 20 is counted as a "Danger ROE" warning."""
    N = 8192
    lo = owl.prp_run(oracle.lib.oracle_next_prime(16 * N), W=64, H=64, block=500, log_step=1000,
                     stop_after=3000)
    assert lo["roe_n"] >= 1000 and lo["n_danger_roe"] == 0
    assert lo["roe_z"] > 25 and lo["roe_max"] < 0.2
    hi = owl.prp_run(oracle.lib.oracle_next_prime(int(20.75 * N)), W=64, H=64, block=500, log_step=1000,
                     stop_after=3000)
    assert hi["roe_n"] >= 1000 and hi["roe_z"] < lo["roe_z"] and hi["roe_max"] > lo["roe_max"]
    if hi["roe_z_avg"] < 20:
        assert hi["n_danger_roe"] >= 1


def test_ll_roe_statistics(owl):
    """2,000 squarings sampled after the first 30, then 400 after the first log step."""
    r = owl.ll_run(86243, log_step=10000, stop_after=20000)
    assert r["finished"] is False and r["k"] == 20000
    assert r["roe_n"] == 2400 and r["roe_z"] > 20 and r["n_danger_roe"] == 0
