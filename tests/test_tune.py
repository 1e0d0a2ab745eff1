"""The autotuner (gpuowl_b200/tune.py; the reference's -tune and -ztune, src/tune.cpp:106-186).

CPU: the primality helpers, the Z statistic against the Gumbel law it assumes, and the tune.txt
row format (src/TuneEntry.cpp:94-105). GPU: one small shape sweep, and the Z-target (Z = 28)
max-bits-per-word search on the 16K FFT, checked against the round-off it implies.
"""
import math
import random

import pytest

from gpuowl_b200 import tune


def test_primes():
    # the reference's Primes: nextPrime(n) is the first odd prime above n, prevPrime(n) the last below
    assert [tune.next_prime(x) for x in (1, 2, 13, 136000000)] == [3, 3, 17, 136000021]
    assert tune.prev_prime(136000000) == 135999991 and tune.prev_prime(17) == 13
    assert tune.is_prime(136181029) and not tune.is_prime(136181029 * 3)


def test_roe_z_of_a_gumbel_sample():
    """For samples drawn from a Gumbel law (miu, beta), Z(x) = (x - miu) / beta."""
    rng = random.Random(7)
    miu, beta = 0.1, 0.015
    v = [miu - beta * math.log(-math.log(rng.random())) for _ in range(200000)]
    assert abs(tune.roe_z(v) - (0.5 - miu) / beta) < 0.3
    assert tune.roe_z([]) == 0.0


def test_tune_txt_rows(tmp_path):
    rows = {1 << 14: (64, 128, 12.5, 0.01), 1 << 15: (128, 128, 11.0, 0.02)}
    out, js = tmp_path / "tune.txt", tmp_path / "tune.json"
    tune.write(rows, 18.0, str(out), str(js))
    lines = out.read_text().splitlines()
    # cost never decreases with the size (a larger FFT is never listed as cheaper)
    assert lines == ["  12.5       64:1:128 # 294912", "  12.5      128:1:128 # 589824"]


def test_tune_rows_with_column_variants(tmp_path):
    """A sweep row names its column variant after the exponent in tune.txt and as element 5 in
    tune.json, where tuned_variant finds it (and a bits/word scan keeps it)."""
    rows = {5 << 18: (512, 1280, 30.0, 0.003, None, 2), 1 << 21: (1024, 1024, 31.0, 0.004, None, 1)}
    out, js = tmp_path / "tune.txt", tmp_path / "tune.json"
    tune.write(rows, 18.0, str(out), str(js))
    assert out.read_text().splitlines() == ["  30.0      512:5:256 # 23592960 v8",
                                            "  31.0       1K:2:512 # 37748736 v16"]
    assert tune.tuned_variant(5 << 18, str(js)) == 2 and tune.tuned_variant(1 << 21, str(js)) == 1
    assert tune.tuned_variant(1 << 22, str(js)) == 0 and tune.tuned_variant(1 << 22, None) == 0


@pytest.mark.gpu
def test_small_sweep_and_z_target(owl):
    rows = tune.tune(14, 14, 50, verbose=False)
    (W, H, us, roe, _, cv), = rows.values()
    assert 2 * W * H == 1 << 14 and us > 0 and roe < 0.1
    assert cv in tune.variants_for(H)
    best, (b1, z1), (b2, z2) = tune.max_bpw_z(1 << 14, W, H, 19.8, verbose=False)
    assert 31 <= z1 <= 37 or abs(z1 - 34) < 4
    assert 20 <= z2 <= 25 or abs(z2 - 22) < 4
    assert b2 > b1 and b2 >= best >= b1
    # the measured ROE-based limit for this FFT is 20.5 (max ROE 0.22 there); Z = 28 lies near it
    assert 19.5 < best < 21.0
