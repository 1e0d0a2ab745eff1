"""GPU parity of the split-precision form (owl_plan_set_split: INT8 tensor-core GEMMs on base-256
digit planes for the 32-point column stages of H = 2048, the 40-point ones of H = 2560 and the
16-point line stages of W = 2048) against the GMP oracle and the plain FP64 form.

Bar: bit-exact words / res64, and a round-off that stays close to the plain form's (the split form
adds about 2^-51 relative error per GEMM output; max ROE at most 2x plain + 0.02 and below 0.35).
"""
import numpy as np
import pytest

from conftest import load_golden, random_words, small_words

pytestmark = pytest.mark.gpu

# H = 2048 shapes: 256K, 2M and the 8M wavefront shape (whose 2048-point lines are split too)
SPLIT_SHAPES = [(4700021, 64, 2048), (37000003, 512, 2048), (136181029, 2048, 2048)]
# W = 2048 shapes whose columns have no split form: the line pass alone on the tensor cores
SPLIT_LINE_SHAPES = [(4500007, 2048, 64), (80000023, 2048, 1280)]


@pytest.mark.parametrize("E,W,H", SPLIT_SHAPES)
@pytest.mark.parametrize("ll", [False, True])
def test_split_square_vs_gmp(owl, oracle, E, W, H, ll):
    n = 20
    with owl.Plan(E, W=W, H=H, split=True) as p:
        start = random_words(E, E * 3 + 7)
        a = p.alloc()
        p.writeIn(a, start)
        p.squareLoop(a, a, n, ll=ll)
        got = p.readOut(a)
    assert np.array_equal(got, oracle.gmp_square(E, start, n, ll=ll))


# H = 2560 shapes (40-point GEMM stage): 640K, 5M and the 20M configuration's shape
SPLIT_SHAPES_2560 = [(5600027, 64, 2560), (90000049, 1024, 2560), (333000017, 4096, 2560)]


@pytest.mark.parametrize("E,W,H", SPLIT_SHAPES_2560)
@pytest.mark.parametrize("ll", [False, True])
def test_split_2560_square_vs_gmp(owl, oracle, E, W, H, ll):
    n = 20 if E < 10 ** 7 else 3
    with owl.Plan(E, W=W, H=H, split=True) as p:
        start = random_words(E, E * 5 + 1)
        a = p.alloc()
        p.writeIn(a, start)
        p.squareLoop(a, a, n, ll=ll)
        got = p.readOut(a)
    assert np.array_equal(got, oracle.gmp_square(E, start, n, ll=ll))


@pytest.mark.parametrize("E,W,H", SPLIT_LINE_SHAPES)
@pytest.mark.parametrize("ll", [False, True])
def test_split_line_pass_vs_gmp(owl, oracle, E, W, H, ll):
    """The line pass's 16-point GEMM stages (W = 2048) with FP64 columns, against GMP."""
    n = 20 if E < 10 ** 7 else 4
    with owl.Plan(E, W=W, H=H, split=owl.SPLIT_LINES) as p:
        start = random_words(E, E * 11 + 3)
        a = p.alloc()
        p.writeIn(a, start)
        p.squareLoop(a, a, n, ll=ll)
        got = p.readOut(a)
    assert np.array_equal(got, oracle.gmp_square(E, start, n, ll=ll))


@pytest.mark.parametrize("E,W,H", [SPLIT_SHAPES[0], SPLIT_SHAPES[2], SPLIT_SHAPES_2560[0], SPLIT_LINE_SHAPES[0]])
@pytest.mark.parametrize("mul3", [False, True])
def test_split_modmul_vs_gmp(owl, oracle, E, W, H, mul3):
    with owl.Plan(E, W=W, H=H, split=all_split(owl, W, H)) as p:
        wa, wb = random_words(E, 15), random_words(E, 16)
        a, b = p.alloc(), p.alloc()
        p.writeIn(a, wa)
        p.writeIn(b, wb)
        p.modMul(a, b, mul3=mul3)
        got = p.readOut(a)
    assert np.array_equal(got, oracle.gmp_mul(E, wa, wb, mul3=mul3))


def test_split_blocks_match_plain_and_roe(owl):
    """2,000 graph-launched squarings at 8M from 3: identical words in both forms; ROE close."""
    E, n = 136181029, 2000
    out = {}
    for split in (False, True):
        with owl.Plan(E, W=2048, H=2048, split=split) as p:
            a = p.alloc()
            p.writeIn(a, small_words(E, 3))
            p.readROE()
            p.squareLoop(a, a, n)
            out[split] = (p.readOut(a), float(p.readROE().max()))
    assert np.array_equal(out[False][0], out[True][0])
    roe_plain, roe_split = out[False][1], out[True][1]
    assert roe_split < 0.35
    assert roe_split <= 2 * roe_plain + 0.02, (roe_plain, roe_split)


def all_split(owl, W, H):
    """Every split-precision pass the shape has."""
    return (owl.SPLIT_COLUMNS if H in (2048, 2560) else 0) | (owl.SPLIT_LINES if W == 2048 else 0)


def test_split_both_passes_at_8m_match_plain(owl):
    """1,000 graph-launched squarings at 8M from 3 with both passes split: identical words to the
    plain form; ROE close."""
    E, n = 136181029, 1000
    out = {}
    for split in (0, owl.SPLIT_COLUMNS | owl.SPLIT_LINES):
        with owl.Plan(E, W=2048, H=2048, split=split) as p:
            assert p.split == split
            a = p.alloc()
            p.writeIn(a, small_words(E, 3))
            p.readROE()
            p.squareLoop(a, a, n)
            out[split] = (p.readOut(a), float(p.readROE().max()))
    (w0, r0), (w1, r1) = out.values()
    assert np.array_equal(w0, w1)
    assert r1 < 0.35 and r1 <= 2 * r0 + 0.02, (r0, r1)


def test_split_blocks_match_plain_at_20m(owl):
    """1,000 graph-launched squarings at the 20M shape (4096 x 2560) from 3: identical words in both
    forms; ROE close."""
    E, n = 331480451, 1000
    out = {}
    for split in (False, True):
        with owl.Plan(E, W=4096, H=2560, split=split) as p:
            a = p.alloc()
            p.writeIn(a, small_words(E, 3))
            p.readROE()
            p.squareLoop(a, a, n)
            out[split] = (p.readOut(a), float(p.readROE().max()))
    assert np.array_equal(out[False][0], out[True][0])
    roe_plain, roe_split = out[False][1], out[True][1]
    assert roe_split < 0.35
    assert roe_split <= 2 * roe_plain + 0.02, (roe_plain, roe_split)


def test_split_prp_driver_gerbicz(owl):
    """The C++ PRP loop (Gerbicz check every block) with the split form: same res64 checkpoints as
    the plain form over 10,000 iterations, no check failure."""
    E = 4700021
    runs = [owl.prp_run(E, W=64, H=2048, block=500, log_step=1000, stop_after=10000, split=s) for s in (False, True)]
    assert runs[1]["n_errors"] == 0 and runs[0]["n_errors"] == 0
    assert runs[1]["k"] == runs[0]["k"] >= 10000
    assert runs[1]["checkpoints"] == runs[0]["checkpoints"] and len(runs[0]["checkpoints"]) >= 10


def test_split_rejects_other_heights(owl):
    """A split flag whose pass has no split form at the plan's shape is refused."""
    with owl.Plan(1000003, W=128, H=256) as p:
        for flags in (True, owl.SPLIT_LINES, 4):
            with pytest.raises(owl.OwlError) as e:
                p.set_split(flags)
            assert e.value.status == -1
    with owl.Plan(4500007, W=2048, H=64) as p:
        with pytest.raises(owl.OwlError):
            p.set_split(owl.SPLIT_COLUMNS)
        p.set_split(owl.SPLIT_LINES)


def test_tc_wait_timeout_probe_keeps_plan_usable(owl, oracle):
    """The tensor-core completion wait is bounded: a barrier nothing arrives on times out with
    ERR_TIMEOUT after the plan's limit, and the plan still computes in the split form."""
    E = 4700021
    with owl.Plan(E, W=64, H=2048, split=True) as p:
        p.set_timeout(20_000_000)  # 20 ms
        assert p.probe_tc_wait_timeout() == owl.ERR_TIMEOUT
        p.set_timeout(2_000_000_000)
        a = p.alloc()
        w = random_words(E, 77)
        p.writeIn(a, w)
        p.squareLoop(a, a, 3)
        assert np.array_equal(p.readOut(a), oracle.gmp_square(E, w, 3))


def test_split_plans_in_one_batch(owl, oracle):
    """Two split-form plans (different widths) squared as one batch graph, against GMP."""
    exps = [(4700021, 64, 2048), (9400013, 128, 2048)]
    plans = [owl.Plan(E, W=W, H=H, split=True) for (E, W, H) in exps]
    try:
        bufs, starts = [], []
        for p in plans:
            b = p.alloc()
            w = random_words(p.E, p.E + 5)
            p.writeIn(b, w)
            bufs.append(b)
            starts.append(w)
        with owl.Batch(plans) as batch:
            batch.square(bufs, 17)
            batch.sync()
        for p, b, w in zip(plans, bufs, starts):
            assert np.array_equal(p.readOut(b), oracle.gmp_square(p.E, w, 17)), p.E
    finally:
        for p in plans:
            p.close()


@pytest.mark.parametrize("name,W,H,flags", [("prp_8m", 2048, 2048, 3), ("prp_20m", 4096, 2560, 1)])
def test_split_prp_driver_golden(owl, name, W, H, flags):
    """The PRP driver (Gerbicz check every block) in the split-precision form at the 8M (both passes
    split) and 20M (column pass split) configurations: res64 at every 1,000 iterations equal to the
    GMP golden table, no check failure."""
    g = load_golden(name)
    r = owl.prp_run(g["E"], W=W, H=H, block=1000, log_step=1000, stop_after=g["iters"], split=flags)
    assert r["n_errors"] == 0 and r["k"] >= g["iters"]
    got = {k: "%016x" % v for k, v in r["checkpoints"]}
    for i, want in enumerate(g["res64"]):
        assert got.get((i + 1) * g["step"]) == want, (i + 1) * g["step"]
