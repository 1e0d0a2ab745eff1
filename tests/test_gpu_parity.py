"""GPU parity: libowl (through the C ABI) against the GMP oracle and the golden res64 tables.

Bar: bit-exact integers -- identical compact words / res64 -- for every case.
"""
import numpy as np
import pytest

from conftest import load_golden, random_words, res64_of, small_words

pytestmark = pytest.mark.gpu

# (E, W, H): every pass-1 / pass-2 instantiation from 8K to 8M words, at 10.5 .. 19 bits/word
SHAPES = [
    (86243, 64, 64), (216091, 64, 128), (500009, 128, 128), (1000003, 128, 256),
    (1999993, 256, 256), (4989349, 256, 512), (9000011, 512, 512), (17000023, 512, 1024),
    (33000001, 1024, 1024), (66000001, 1024, 2048), (136181029, 2048, 2048),
]


@pytest.mark.parametrize("E,W,H", SHAPES[:7])
@pytest.mark.parametrize("ll", [False, True])
def test_square_random_vs_gmp(owl, oracle, E, W, H, ll):
    """n squarings of a random residue equal GMP's, word for word."""
    n = 20
    with owl.Plan(E, W=W, H=H) as p:
        start = random_words(E, E * 7 + 1)
        a = p.alloc()
        p.writeIn(a, start)
        p.squareLoop(a, a, n, ll=ll)
        got = p.readOut(a)
    want = oracle.gmp_square(E, start, n, ll=ll)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("E,W,H", SHAPES[7:])
def test_square_large_shapes_vs_gmp(owl, oracle, E, W, H):
    n = 6
    with owl.Plan(E, W=W, H=H) as p:
        start = random_words(E, E + 3)
        a = p.alloc()
        p.writeIn(a, start)
        p.squareLoop(a, a, n)
        got = p.readOut(a)
    want = oracle.gmp_square(E, start, n)
    assert np.array_equal(got, want)


# 5 * 2^k FFT lengths (radix-5 middle stage of the column FFT, H = 640, 1280, 2560) and the
# 512-thread 4096-point instantiations, up to the 20M (5 * 2^22) and 32M lengths
SHAPES_WIDE = [
    (1300021, 64, 640), (2500009, 64, 1280), (20000003, 1024, 640), (40000003, 1024, 1280),
    (80000023, 2048, 1280), (270000017, 2048, 4096), (333000017, 4096, 2560), (536000009, 4096, 4096),
]


@pytest.mark.parametrize("E,W,H", SHAPES_WIDE)
def test_square_radix5_and_4k_shapes_vs_gmp(owl, oracle, E, W, H):
    n = 4
    with owl.Plan(E, W=W, H=H) as p:
        start = random_words(E, E + 11)
        a = p.alloc()
        p.writeIn(a, start)
        p.squareLoop(a, a, n)
        got = p.readOut(a)
        roe = float(p.readROE().max())
    want = oracle.gmp_square(E, start, n)
    assert np.array_equal(got, want)
    assert roe < 0.3


@pytest.mark.parametrize("E,W,H", [SHAPES[2], SHAPES[5], SHAPES[8], SHAPES_WIDE[0]])
def test_square_without_roe(owl, oracle, E, W, H):
    """OWL_SQ_NO_ROE: the line passes built without the round-off measurement give the same words
    (GMP), record no round-off, and mix with measured blocks."""
    n = 20
    with owl.Plan(E, W=W, H=H) as p:
        start = random_words(E, 7)
        a = p.alloc()
        p.writeIn(a, start)
        p.readROE()
        p.squareLoop(a, a, n, roe=False)
        assert p.readROE().size == 0
        p.squareLoop(a, a, n)
        roe = p.readROE()
        assert roe.size == n and 0 < roe.max() < 0.4
        got = p.readOut(a)
    assert np.array_equal(got, oracle.gmp_square(E, start, 2 * n))


@pytest.mark.parametrize("E,W,H", [SHAPES[0], SHAPES[3], SHAPES[5], SHAPES[8]])
def test_mul3_last(owl, oracle, E, W, H):
    """squareLoop with doTailMul3: the last squaring is multiplied by 3 (Gerbicz aux)."""
    n = 7
    with owl.Plan(E, W=W, H=H) as p:
        start = random_words(E, 99)
        a = p.alloc()
        p.writeIn(a, start)
        p.squareLoop(a, a, n, mul3=True)
        got = p.readOut(a)
    want = oracle.gmp_mul(E, oracle.gmp_square(E, start, n), small_words(E, 3))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("E,W,H", [SHAPES[0], SHAPES[2], SHAPES[5], SHAPES[8], SHAPES[10], SHAPES_WIDE[2]])
@pytest.mark.parametrize("mul3", [False, True])
def test_modmul_vs_gmp(owl, oracle, E, W, H, mul3):
    with owl.Plan(E, W=W, H=H) as p:
        wa, wb = random_words(E, 5), random_words(E, 6)
        a, b = p.alloc(), p.alloc()
        p.writeIn(a, wa)
        p.writeIn(b, wb)
        p.modMul(a, b, mul3=mul3)
        got = p.readOut(a)
        # the second operand is untouched
        assert np.array_equal(p.readOut(b), oracle.gmp_square(E, wb, 0))
    assert np.array_equal(got, oracle.gmp_mul(E, wa, wb, mul3=mul3))


def test_write_read_roundtrip_and_res64(owl, oracle):
    E = 4989349
    with owl.Plan(E) as p:
        w = random_words(E, 1234)
        a = p.alloc()
        p.writeIn(a, w)
        assert np.array_equal(p.readOut(a), w)
        assert p.bufResidue(a) == res64_of(w)
        # digits agree with the oracle's expandBits
        assert np.array_equal(p.read_digits(a), oracle.expand(E, p.N, w))
        p.squareLoop(a, a, 3)
        out = p.readOut(a)
        assert p.bufResidue(a) == res64_of(out)


def test_is_equal_and_sum64(owl):
    E = 216091
    with owl.Plan(E) as p:
        a, b = p.alloc(), p.alloc()
        w = random_words(E, 77)
        p.writeIn(a, w)
        p.copy(b, a)
        assert p.isEqual(a, b)
        d = p.read_digits(a)
        d[12345 % p.N] += 1
        p.write_digits(b, d)
        assert not p.isEqual(a, b)
        want = int(np.ascontiguousarray(p.read_digits(a)).view(np.uint64).sum(dtype=np.uint64))
        assert p.sum64(a) == want


@pytest.mark.parametrize("E", [86243, 110503, 132049])
def test_mersenne_prime_prp_is_9(owl, E):
    """M_E prime: 3^(2^E) = 9 mod M_E (the reference's equals9, src/Gpu.cpp:1036-1040)."""
    with owl.Plan(E) as p:
        a = p.alloc()
        p.writeIn(a, small_words(E, 3))
        p.squareLoop(a, a, E)
        w = p.readOut(a)
    assert w[0] == 9 and not w[1:].any()


@pytest.mark.parametrize("E", [86243, 132049])
def test_mersenne_prime_ll_is_0(owl, E):
    """M_E prime: the LL sequence from 4 reaches 0 after E-2 steps."""
    with owl.Plan(E) as p:
        a = p.alloc()
        p.writeIn(a, small_words(E, 4))
        p.squareLoop(a, a, E - 2, ll=True)
        w = p.readOut(a)
    # 0 mod M_E may come back as 0 or as M_E itself (all ones)
    full = np.full_like(w, 0xFFFFFFFF)
    if E % 32:
        full[-1] = (1 << (E % 32)) - 1
    assert not w.any() or np.array_equal(w, full)


def _run_golden(owl, item, shape=None):
    E, step, iters = item["E"], item["step"], item["iters"]
    ll = item["kind"] == "ll"
    kw = {} if shape is None else dict(W=shape[0], H=shape[1])
    with owl.Plan(E, **kw) as p:
        a = p.alloc()
        p.writeIn(a, small_words(E, item["start"]))
        got = []
        for _ in range(iters // step):
            p.squareLoop(a, a, step, ll=ll)
            got.append("%016x" % p.bufResidue(a))
        roe = p.readROE()
    return got, float(roe.max()) if roe.size else 0.0


def test_golden_small(owl):
    g = load_golden("small")
    for item in g["items"]:
        if item["E"] < 65536:
            continue  # below the smallest FFT (N = 8K at <= 19 bits/word is fine, but 2 bits/word is not)
        got, roe = _run_golden(owl, item)
        assert got == item["res64"], item["E"]
        assert roe < 0.3


def test_golden_prp_256k(owl):
    """PRP-3 at 256K, E from seed in [4.8M, 5.0M] (19.03 bits/word), 20,000 iterations."""
    g = load_golden("prp_256k")
    got, roe = _run_golden(owl, g)
    assert got == g["res64"]
    assert roe < 0.45


@pytest.mark.parametrize("name", ["prp_8m", "ll_8m"])
def test_golden_8m(owl, name):
    """8M FFT (W=H=2048), E from seed in [136M, 139M], 10,000 iterations: res64 every 1,000,
    and the max round-off stays within the 0.35 bound."""
    g = load_golden(name)
    got, roe = _run_golden(owl, g, shape=(2048, 2048))
    assert got == g["res64"]
    assert roe <= 0.35


def test_wait_timeout_probe_keeps_plan_usable(owl, oracle):
    """A device wait that nothing ends returns OWL_ERR_TIMEOUT; the plan then still computes."""
    E = 86243
    with owl.Plan(E) as p:
        p.set_timeout(5_000_000)  # 5 ms
        assert p.probe_wait_timeout() == owl.ERR_TIMEOUT
        p.set_timeout(2_000_000_000)
        a = p.alloc()
        w = random_words(E, 3)
        p.writeIn(a, w)
        p.squareLoop(a, a, 5)
        assert np.array_equal(p.readOut(a), oracle.gmp_square(E, w, 5))


@pytest.mark.parametrize("E", [216091, 4989349])
def test_gerbicz_identity_and_injected_fault(owl, E):
    """Reference PRP loop + doCheck (src/Gpu.cpp:738-771): after blocks of
    check *= data; data <- data^(2^B), the identity check^(2^B) * 3 == check * data
    holds and isEqual sees it on the digits; one flipped word in data breaks it."""
    B = 40
    with owl.Plan(E) as p:
        data, check, aux = p.alloc(), p.alloc(), p.alloc()
        p.writeIn(data, small_words(E, 3))
        p.writeIn(check, small_words(E, 1))
        for _ in range(3):
            p.modMul(check, data)
            p.squareLoop(data, data, B)
        saved = p.alloc()
        p.copy(saved, check)
        p.squareLoop(aux, check, B, mul3=True)
        p.modMul(check, data)
        assert p.isEqual(check, aux)
        # fault injected on the host between blocks: the check must fail
        d = p.read_digits(data)
        d[777] ^= 1
        p.write_digits(data, d)
        p.copy(check, saved)
        p.modMul(check, data)
        assert not p.isEqual(check, aux)


def test_batch_of_uneven_exponents_matches_gmp(owl, oracle):
    """Exponents with different FFT shapes squared as one graph launch, twice in a row."""
    exps = [(1000003, 128, 256), (1999993, 256, 256), (4989349, 256, 512), (2302981, 256, 256),
            (9000011, 512, 512), (500009, 128, 128)]
    plans = [owl.Plan(E, W=W, H=H) for (E, W, H) in exps]
    try:
        bufs, starts = [], []
        for p in plans:
            b = p.alloc()
            w = random_words(p.E, p.E + 11)
            p.writeIn(b, w)
            bufs.append(b)
            starts.append(w)
        with owl.Batch(plans) as batch:
            batch.square(bufs, 17)
            batch.square(bufs, 17)
            batch.sync()
        for p, b, w in zip(plans, bufs, starts):
            assert np.array_equal(p.readOut(b), oracle.gmp_square(p.E, w, 34)), p.E
    finally:
        for p in plans:
            p.close()


def test_batch64_golden(owl):
    """The 64-exponent batch (log-uniform in [1M, 20M], FFT at <= 19 bits/word) run as one graph per
    1,000-iteration block: res64 after 1,000 and 2,000 iterations equal the GMP golden table."""
    golden = load_golden("batch64")
    if golden is None:
        pytest.skip("golden table not generated")
    plans = []
    for it in golden["items"]:
        _, W, H = owl.fft_choose(it["E"], 19.0)
        plans.append(owl.Plan(it["E"], W=W, H=H))
    try:
        bufs = []
        for p in plans:
            b = p.alloc()
            p.writeIn(b, small_words(p.E, 3))
            bufs.append(b)
        got = [[] for _ in plans]
        with owl.Batch(plans) as batch:
            for _ in range(2):
                batch.square(bufs, 1000)
                batch.sync()
                for i, (p, b) in enumerate(zip(plans, bufs)):
                    got[i].append("%016x" % p.bufResidue(b))
        for it, g in zip(golden["items"], got):
            assert g == it["res64"][:2], it["E"]
    finally:
        for p in plans:
            p.close()


def test_batch64_10k_golden(owl):
    """All 64 exponents of the batch (9 FFT sizes from 64K to 1M, plans of one shape as grouped
    launches) for 10,000 iterations in one batch: res64 at every 1,000 equal the GMP golden table
    (640 checkpoints)."""
    golden = load_golden("batch64_10k")
    plans = []
    for it in golden["items"]:
        _, W, H = owl.fft_choose(it["E"], 19.0)
        plans.append(owl.Plan(it["E"], W=W, H=H))
    try:
        bufs = []
        for p in plans:
            b = p.alloc()
            p.writeIn(b, small_words(p.E, 3))
            bufs.append(b)
        got = [[] for _ in plans]
        with owl.Batch(plans) as batch:
            for blk in range(10):
                batch.square(bufs, 1000, roe=blk < 2)
                batch.sync()
                for i, (p, b) in enumerate(zip(plans, bufs)):
                    got[i].append("%016x" % p.bufResidue(b))
        for it, g in zip(golden["items"], got):
            assert g == it["res64"], it["E"]
    finally:
        for p in plans:
            p.close()


@pytest.mark.parametrize("ll", [False, True])
def test_batch_grouped_launches_vs_gmp(owl, oracle, ll):
    """Five plans of one shape (grouped launches) and one of another, squared together: each equals
    GMP; the round-off is recorded per plan."""
    exps = [86243, 86249, 100003, 110503, 120011]
    plans = [owl.Plan(E, W=64, H=64) for E in exps] + [owl.Plan(500009, W=128, H=128)]
    try:
        bufs, starts = [], []
        for p in plans:
            b = p.alloc()
            w = random_words(p.E, p.E ^ 0xBA7C)
            p.writeIn(b, w)
            bufs.append(b)
            starts.append(w)
            p.readROE()
        with owl.Batch(plans) as batch:
            batch.square(bufs, 30, ll=ll)
            batch.sync()
        for p, b, w in zip(plans, bufs, starts):
            assert np.array_equal(p.readOut(b), oracle.gmp_square(p.E, w, 30, ll=ll)), p.E
            roe = p.readROE()
            assert roe.size == 30 and 0 < roe.max() < 0.3
    finally:
        for p in plans:
            p.close()


# every column variant besides the shape's default one, on a shape of each kind it is built for
# (the defaults: 8 values a thread at 128 x 256, 256 x 256 and 512 x 512, two CTAs per SM at
# 4096 x 2560, else 16 values a thread)
VARIANT_CASES = [
    (86243, 64, 64, "v8"), (500009, 128, 128, "v8"), (4989349, 256, 512, "v8"), (33000001, 1024, 1024, "v8"),
    (136181029, 2048, 2048, "v8"), (1300021, 64, 640, "v8"), (2500009, 64, 1280, "v8"),
    (80000023, 2048, 1280, "v8"), (1999993, 256, 256, "v16"), (9000011, 512, 512, "v16"),
    (333000017, 4096, 2560, "v16"),
]


@pytest.mark.parametrize("E,W,H,variant", VARIANT_CASES)
def test_column_variants_vs_gmp(owl, oracle, E, W, H, variant):
    """A plan on another column variant (owl_plan_set_column_variant) squares bit-exactly: GMP's
    result, and the same digits as the default variant's plan."""
    cv = {v: k for k, v in owl.COL_NAMES.items()}[variant]
    assert owl.column_variant_supported(H, cv)
    with owl.Plan(E, W=W, H=H) as p:
        assert p.column_variant != cv
    n = 12 if E < 10 ** 7 else 4
    start = random_words(E, E ^ 0xC01)
    got = {}
    for v in (owl.COL_AUTO, cv):
        with owl.Plan(E, W=W, H=H, column_variant=v) as p:
            assert v == owl.COL_AUTO or p.column_variant == cv
            a = p.alloc()
            p.writeIn(a, start)
            p.squareLoop(a, a, n)
            got[v] = p.readOut(a)
            assert p.readROE().max() < 0.3
    assert np.array_equal(got[cv], got[owl.COL_AUTO])
    assert np.array_equal(got[cv], oracle.gmp_square(E, start, n))


def test_column_variant_rules(owl):
    """Variants not built for the plan's H are refused, OWL_COL_AUTO restores the default, and a
    switch drops the plan's graphs (the next block still equals the default plan's)."""
    with owl.Plan(4989349, W=256, H=512) as p:
        default = p.column_variant
        assert default in (owl.COL_V16, owl.COL_V8)
        with pytest.raises(owl.OwlError):
            p.set_column_variant(owl.COL_V16_OCC2)
        with pytest.raises(owl.OwlError):
            p.set_column_variant(9)
        assert p.column_variant == default
        a = p.alloc()
        p.writeIn(a, small_words(p.E, 3))
        p.squareLoop(a, a, 20)                          # a graph of the default variant
        p.set_column_variant(owl.COL_V8 if default == owl.COL_V16 else owl.COL_V16)
        p.squareLoop(a, a, 20)
        p.set_column_variant(owl.COL_AUTO)
        assert p.column_variant == default
        p.squareLoop(a, a, 20)
        r1 = p.bufResidue(a)
    with owl.Plan(4989349, W=256, H=512) as q:
        b = q.alloc()
        q.writeIn(b, small_words(q.E, 3))
        q.squareLoop(b, b, 60)
        assert q.bufResidue(b) == r1
    assert not owl.column_variant_supported(4096, owl.COL_V8)
    assert not owl.column_variant_supported(2560, owl.COL_V8)
    assert owl.column_variant_supported(2560, owl.COL_V16_OCC2)


def test_batch_groups_split_by_column_variant(owl, oracle):
    """Plans of one shape on two column variants are squared in one batch (one grouped launch per
    variant): each equals GMP."""
    exps = [86243, 86249, 100003, 110503]
    plans = [owl.Plan(E, W=64, H=64, column_variant=(owl.COL_V8 if i % 2 else owl.COL_V16))
             for i, E in enumerate(exps)]
    try:
        bufs, starts = [], []
        for p in plans:
            b = p.alloc()
            w = random_words(p.E, p.E ^ 0x5EED)
            p.writeIn(b, w)
            bufs.append(b)
            starts.append(w)
        with owl.Batch(plans) as batch:
            batch.square(bufs, 25)
            batch.sync()
        for p, b, w in zip(plans, bufs, starts):
            assert np.array_equal(p.readOut(b), oracle.gmp_square(p.E, w, 25)), (p.E, p.column_variant)
    finally:
        for p in plans:
            p.close()


def _pattern_words(E, N, pattern):
    """0: 3, 1: 2^E - 1, 2: every raw digit 2^(bits-1) - 1 (one carry runs through all digits),
    3: zero, 4: 2^E - 2, else random."""
    nw = (E - 1) // 32 + 1
    if pattern == 0:
        return small_words(E, 3)
    if pattern in (1, 4):
        w = np.full(nw, 0xffffffff, dtype=np.uint32)
        w[-1] &= (1 << (E % 32)) - 1
        if pattern == 4:
            w[0] -= 1
        return w
    if pattern == 2:
        x, off = 0, 0
        for k in range(N):
            nxt = -(-(k + 1) * E // N)
            ln = nxt - off
            x |= ((1 << (ln - 1)) - 1) << off
            off = nxt
        return np.frombuffer(x.to_bytes(4 * nw, "little"), dtype=np.uint32).copy()
    if pattern == 3:
        return np.zeros(nw, dtype=np.uint32)
    return random_words(E, pattern)


@pytest.mark.parametrize("E,W,H", [SHAPES[0], SHAPES[5], SHAPES[10], SHAPES_WIDE[0]])
@pytest.mark.parametrize("pattern", [0, 1, 2, 3, 4, 77])
def test_device_expand_compact_match_host(owl, oracle, E, W, H, pattern):
    """owl_write_words / owl_read_words convert on the device; the digits and words must equal the
    host restatement of the reference's expandBits / compactBits bit for bit."""
    with owl.Plan(E, W=W, H=H) as p:
        if pattern == 2 and p.N > (1 << 18):
            pytest.skip("pattern built digit by digit in Python; small N only")
        words = _pattern_words(E, p.N, pattern)
        a = p.alloc()
        p.writeIn(a, words)
        digits = p.read_digits(a)
        assert np.array_equal(digits, oracle.expand(E, p.N, words))
        assert np.array_equal(p.readOut(a), oracle.compact(E, p.N, digits))
