"""Autotuner for FFT shapes (replaces the reference's -tune, src/tune.cpp:106-186, which times
each FFT with Gpu::timePRP and writes tune.txt).

    python -m gpuowl_b200.tune [--min-lg 13] [--max-lg 23] [--iters 200] [--out tune.txt]
    python -m gpuowl_b200.tune --bpw-scan tune.json [--criterion z|roe] --out bpw.txt

For every FFT size N = 2^lg, and N = 5 * 2^(lg-3) with --five, it times each W x H split the library
supports (W a power of two in [64, 4096]; H a power of two in [64, 4096] with H/W in {1/2, 1, 2, 4},
or H in {640, 1280, 2560}) and, for each split, every column-pass variant built for its H (the radix
plan and tile of the column FFT: 16 or 8 values a thread, one or two CTAs per SM; include/owl.h
OWL_COL_*), by the time per squaring of a graph-launched block (at an exponent of 18 bits per word), keeps the
fastest, and records its max round-off. Output:
  - tune.txt in the reference's format, "%6.1f %14s # %u" = microseconds per iteration, shape,
    largest exponent (src/TuneEntry.cpp:94-105), rows in increasing cost and exponent, followed by
    the column variant's name;
  - tune.json, {"N": [W, H, us_per_iter, max_roe, max_bpw or null, column_variant]}, read by
    fft_choose(..., tune=path) and tuned_variant(N, path).

    python -m gpuowl_b200.tune --shapes 4096x2560 --variants   # per-pass times of every variant
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def spec(W, H):
    """The reference's W:M:H shape grammar, H = M * height (height 256, 512 or 1K) when possible."""
    def k(n):
        return "%dK" % (n // 1024) if n % 1024 == 0 else str(n)
    for h in (1024, 512, 256):
        if H % h == 0 and 2 <= H // h <= 16:
            return "%s:%d:%s" % (k(W), H // h, k(h))
    return "%s:1:%s" % (k(W), k(H))


def candidates(N):
    hN = N // 2
    out = []
    for w in (64, 128, 256, 512, 1024, 2048, 4096):
        h = hN // w
        if w * h != hN:
            continue
        if h in (640, 1280, 2560) or (64 <= h <= 4096 and h in (w // 2, w, 2 * w, 4 * w)):
            out.append((w, h))
    return out


def sizes(min_lg, max_lg, five):
    out = []
    for lg in range(min_lg, max_lg + 1):
        if five and lg >= 3:
            out.append(5 << (lg - 3))
        out.append(1 << lg)
    return out


def next_odd_exponent(x):
    x = int(x) | 1
    return x


def variants_for(H):
    """The column-pass variants built for columns of H points (OWL_COL_V16 first)."""
    import gpuowl_b200 as owl
    return [v for v in (owl.COL_V16, owl.COL_V8, owl.COL_V16_OCC2) if owl.column_variant_supported(H, v)]


def tune(min_lg, max_lg, iters, max_bpw=18.0, device=0, verbose=True, five=False, variants=True):
    import numpy as np
    import gpuowl_b200 as owl
    from gpuowl_b200 import build
    build.build()
    rows = {}
    for N in sizes(min_lg, max_lg, five):
        E = next_odd_exponent(N * max_bpw * 0.98)
        best = None
        for (W, H) in candidates(N):
            for cv in (variants_for(H) if variants else [owl.COL_AUTO]):
                with owl.Plan(E, device=device, W=W, H=H, column_variant=cv) as p:
                    b = p.alloc()
                    rng = np.random.default_rng(N)
                    w = rng.integers(0, 2 ** 32, size=p.nwords, dtype=np.uint64).astype(np.uint32)
                    if E % 32:
                        w[-1] &= (1 << (E % 32)) - 1
                    p.writeIn(b, w)
                    p.profile_square(b, 20)  # warm
                    p.readROE()
                    p.profile_square(b, iters)
                    roe = float(p.readROE().max())
                    us = block_us(p, b, iters)
                    cv = p.column_variant
                if verbose:
                    print("N=%-9d %-14s %-8s %8.2f us/iter  max ROE %.4f"
                          % (N, spec(W, H), owl.COL_NAMES[cv], us, roe), flush=True)
                if best is None or us < best[2]:
                    best = (W, H, us, roe, None, cv)
        if best:
            rows[N] = best
    return rows


def block_us(p, b, iters, reps=2):
    """Microseconds per squaring of a graph-launched block of `iters` squarings, wall clock from
    launch to completion (the reference's timePRP measures the same way), best of `reps` blocks.
    The per-pass stamps of profile_square overlap where a pass starts as a programmatic dependent
    of the one before, so their sum is not the iteration time."""
    import time
    p.squareLoop(b, b, iters)  # captures the block's graph
    p.sync()
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        p.squareLoop(b, b, iters)
        p.sync()
        dt = 1e6 * (time.perf_counter() - t0) / iters
        best = dt if best is None else min(best, dt)
    return best


def tuned_variant(N, tune_json):
    """The column variant tune.json holds for FFT size N (OWL_COL_AUTO when it holds none)."""
    import gpuowl_b200 as owl
    if not tune_json or not os.path.exists(tune_json):
        return owl.COL_AUTO
    with open(tune_json) as f:
        v = json.load(f).get(str(int(N)))
    return int(v[5]) if v and len(v) >= 6 and v[5] else owl.COL_AUTO


def profile_shapes(shapes, iters, bpw=16.0, device=0, split=False, variants=False):
    """Per-kernel device time of `iters` squarings on each W x H shape (the -time profile per shape),
    and the time per squaring of a whole block (block_us): E is the first odd number above N * bpw,
    the residue random; one untimed block first. With
    `split` (OWL_SPLIT_* flags) the column pass (H = 2048 or 2560) and / or the line pass (W = 2048)
    run in the split-precision form; with `variants` every
    column variant built for H is timed, else the shape's default. The res64 after the timed block
    is returned with each row (the same for every variant of a shape)."""
    import numpy as np
    import gpuowl_b200 as owl
    from gpuowl_b200 import build
    build.build()
    rows = []
    for (W, H) in shapes:
        N = 2 * W * H
        E = next_odd_exponent(N * bpw)
        for cv in (variants_for(H) if variants else [owl.COL_AUTO]):
            with owl.Plan(E, device=device, W=W, H=H, split=split, column_variant=cv) as p:
                b = p.alloc()
                rng = np.random.default_rng(N)
                w = rng.integers(0, 2 ** 32, size=p.nwords, dtype=np.uint64).astype(np.uint32)
                if E % 32:
                    w[-1] &= (1 << (E % 32)) - 1
                p.writeIn(b, w)
                p.profile_square(b, iters)
                p.readROE()
                prof = p.profile_square(b, iters)
                roe = float(p.readROE().max())
                res = p.bufResidue(b)
                total = block_us(p, b, iters)
                cv = p.column_variant
            us2 = 1e3 * prof["pass2"][0] / prof["pass2"][1]
            us1 = 1e3 * prof["pass1"][0] / prof["pass1"][1]
            rows.append((N, W, H, total, us2, us1, roe, cv, res))
            print("N=%-9d %-14s %-8s %8.2f us/iter  column pass %7.2f us  line pass %7.2f us  max ROE %.4f  "
                  "res64 %016x" % (N, spec(W, H), owl.COL_NAMES[cv], total, us2, us1, roe, res), flush=True)
    return rows


def roe_at(N, W, H, bpw, iters, device=0):
    """Max round-off of `iters` squarings of a random residue at E = N * bpw (odd) on W x H."""
    import numpy as np
    import gpuowl_b200 as owl
    E = next_odd_exponent(N * bpw)
    with owl.Plan(E, device=device, W=W, H=H) as p:
        b = p.alloc()
        rng = np.random.default_rng(E)
        w = rng.integers(0, 2 ** 32, size=p.nwords, dtype=np.uint64).astype(np.uint32)
        if E % 32:
            w[-1] &= (1 << (E % 32)) - 1
        p.writeIn(b, w)
        p.squareLoop(b, b, 20)
        p.readROE()
        done = 0
        while done < iters:
            n = min(1000, iters - done)
            p.squareLoop(b, b, n)
            done += n
        return float(p.readROE().max())


def is_prime(n):
    """Deterministic Miller-Rabin for n < 3.3e24 (the bases 2..41)."""
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41)
    for p in small:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def prev_prime(n):
    """The largest odd prime below n (Primes::prevPrime, src/Primes.cpp:37-43)."""
    n = int(n) - 1
    n -= (n % 2 == 0)
    while not is_prime(n):
        n -= 2
    return n


def next_prime(n):
    """The smallest odd prime above n (Primes::nextPrime, src/Primes.cpp:45-50)."""
    n = int(n) + 1
    n += (n % 2 == 0)
    while not is_prime(n):
        n += 2
    return n


def roe_z(values, x=0.5):
    """Z of a sample of per-squaring round-off maxima: the reference's Gumbel fit (RoeInfo,
    src/Gpu.h:62-81; roeStat, src/Gpu.cpp:311-327): beta = sd sqrt(6)/pi, miu = mean - gamma beta,
    Z = (x - miu) / beta."""
    import math
    n = len(values)
    if n == 0:
        return 0.0
    s = sum(float(v) for v in values)
    s2 = sum(float(v) * float(v) for v in values)
    sd = math.sqrt(max(0.0, n * s2 - s * s)) / n
    beta = sd * 0.779696801233676
    miu = s / n - beta * 0.577215664901533
    return (x - miu) / beta if beta > 0 else 0.0


def z_for_bpw(N, W, H, bpw, count=1, device=0, block=200, iters=2000, warmup=50):
    """The reference's Tune::zForBpw (src/tune.cpp:174-186) with its measureROE loop (Gpu.cpp:1276-1320:
    50 warm-up squarings, then 2,000 in blocks of 200): Z of the per-squaring round-off at
    E = prevPrime(N bpw) (count 1) or the `count` primes after N bpw, averaged."""
    import numpy as np
    import gpuowl_b200 as owl
    E = prev_prime(N * bpw) if count == 1 else next_prime(N * bpw)
    total = 0.0
    for _ in range(count):
        with owl.Plan(E, device=device, W=W, H=H) as p:
            b = p.alloc()
            p.writeIn(b, [3] + [0] * (p.nwords - 1))
            p.squareLoop(b, b, warmup)
            p.readROE()
            sample = []
            for _ in range(iters // block):
                p.squareLoop(b, b, block)
                sample.extend(float(v) for v in p.readROE())
        total += roe_z(sample)
        E = next_prime(E + 1)
    return total / count


# the plan's limit on bits per word (owl_plan_create accepts E / N <= 21)
BPW_CAP = 20.99


def max_bpw_z(N, W, H, guess, device=0, target=28.0, sample_size=5, verbose=True):
    """Tune::maxBpw (src/tune.cpp:106-172): bits per word at which the round-off Z is `target` (28).
    A search finds a bpw with Z in [31, 37] and one with Z in [20, 25], each re-measured on
    `sample_size` exponents; the result interpolates between the two. `guess` is where the search
    starts (the reference starts 9 steps below its table's value). The reference steps by a fixed
    estimate of dbpw/dZ tuned at 4M-7.5M; here the step comes from the points measured so far (a
    secant between the nearest points on either side of the band once it is bracketed), which also
    holds for the small FFTs, where Z changes faster with bpw."""
    import math
    step0 = 0.015 + (math.log2(N) - math.log2(4.0 * 1024 * 1024)) / \
        (math.log2(7.5 * 1024 * 1024) - math.log2(4.0 * 1024 * 1024)) * (0.012 - 0.015)
    step0 = min(max(step0, 0.005), 0.025)
    seen = []

    def z_at(bpw, count=1):
        z = z_for_bpw(N, W, H, bpw, count, device)
        if verbose:
            print("N=%-9d %-14s bpw %.3f  Z %.2f%s" % (N, spec(W, H), bpw, z, " (x%d)" % count if count > 1 else ""),
                  flush=True)
        if count == 1:
            seen.append((bpw, z))
        return z

    def search(bpw, lo, hi, aim):
        for _ in range(30):
            bpw = min(max(bpw, 8.0), BPW_CAP)
            z = z_at(bpw)
            if lo <= z <= hi:
                break
            safe = [p for p in seen if p[1] > aim]    # Z above the aim: bpw can grow
            risky = [p for p in seen if p[1] < aim]
            if safe and risky:
                a = max(safe)                          # the highest safe bpw
                b = min(risky)                         # the lowest risky bpw
                nxt = a[0] + (b[0] - a[0]) * (a[1] - aim) / (a[1] - b[1])
            else:
                # one side only: step by the local slope if two points exist, else by the default
                pts = sorted(seen)[-2:] if safe else sorted(seen)[:2]
                slope = (pts[1][0] - pts[0][0]) / (pts[0][1] - pts[1][1]) if len(pts) == 2 and pts[0][1] != pts[1][1] else 0
                slope = slope if slope > 0 else step0
                nxt = bpw + min(max((z - aim) * slope, -0.5), 0.5)
            if z > hi and bpw >= BPW_CAP:
                break                                  # safe up to the plan's limit
            bpw = nxt
        z = (z + (sample_size - 1) * z_at(bpw, sample_size - 1)) / sample_size
        return bpw, z

    bpw1, z1 = search(guess, 31.0, 37.0, 34.0)
    bpw2, z2 = search(bpw1 + 0.1, 20.0, 25.0, 22.0)
    if z1 == z2:
        return bpw2, (bpw1, z1), (bpw2, z2)
    return bpw2 + (bpw1 - bpw2) * (target - z2) / (z1 - z2), (bpw1, z1), (bpw2, z2)


def bpw_scan_z(shapes, device=0, verbose=True):
    """The max-bpw table by the reference's criterion (round-off Z = 28): {N: (W, H, max_bpw, points)}."""
    from gpuowl_b200 import build
    build.build()
    out = {}
    for (N, W, H) in shapes:
        import math
        guess = 19.2 - 0.3 * (math.log2(N) - 18.0) - 0.2  # a little below the library's default limit
        best, p1, p2 = max_bpw_z(N, W, H, guess, device, verbose=verbose)
        out[N] = (W, H, best, [p1, p2])
    return out


def write_bpw_z(table, out_txt):
    with open(out_txt, "w") as f:
        f.write("# max bits/word at round-off Z = 28 (the reference's Tune::maxBpw criterion), "
                "interpolated between a Z ~ 34 and a Z ~ 22 measurement\n")
        f.write("# N  spec  max_bpw  (bpw:Z bpw:Z)\n")
        for N in sorted(table):
            W, H, best, pts = table[N]
            f.write("%9d %14s %6.2f  %s\n" % (N, spec(W, H), best, " ".join("%.3f:%.2f" % p for p in pts)))


def bpw_scan(shapes, iters, limit=0.3, start=16.0, step=0.25, device=0, verbose=True):
    """The reference's BPW table (src/fftbpw.h, measured by its -ztune) for this library's FFTs:
    for each (N, W, H) the largest bits per word, on a `step` grid from `start`, whose max round-off
    over `iters` squarings stays below `limit`. Returns {N: (W, H, max_bpw, [(bpw, roe), ...])}."""
    from gpuowl_b200 import build
    build.build()
    out = {}
    for (N, W, H) in shapes:
        curve, best = [], None
        bpw = start
        while bpw <= 21.0:
            roe = roe_at(N, W, H, bpw, iters, device)
            curve.append((bpw, roe))
            if verbose:
                print("N=%-9d %-14s bpw %.2f  max ROE %.4f" % (N, spec(W, H), bpw, roe), flush=True)
            if roe >= limit:
                break
            best = bpw
            bpw += step
        out[N] = (W, H, best, curve)
    return out


def write_bpw(table, limit, iters, out_txt):
    with open(out_txt, "w") as f:
        f.write("# max bits/word with max ROE < %.2f over %d squarings of a random residue\n" % (limit, iters))
        f.write("# N  spec  max_bpw  (bpw:roe ...)\n")
        for N in sorted(table):
            W, H, best, curve = table[N]
            f.write("%9d %14s %6s  %s\n" % (N, spec(W, H), "%.2f" % best if best else "-",
                                           " ".join("%.2f:%.3f" % c for c in curve)))


def write(rows, max_bpw, out_txt, out_json):
    import gpuowl_b200 as owl
    lines, prev_cost = [], 0.0
    for N in sorted(rows):
        W, H, us, roe = rows[N][:4]
        cv = rows[N][5] if len(rows[N]) >= 6 else None
        cost = max(us, prev_cost)
        prev_cost = cost
        lines.append("%6.1f %14s # %u" % (cost, spec(W, H), int(N * max_bpw)) +
                     (" " + owl.COL_NAMES[cv] if cv in owl.COL_NAMES else ""))
    with open(out_txt, "w") as f:
        f.write("\n".join(lines) + "\n")
    with open(out_json, "w") as f:
        json.dump({str(N): list(v) for N, v in rows.items()}, f, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--min-lg", type=int, default=13)
    ap.add_argument("--max-lg", type=int, default=23)
    ap.add_argument("--iters", type=int, default=200)
    ap.add_argument("--bpw", type=float, default=18.0)
    ap.add_argument("--out", default="tune.txt")
    ap.add_argument("--json", default="tune.json")
    ap.add_argument("--five", action="store_true", help="also the 5 * 2^k FFT lengths")
    ap.add_argument("--bpw-scan", metavar="TUNE_JSON", help="measure the max bits/word of the shapes in TUNE_JSON")
    ap.add_argument("--roe-limit", type=float, default=0.3,
                    help="with --bpw-scan --criterion roe: the max round-off allowed")
    ap.add_argument("--criterion", default="z", choices=["z", "roe"],
                    help="with --bpw-scan: round-off Z = 28 (the reference's) or max round-off < --roe-limit")
    ap.add_argument("--shapes", metavar="WxH,...", help="per-pass times of these shapes (at 16 bits/word)")
    ap.add_argument("--split", type=int, nargs="?", const=1, default=0, metavar="FLAGS",
                    help="with --shapes: the split-precision form (1 column pass, 2 line pass, 3 both)")
    ap.add_argument("--variants", action="store_true",
                    help="with --shapes: time every column variant built for the shape's H")
    ap.add_argument("--no-variants", action="store_true", help="sweep: the shapes' default column variants only")
    a = ap.parse_args()
    if a.shapes:
        profile_shapes([tuple(int(v) for v in s.split("x")) for s in a.shapes.split(",")], a.iters,
                       split=a.split, variants=a.variants)
        return
    if a.bpw_scan:
        with open(a.bpw_scan) as f:
            t = json.load(f)
        shapes = [(int(N), v[0], v[1]) for N, v in t.items()
                  if (1 << a.min_lg) <= int(N) <= (1 << a.max_lg)]
        if a.criterion == "z":
            table = bpw_scan_z(sorted(shapes))
            write_bpw_z(table, a.out)
        else:
            table = bpw_scan(sorted(shapes), a.iters, a.roe_limit)
            write_bpw(table, a.roe_limit, a.iters, a.out)
        for N, (W, H, best, _) in table.items():
            if best and str(N) in t:
                t[str(N)] = list(t[str(N)][:4]) + [best] + list(t[str(N)][5:])
        with open(a.json, "w") as f:
            json.dump(t, f, indent=1)
        print(open(a.out).read())
        return
    rows = tune(a.min_lg, a.max_lg, a.iters, a.bpw, five=a.five, variants=not a.no_variants)
    write(rows, a.bpw, a.out, a.json)
    print(open(a.out).read())


if __name__ == "__main__":
    main()
