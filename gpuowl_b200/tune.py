"""Autotuner for FFT shapes (replaces the reference's -tune, src/tune.cpp:106-186, which times
each FFT with Gpu::timePRP and writes tune.txt).

    python -m gpuowl_b200.tune [--min-lg 13] [--max-lg 23] [--iters 200] [--out tune.txt]

For every FFT size N = 2^lg, and N = 5 * 2^(lg-3) with --five, it times each W x H split the library
supports (W a power of two in [64, 4096]; H a power of two in [64, 4096] with H/W in {1/2, 1, 2, 4},
or H in {640, 1280, 2560}) with owl_profile_square (device time of the two passes per
squaring, at an exponent of 18 bits per word), keeps the fastest split, and records its max
round-off. Output:
  - tune.txt in the reference's format, "%6.1f %14s # %u" = microseconds per iteration, shape,
    largest exponent (src/TuneEntry.cpp:94-105), rows in increasing cost and exponent;
  - tune.json, {"N": [W, H, us_per_iter, max_roe]}, read by fft_choose(..., tune=path).
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


def tune(min_lg, max_lg, iters, max_bpw=18.0, device=0, verbose=True, five=False):
    import numpy as np
    import gpuowl_b200 as owl
    from gpuowl_b200 import build
    build.build()
    rows = {}
    for N in sizes(min_lg, max_lg, five):
        E = next_odd_exponent(N * max_bpw * 0.98)
        best = None
        for (W, H) in candidates(N):
            with owl.Plan(E, device=device, W=W, H=H) as p:
                b = p.alloc()
                rng = np.random.default_rng(N)
                w = rng.integers(0, 2 ** 32, size=p.nwords, dtype=np.uint64).astype(np.uint32)
                if E % 32:
                    w[-1] &= (1 << (E % 32)) - 1
                p.writeIn(b, w)
                p.profile_square(b, 20)  # warm
                p.readROE()
                prof = p.profile_square(b, iters)
                us = 1e3 * (prof["pass2"][0] + prof["pass1"][0] + prof["edge"][0]) / iters
                roe = float(p.readROE().max())
            if verbose:
                print("N=%-9d %-14s %8.2f us/iter  max ROE %.4f" % (N, spec(W, H), us, roe), flush=True)
            if best is None or us < best[2]:
                best = (W, H, us, roe)
        if best:
            rows[N] = best
    return rows


def profile_shapes(shapes, iters, bpw=16.0, device=0, split=False):
    """Per-kernel device time of `iters` squarings on each W x H shape (the -time profile per shape):
    E is the first odd number above N * bpw, the residue random; one untimed block first. With
    `split` the column pass runs in the split-precision form (H = 2048 only)."""
    import numpy as np
    import gpuowl_b200 as owl
    from gpuowl_b200 import build
    build.build()
    rows = []
    for (W, H) in shapes:
        N = 2 * W * H
        E = next_odd_exponent(N * bpw)
        with owl.Plan(E, device=device, W=W, H=H, split=split) as p:
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
        us2 = 1e3 * prof["pass2"][0] / prof["pass2"][1]
        us1 = 1e3 * prof["pass1"][0] / prof["pass1"][1]
        total = 1e3 * (prof["pass2"][0] + prof["pass1"][0] + prof["edge"][0]) / iters
        rows.append((N, W, H, total, us2, us1, roe))
        print("N=%-9d %-14s %8.2f us/iter  column pass %7.2f us  line pass %7.2f us  max ROE %.4f"
              % (N, spec(W, H), total, us2, us1, roe), flush=True)
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
    lines, prev_cost = [], 0.0
    for N in sorted(rows):
        W, H, us, roe = rows[N]
        cost = max(us, prev_cost)
        prev_cost = cost
        lines.append("%6.1f %14s # %u" % (cost, spec(W, H), int(N * max_bpw)))
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
    ap.add_argument("--roe-limit", type=float, default=0.3)
    ap.add_argument("--shapes", metavar="WxH,...", help="per-pass times of these shapes (at 16 bits/word)")
    ap.add_argument("--split", action="store_true", help="with --shapes: the split-precision column pass")
    a = ap.parse_args()
    if a.shapes:
        profile_shapes([tuple(int(v) for v in s.split("x")) for s in a.shapes.split(",")], a.iters,
                       split=a.split)
        return
    if a.bpw_scan:
        with open(a.bpw_scan) as f:
            t = json.load(f)
        shapes = [(int(N), v[0], v[1]) for N, v in t.items()
                  if (1 << a.min_lg) <= int(N) <= (1 << a.max_lg)]
        table = bpw_scan(sorted(shapes), a.iters, a.roe_limit)
        write_bpw(table, a.roe_limit, a.iters, a.out)
        for N, (W, H, best, _) in table.items():
            if best and str(N) in t:
                t[str(N)] = list(t[str(N)][:4]) + [best]
        with open(a.json, "w") as f:
            json.dump(t, f, indent=1)
        print(open(a.out).read())
        return
    rows = tune(a.min_lg, a.max_lg, a.iters, a.bpw, five=a.five)
    write(rows, a.bpw, a.out, a.json)
    print(open(a.out).read())


if __name__ == "__main__":
    main()
