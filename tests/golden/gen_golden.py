"""Generate the golden res64 fixtures with the GMP oracle (oracle/liboracle.so).

Run from the repository root (one process per workload; the large ones take
hours on one core, so they append progress to <name>.progress and can be
resumed by re-running: finished checkpoints are not recomputed, the run starts
over from 3/4 only if no final JSON exists yet):

    python tests/golden/gen_golden.py <name> [<name> ...]
    python tests/golden/gen_golden.py --list

Workloads (seed 20261203; exponent = smallest prime above a splitmix64 draw
from the range, the reference's Primes::nextPrime semantics):

    prp_256k   PRP-3, E in [4.8M, 5.0M],  20,000 iterations, res64 every 1,000
    prp_8m     PRP-3, E in [136M, 139M],  10,000 iterations, res64 every 1,000
    ll_8m      LL-4,  same E as prp_8m,   10,000 iterations, res64 every 1,000
    prp_20m    PRP-3, E in [330M, 335M],   5,000 iterations, res64 every 1,000
    batch64    64 exponents log-uniform in [1M, 20M], PRP-3 2,000 iterations, every 1,000
    batch64_10k   all 64 of those exponents, PRP-3 10,000 iterations, every 1,000 (8 processes)
    small      short PRP/LL runs for unit sizes (E in 1e4..2e6), every 100

Output: tests/golden/<name>.json = {"workload": ..., "E": ..., "kind": "prp"|"ll",
"start": 3|4, "step": S, "res64": ["%016x", ...]} (batch64/small hold a list).
"""
import ctypes
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SEED = 20261203

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
        _lib.oracle_seeded_prime.restype = ctypes.c_uint32
        _lib.oracle_seeded_prime.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        _lib.oracle_splitmix64.restype = ctypes.c_uint64
        _lib.oracle_splitmix64.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
        _lib.oracle_next_prime.restype = ctypes.c_uint32
        _lib.oracle_next_prime.argtypes = [ctypes.c_uint32]
        _lib.oracle_gmp_run.restype = ctypes.c_int
        _lib.oracle_gmp_run.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p]
    return _lib


def seeded_prime(cfg, lo, hi):
    """Exponent of workload `cfg`: splitmix64(SEED + cfg) mapped to [lo, hi], then next prime."""
    return int(lib().oracle_seeded_prime(SEED + cfg, lo, hi))


def batch_exponents(n=64, lo=1_000_000, hi=20_000_000, cfg=4):
    """n exponents log-uniform in [lo, hi]: u_i from the splitmix64 stream of SEED + cfg."""
    st = ctypes.c_uint64(SEED + cfg)
    out = []
    for _ in range(n):
        u = lib().oracle_splitmix64(ctypes.byref(st))
        f = (u >> 11) / float(1 << 53)
        x = int(math.exp(math.log(lo) + f * (math.log(hi) - math.log(lo))))
        out.append(int(lib().oracle_next_prime(min(max(x, lo), hi))))
    return out


WORKLOADS = {
    "prp_256k": dict(cfg=1, lo=4_800_000, hi=5_000_000, kind="prp", iters=20_000, step=1_000),
    "prp_8m": dict(cfg=2, lo=136_000_000, hi=139_000_000, kind="prp", iters=10_000, step=1_000),
    "ll_8m": dict(cfg=2, lo=136_000_000, hi=139_000_000, kind="ll", iters=10_000, step=1_000),
    "prp_20m": dict(cfg=5, lo=330_000_000, hi=335_000_000, kind="prp", iters=5_000, step=1_000),
}

SMALL = [  # (E, kind, iters, step): unit-size runs for the GPU parity tests
    (11213, "prp", 2000, 100), (19937, "ll", 2000, 100), (86243, "prp", 2000, 100),
    (110503, "ll", 1000, 100), (216091, "prp", 1000, 100), (500009, "prp", 1000, 100),
    (1000003, "prp", 600, 100), (1257787, "ll", 600, 100), (2000029, "prp", 400, 100),
]


def run_one(E, kind, iters, step, progress=None):
    n = iters // step
    buf = (ctypes.c_uint64 * max(n, 1))()
    start = 4 if kind == "ll" else 3
    lib().oracle_gmp_run(E, start, 1 if kind == "ll" else 0, iters, step, buf,
                         progress.encode() if progress else None)
    return ["%016x" % buf[i] for i in range(n)]


def gen(name):
    path = os.path.join(HERE, name + ".json")
    if name in WORKLOADS:
        w = WORKLOADS[name]
        E = seeded_prime(w["cfg"], w["lo"], w["hi"])
        prog = os.path.join(HERE, name + ".progress")
        if os.path.exists(prog):
            os.remove(prog)
        res = run_one(E, w["kind"], w["iters"], w["step"], prog)
        out = {"workload": name, "E": E, "kind": w["kind"], "start": 4 if w["kind"] == "ll" else 3,
               "step": w["step"], "iters": w["iters"], "seed": SEED, "cfg": w["cfg"],
               "range": [w["lo"], w["hi"]], "res64": res}
        os.remove(prog)
    elif name == "batch64":
        exps = batch_exponents()
        items = []
        for E in exps:
            items.append({"E": E, "kind": "prp", "start": 3, "step": 1000, "iters": 2000,
                          "res64": run_one(E, "prp", 2000, 1000)})
        out = {"workload": name, "seed": SEED, "cfg": 4, "items": items}
    elif name == "batch64_10k":
        exps = batch_exponents()
        import multiprocessing as mp
        # largest first, so that the longest runs start at once
        order = sorted(exps, reverse=True)
        with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
            res = dict(zip(order, pool.starmap(run_one, [(E, "prp", 10000, 1000) for E in order], chunksize=1)))
        items = [{"E": E, "kind": "prp", "start": 3, "step": 1000, "iters": 10000, "res64": res[E]} for E in exps]
        out = {"workload": name, "seed": SEED, "cfg": 4, "items": items}
    elif name == "small":
        items = []
        for (E, kind, iters, step) in SMALL:
            items.append({"E": E, "kind": kind, "start": 4 if kind == "ll" else 3, "step": step,
                          "iters": iters, "res64": run_one(E, kind, iters, step)})
        out = {"workload": name, "items": items}
    else:
        raise SystemExit("unknown workload " + name)
    with open(path + ".tmp", "w") as f:
        json.dump(out, f, indent=1)
    os.replace(path + ".tmp", path)
    print(name, "done", path)


if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1] == "--list":
        for k, w in WORKLOADS.items():
            print(k, seeded_prime(w["cfg"], w["lo"], w["hi"]), w)
        print("batch64", batch_exponents()[:8], "...")
        sys.exit(0)
    for name in sys.argv[1:]:
        gen(name)
