"""Command line front end, shaped like the reference's prpll options (src/Args.cpp):

    python -m gpuowl_b200 -prp E [-proof P] [-block B] [-dir D] [-device N] [-split [FLAGS]] [-tuned FILE]
    python -m gpuowl_b200 -ll E [-dir D] [-device N] [-tuned FILE]
    python -m gpuowl_b200 -verify FILE.proof [-device N]
    python -m gpuowl_b200 -work [-dir D] [-pool DIR] [-instance N] [-proof P]   # worktodo-N.txt loop
    python -m gpuowl_b200 -tune [-five]                                          # tune.txt

Results of -work go to <dir>/results-<instance>.txt as the reference's JSON lines. -split takes the
OWL_SPLIT_* flags (1 column pass, 2 line pass, 3 both; bare -split = 1). -tuned FILE (a tune.json of
-tune or gpuowl_b200.tune) picks each exponent's FFT split and column variant from that table, as the
reference picks its FFT from tune.txt.
"""
import argparse
import json
import sys

import gpuowl_b200 as owl


def main(argv=None):
    ap = argparse.ArgumentParser(prog="gpuowl_b200", prefix_chars="-")
    ap.add_argument("-prp", type=int)
    ap.add_argument("-ll", type=int)
    ap.add_argument("-verify")
    ap.add_argument("-work", action="store_true")
    ap.add_argument("-tune", action="store_true")
    ap.add_argument("-five", action="store_true")
    ap.add_argument("-proof", type=int, default=0)
    ap.add_argument("-block", type=int, default=1000)
    ap.add_argument("-dir", default=".")
    ap.add_argument("-pool")
    ap.add_argument("-instance", type=int, default=0)
    ap.add_argument("-device", type=int, default=0)
    ap.add_argument("-split", type=int, nargs="?", const=1, default=0,
                    help="split-precision form: 1 column pass (H = 2048, 2560), 2 line pass (W = 2048), 3 both")
    ap.add_argument("-tuned", help="tune.json: FFT split and column variant per FFT size")
    ap.add_argument("-verbose", action="store_true")
    a = ap.parse_args(argv)

    def shape(E):
        """(W, H, column variant) for E: the tuned table's when -tuned is given, else the library's."""
        if not a.tuned:
            return 0, 0, 0
        from gpuowl_b200 import tune
        N, W, H = owl.fft_choose(E, tune=a.tuned)
        return W, H, tune.tuned_variant(N, a.tuned)

    if a.prp:
        W, H, cv = shape(a.prp)
        r = owl.prp_run(a.prp, device=a.device, block=a.block, save_dir=a.dir, proof_power=a.proof, W=W, H=H,
                        split=a.split, verbose=a.verbose, column_variant=cv)
        print(json.dumps({k: v for k, v in r.items() if k != "checkpoints"}))
    elif a.ll:
        W, H, cv = shape(a.ll)
        r = owl.ll_run(a.ll, device=a.device, save_dir=a.dir, W=W, H=H, split=a.split, verbose=a.verbose,
                       column_variant=cv)
        print(json.dumps({k: v for k, v in r.items() if k != "checkpoints"}))
    elif a.verify:
        valid, prime = owl.proof_verify(a.verify, device=a.device)
        print(json.dumps({"proof": a.verify, "valid": valid, "probable_prime": prime}))
        return 0 if valid else 1
    elif a.work:
        while True:
            t = owl.worktodo_get(a.dir, a.instance, a.pool)
            if t is None:
                break
            W, H, cv = shape(t.exponent)
            print(owl.task_run(t, a.dir, a.instance, device=a.device, proof_power=a.proof, block=a.block, W=W, H=H,
                               split=a.split, column_variant=cv), flush=True)
    elif a.tune:
        from gpuowl_b200 import tune
        rows = tune.tune(13, 25, 200, five=a.five)
        tune.write(rows, 18.0, "tune.txt", "tune.json")
        print(open("tune.txt").read())
    else:
        ap.print_help()
    return 0


if __name__ == "__main__":
    sys.exit(main())
