"""The command line front end (python -m gpuowl_b200, shaped like the reference's prpll options)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def run_cli(*args, timeout=600):
    r = subprocess.run([sys.executable, "-m", "gpuowl_b200"] + [str(a) for a in args], cwd=ROOT,
                       capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout, r.stderr


def test_cli_help_lists_the_options():
    rc, out, _ = run_cli()
    assert rc == 0
    for opt in ("-prp", "-ll", "-verify", "-work", "-tune", "-split", "-tuned", "-proof"):
        assert opt in out


@pytest.mark.gpu
def test_cli_prp_with_the_tuned_table_and_split_flags(tmp_path):
    """M86243 is prime: -prp with the committed tune table (its split and column variant for the 8K
    FFT) says so, and so does -ll; -split 2 on a shape without a split line pass is refused."""
    table = os.path.join(ROOT, "gpuowl_b200", "tune_b200.json")
    rc, out, err = run_cli("-prp", 86243, "-dir", tmp_path, "-tuned", table)
    assert rc == 0, err[-2000:]
    r = json.loads(out.strip().splitlines()[-1])
    assert r["is_prime"] and r["finished"] and r["n_errors"] == 0
    rc, out, err = run_cli("-ll", 86243, "-dir", tmp_path / "ll", "-tuned", table)
    assert rc == 0, err[-2000:]
    assert json.loads(out.strip().splitlines()[-1])["is_prime"]
    rc, out, err = run_cli("-prp", 86243, "-dir", tmp_path / "split", "-split", 2)
    assert rc != 0 and "split" in err
