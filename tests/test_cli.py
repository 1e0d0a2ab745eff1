"""The command-line front end (python -m gpuowl_b200)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def _run(args, cwd=None):
    return subprocess.run([sys.executable, "-m", "gpuowl_b200"] + args, capture_output=True, text=True,
                          cwd=cwd or ROOT, timeout=600, env=dict(os.environ, PYTHONPATH=ROOT))


def test_cli_help():
    r = _run([])
    assert r.returncode == 0 and "-prp" in r.stdout and "-work" in r.stdout


@pytest.mark.gpu
def test_cli_prp_with_proof_and_verify(owl, tmp_path):
    r = _run(["-prp", "86243", "-proof", "2", "-block", "500", "-dir", str(tmp_path)])
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["is_prime"] and out["finished"] and out["proof_power"] == 2
    v = _run(["-verify", out["proof_file"]])
    assert v.returncode == 0 and json.loads(v.stdout.strip().splitlines()[-1])["probable_prime"]


@pytest.mark.gpu
def test_cli_worktodo_loop(owl, tmp_path):
    (tmp_path / "worktodo-0.txt").write_text("Test=86243\nPRP=86249\n")
    r = _run(["-work", "-dir", str(tmp_path)])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in (tmp_path / "results-0.txt").read_text().splitlines()]
    assert [(l["exponent"], l["worktype"], l["status"]) for l in lines] == [(86243, "LL", "P"), (86249, "PRP-3", "C")]
    assert (tmp_path / "worktodo-0.txt").read_text() == ""


def test_cli_help_lists_the_split_and_tuned_options():
    r = _run([])
    assert r.returncode == 0
    for opt in ("-ll", "-verify", "-tune", "-split", "-tuned", "-proof"):
        assert opt in r.stdout


@pytest.mark.gpu
def test_cli_prp_with_the_tuned_table_and_split_flags(owl, tmp_path):
    """M86243 is prime: -prp with the committed tune table (its split and column variant for the 8K
    FFT) says so, and so does -ll; -split 2 on a shape without a split line pass is refused."""
    table = os.path.join(ROOT, "gpuowl_b200", "tune_b200.json")
    r = _run(["-prp", "86243", "-dir", str(tmp_path), "-tuned", table])
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["is_prime"] and out["finished"] and out["n_errors"] == 0
    r = _run(["-ll", "86243", "-dir", str(tmp_path / "ll"), "-tuned", table])
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1])["is_prime"]
    r = _run(["-prp", "86243", "-dir", str(tmp_path / "split"), "-split", "2"])
    assert r.returncode != 0 and "split" in r.stderr
