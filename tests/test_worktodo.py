"""The work layer (reference src/Worktodo.cpp, src/Task.cpp): worktodo lines, the pooled work
queue, task results as JSON lines, CERT squarings, and the MD5 reported for proofs."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import random_words


@pytest.fixture(scope="module")
def lib():
    import gpuowl_b200 as g
    from gpuowl_b200 import build as b
    b.build()
    g.load()
    return g


# line formats from the comments of src/Worktodo.cpp:23-25, and lines the parser ignores
@pytest.mark.parametrize("line,want", [
    ("PRP=FEEE9DCD59A0855711265C1165C4C693,1,2,124647911,-1,77,0",
     ("PRP", 124647911, 0, "FEEE9DCD59A0855711265C1165C4C693")),
    ("DoubleCheck=E0F583710728343C61643028FBDBA0FB,70198703,75,1",
     ("LL", 70198703, 0, "E0F583710728343C61643028FBDBA0FB")),
    ("Cert=B2EE67DC0A514753E488794C9DD6F6BD,1,2,82997591,-1,162105",
     ("CERT", 82997591, 162105, "B2EE67DC0A514753E488794C9DD6F6BD")),
    ("PRP=N/A,1,2,86243,-1,70,0", ("PRP", 86243, 0, "")),
    ("Test=86243", ("LL", 86243, 0, "")),
    ("PRPDC=86249\n", ("PRP", 86249, 0, "")),
    ("# a comment", None),
    ("Factor=12345,70,71", None),
    ("PRP=999", None),
    ("Cert=B2EE67DC0A514753E488794C9DD6F6BD,1,2,82997591,-1,50", None),
    ("", None),
])
def test_worktodo_parse(lib, line, want):
    t = lib.worktodo_parse(line)
    if want is None:
        assert t is None
    else:
        d = t.as_dict()
        assert (d["kind"], d["exponent"], d["squarings"], d["aid"]) == want
        assert d["line"] == line.rstrip("\n")


def test_worktodo_best_and_pool(lib, tmp_path):
    local, master = tmp_path / "w", tmp_path / "m"
    local.mkdir()
    master.mkdir()
    (master / "worktodo.txt").write_text("PRP=500009\nTest=216091\nCert=B2EE67DC0A514753E488794C9DD6F6BD,1,2,110503,-1,5000\n")
    # empty local file: the best global task (a CERT first) moves to worktodo-3.txt
    t = lib.worktodo_get(local, 3, master)
    assert t.as_dict()["kind"] == "CERT" and t.exponent == 110503
    assert "Cert=" in (local / "worktodo-3.txt").read_text()
    assert "Cert=" not in (master / "worktodo.txt").read_text()
    # the local file now wins
    assert lib.worktodo_get(local, 3, master).exponent == 110503
    (local / "worktodo-3.txt").write_text("PRP=500009\nTest=216091\n")
    assert lib.worktodo_get(local, 3).exponent == 216091
    assert lib.worktodo_get(tmp_path / "nowhere", 0) is None


def test_file_md5(lib, tmp_path):
    rng = np.random.default_rng(3)
    for n in (0, 55, 56, 63, 64, 65, 100000):
        p = tmp_path / ("f%d" % n)
        data = rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()
        p.write_bytes(data)
        assert lib.file_md5(p) == hashlib.md5(data).hexdigest()


def _int(words):
    return int.from_bytes(np.asarray(words, dtype=np.uint32).tobytes(), "little")


@pytest.mark.gpu
def test_cert_task_matches_python(owl, tmp_path):
    E, sq = 86243, 3000
    M = (1 << E) - 1
    nb = (E - 1) // 8 + 1
    start = _int(random_words(E, 9))
    (tmp_path / ("M%d.cert" % E)).write_bytes(start.to_bytes(nb, "little"))
    (tmp_path / "worktodo-0.txt").write_text("Cert=B2EE67DC0A514753E488794C9DD6F6BD,1,2,%d,-1,%d\n" % (E, sq))
    t = owl.worktodo_get(tmp_path, 0)
    line = json.loads(owl.task_run(t, tmp_path, 0))
    x = pow(start, 1 << sq, M)
    digest = hashlib.sha3_256(x.to_bytes(nb, "little")).digest()
    # the digest printed as one little-endian 256-bit number, most significant digit first
    assert line["sha3-hash"] == int.from_bytes(digest, "little").to_bytes(32, "big").hex()
    assert line["worktype"] == "Cert" and line["squarings"] == sq and line["exponent"] == E
    assert not (tmp_path / ("M%d.cert" % E)).exists()
    assert (tmp_path / "worktodo-0.txt").read_text() == ""
    assert json.loads((tmp_path / "results-0.txt").read_text().splitlines()[-1]) == line


@pytest.mark.gpu
def test_prp_and_ll_tasks_write_results(owl, tmp_path):
    (tmp_path / "worktodo-1.txt").write_text("PRP=N/A,1,2,86243,-1,70,0\nDoubleCheck=86249\n")
    t = owl.worktodo_get(tmp_path, 1)
    assert t.exponent == 86243
    prp = json.loads(owl.task_run(t, tmp_path, 1, proof_power=3, block=500))
    assert prp["status"] == "P" and prp["worktype"] == "PRP-3" and prp["residue-type"] == 1
    assert prp["res64"] == "0000000000000001" and prp["errors"] == {"gerbicz": 0}
    pf = tmp_path / "proof" / "86243-3.proof"
    assert prp["proof"] == {"version": 1, "power": 3, "hashsize": 64,
                            "md5": hashlib.md5(pf.read_bytes()).hexdigest()}
    t = owl.worktodo_get(tmp_path, 1)
    assert t.exponent == 86249 and t.as_dict()["kind"] == "LL"
    ll = json.loads(owl.task_run(t, tmp_path, 1))
    assert ll["status"] == "C" and ll["worktype"] == "LL" and ll["fft-length"] > 0
    assert owl.worktodo_get(tmp_path, 1) is None
    assert len((tmp_path / "results-1.txt").read_text().splitlines()) == 2
