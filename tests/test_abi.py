"""The C ABI (include/owl.h): the library builds for sm_100a, loads without a GPU, exports every
declared entry point, and its no-device paths fail cleanly."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in ("owl.h", "owl_host.h")]


def declared():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        names |= set(re.findall(r"^\s*(?:int|const char\*|void|uint32_t|uint64_t)\s+(owl_\w+)\s*\(", src, re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from gpuowl_b200 import build
    build.build()
    import gpuowl_b200 as g
    return g.load()


def test_header_declares_the_boundary():
    names = declared()
    for must in ("owl_plan_create", "owl_square", "owl_modmul", "owl_res64", "owl_read_words",
                 "owl_write_words", "owl_is_equal", "owl_read_roe", "owl_probe_wait_timeout", "owl_exp_mul",
                 "owl_plan_set_split", "owl_prp_run", "owl_ll_run", "owl_proof_verify", "owl_task_run",
                 "owl_cert_run", "owl_worktodo_get", "owl_sha3_256", "owl_crc32"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "gpuowl_b200", "libowl.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s+(owl_\w+)$", out, re.M))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


def test_build_targets_sm100a_only():
    from gpuowl_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_abi_version_and_errors(lib):
    assert lib.owl_abi_version() == 1
    assert lib.owl_error_string(-4) == b"device wait timeout"
    # null / bogus arguments fail with a status, never a crash
    assert lib.owl_plan_destroy(None) == -1
    assert lib.owl_square(None, None, None, 1, 0) == -1


def test_fft_choice_matches_the_configs(lib):
    import gpuowl_b200 as g
    assert g.fft_choose(4989349) == (262144, 256, 512)        # 256K (reference 256:2:256)
    assert g.fft_choose(136181029) == (8388608, 2048, 2048)   # 8M  (reference 1K:8:512)
    assert g.fft_choose(333000017) == (20971520, 4096, 2560)  # 20M = 5 * 2^22 (reference 4K:5:512)
    assert g.fft_choose(40000003) == (5 << 19, 1024, 1280)   # 2.5M, between 2M and 4M
    with pytest.raises(g.OwlError):
        g.fft_choose(3_000_000_000)


def test_plan_without_device_reports_nodev(lib):
    import gpuowl_b200 as g
    if g.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(g.OwlError) as e:
        g.Plan(86243)
    assert e.value.status == -5


def test_tuner_shape_grammar_and_candidates():
    from gpuowl_b200 import tune
    assert tune.spec(2048, 2048) == "2K:2:1K"
    assert tune.spec(256, 512) == "256:2:256"
    assert tune.spec(64, 64) == "64:1:64"
    assert tune.spec(4096, 2560) == "4K:5:512"
    assert (2048, 2048) in tune.candidates(1 << 23) and (1024, 4096) in tune.candidates(1 << 23)
    assert (4096, 2560) in tune.candidates(5 << 22)
    for N in tune.sizes(13, 25, five=True):
        for (w, h) in tune.candidates(N):
            assert 2 * w * h == N


def test_tune_file_format(tmp_path):
    from gpuowl_b200 import tune
    rows = {1 << 18: (256, 512, 21.3, 0.1), 1 << 23: (2048, 2048, 117.0, 0.03)}
    tune.write(rows, 18.0, tmp_path / "tune.txt", tmp_path / "tune.json")
    lines = open(tmp_path / "tune.txt").read().splitlines()
    assert lines[0] == "%6.1f %14s # %u" % (21.3, "256:2:256", 4718592)
    assert lines[1].split()[1] == "2K:2:1K"


def test_fft_choose_with_measured_bpw_table(lib, tmp_path):
    """With a tune file that carries measured max bits/word, the smallest FFT whose limit covers E
    is chosen (reference FFTConfig::bestFit over fftbpw.h)."""
    import json
    import gpuowl_b200 as g
    t = {str(1 << 23): [2048, 2048, 114.2, 0.15, 18.0], str(5 << 22): [4096, 2560, 391.1, 0.24, 17.75],
         str(1 << 24): [4096, 2048, 259.8, 0.22, 17.75]}
    p = tmp_path / "tune.json"
    p.write_text(json.dumps(t))
    assert g.fft_choose(150000001, tune=str(p)) == (1 << 23, 2048, 2048)     # 17.9 bits/word
    assert g.fft_choose(152000001, tune=str(p)) == (1 << 24, 4096, 2048)     # 18.1 > 18.0 at 8M
    assert g.fft_choose(333000017, tune=str(p)) == (5 << 22, 4096, 2560)     # 19.8 at 16M, 15.9 at 20M
    # an exponent below 8 bits/word of every measured size falls back to the library's size and
    # takes that size's tuned split: M86243 on the 8K FFT of the committed table
    committed = os.path.join(ROOT, "gpuowl_b200", "tune_b200.json")
    assert g.fft_choose(86243, tune=committed) == (8192, 64, 64)
