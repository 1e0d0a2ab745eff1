"""CPU run of libowl's kernel source (tests/emu, AddressSanitizer build) against GMP.

The emulator compiles gpuowl_b200/csrc/owl_kernels.cuh unchanged as host C++;
each CUDA thread is a host thread. This checks index arithmetic, the carry
chain and the numerics at small FFT sizes before any GPU run, and ASan
flags every out-of-bounds access.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, random_words, small_words

EMU_DIR = os.path.join(ROOT, "tests", "emu")
CSRC = os.path.join(ROOT, "gpuowl_b200", "csrc")
EXE = os.path.join(ROOT, "tests", "emu", "owl_emu")


@pytest.fixture(scope="module")
def emu():
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    srcs = [os.path.join(EMU_DIR, f) for f in ("emu_main.cpp", "owl_emu_rt.hpp")] + \
        [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".inc", ".hpp"))]
    if not os.path.exists(EXE) or any(os.path.getmtime(s) > os.path.getmtime(EXE) for s in srcs):
        cmd = ["g++", "-std=c++20", "-O1", "-g", "-fsanitize=address", "-fno-omit-frame-pointer",
               "-DOWL_EMU", "-I", CSRC, "-I", EMU_DIR, "-o", EXE, os.path.join(EMU_DIR, "emu_main.cpp"),
               "-lpthread"]
        subprocess.run(cmd, check=True, capture_output=True)
    return EXE


def run(exe, *args, **extra_env):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", **extra_env)
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, (r.stdout[-1000:], r.stderr[-4000:])
    lines = r.stdout.strip().split("\n")
    roe = float(lines[0].split()[1])
    return roe, np.array([int(x, 16) for x in lines[1].split()], dtype=np.uint32)


@pytest.mark.parametrize("E,W,H,n,flags", [
    (86243, 64, 64, 40, 0),       # PRP from 3
    (86243, 64, 64, 40, 2),       # LL from 4
    (110503, 64, 64, 30, 1),      # MUL3 on the last step
    (500009, 128, 128, 24, 0),    # radix-16 first stages, two-level twiddles
    (1300021, 64, 640, 4, 2),     # H = 5 * 128: radix-5 middle stage of the column FFT, LL
    (4456451, 2048, 64, 3, 0),    # the 8M shape's line pass (2048 points, 16 x 16 x 8) on 64 lines
])
def test_emulated_square_matches_gmp(emu, oracle, E, W, H, n, flags):
    roe, got = run(emu, "square", E, W, H, n, flags, 0)
    ll = bool(flags & 2)
    want = oracle.gmp_square(E, small_words(E, 4 if ll else 3), n, ll=ll)
    if flags & 1:
        want = oracle.gmp_mul(E, want, small_words(E, 3))
    assert np.array_equal(got, want)
    assert roe < 0.1


@pytest.mark.parametrize("mul3", [0, 1])
def test_emulated_modmul_matches_gmp(emu, oracle, mul3):
    E = 110503
    roe, got = run(emu, "modmul", E, 64, 64, mul3, 11, 22)
    want = oracle.gmp_mul(E, random_words(E, 11), random_words(E, 22), mul3=bool(mul3))
    assert np.array_equal(got, want)


def splitmix_words(E, seed):
    """The emulator's random start (splitmix64 stream, one word per draw, top word masked to E bits)."""
    m = (1 << 64) - 1
    s, out = seed, []
    for _ in range((E - 1) // 32 + 1):
        s = (s + 0x9e3779b97f4a7c15) & m
        z = s
        z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & m
        z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & m
        out.append((z ^ (z >> 31)) & 0xffffffff)
    w = np.array(out, dtype=np.uint32)
    if E % 32:
        w[-1] &= (1 << (E % 32)) - 1
    return w


@pytest.mark.parametrize("E,W,H,n,seed", [
    (1300021, 64, 640, 3, 7),     # 5 * 2^14 words, radix plan 16 * 5 * 8
    (2500009, 64, 1280, 2, 9),    # 5 * 2^15 words, radix plan 16 * 2 * 5 * 8
    (5600027, 64, 2560, 2, 11),   # 5 * 2^16 words, radix plan 16 * 4 * 5 * 8 (the 20M column FFT)
])
def test_emulated_radix5_random_start(emu, oracle, E, W, H, n, seed):
    roe, got = run(emu, "square", E, W, H, n, 0, seed)
    want = oracle.gmp_square(E, splitmix_words(E, seed), n)
    assert np.array_equal(got, want)
    assert 0 < roe < 0.1


@pytest.mark.parametrize("E,W,H", [(4700021, 64, 2048), (5600027, 64, 2560), (4500007, 2048, 64)])
@pytest.mark.parametrize("mode", ["square", "modmul"])
def test_emulated_split_precision_column_pass(emu, oracle, mode, E, W, H):
    """The split-precision passes on the emulated tensor cores (descriptor decoding, digit planes,
    accumulators): the 32-point GEMM stage of 2048-point columns, the 40-point one of 2560-point
    columns (K padded to 96 bytes in two panels, outputs in chunks of 32, 32 and 16 values), and the
    16-point one of 2048-point lines (the line pass's, two M = 128 tiles, no-swizzle operands)."""
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", OWL_EMU_SPLIT="3")
    args = ["square", E, W, H, 2, 0, 7] if mode == "square" else ["modmul", E, W, H, 1, 11, 22]
    r = subprocess.run([emu] + [str(a) for a in args], capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, (r.stdout[-1000:], r.stderr[-4000:])
    lines = r.stdout.strip().split("\n")
    got = np.array([int(x, 16) for x in lines[1].split()], dtype=np.uint32)
    if mode == "square":
        want = oracle.gmp_square(E, splitmix_words(E, 7), 2)
    else:
        want = oracle.gmp_mul(E, splitmix_words(E, 11), splitmix_words(E, 22), mul3=True)
    assert np.array_equal(got, want)
    assert 0 < float(lines[0].split()[1]) < 0.1


@pytest.mark.parametrize("nb,seed", [(1, 1), (17, 2), (256, 3), (257, 4), (8192, 5), (20480, 6)])
def test_emulated_pack_chain(emu, nb, seed):
    """The block-carry chain of the word conversion (one CTA: per-thread runs of blocks, a scan of
    the runs, then each run walked with its carry in) against its serial definition."""
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1")
    r = subprocess.run([emu, "chain", str(nb), str(seed)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0 and r.stdout.strip() == "chain ok", (r.stdout[-500:], r.stderr[-2000:])


@pytest.mark.parametrize("E,N,pattern", [(216091, 16384, p) for p in range(6)] + [(327691, 20480, 2)])
def test_emulated_device_expand_compact(emu, E, N, pattern):
    """owl_pack.cuh kernels against owl_words.hpp (3, 2^E-1, an all-propagating carry, 0, 2^E-2, random)."""
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1")
    r = subprocess.run([emu, "pack", str(E), str(N), str(pattern)], capture_output=True, text=True, timeout=600,
                       env=env)
    assert r.returncode == 0 and "pack ok" in r.stdout, (r.stdout[-500:], r.stderr[-2000:])


@pytest.mark.parametrize("E,W,H,n,flags", [(86243, 64, 64, 40, 0), (500009, 128, 128, 24, 2)])
def test_emulated_square_without_roe_matches_gmp(emu, oracle, E, W, H, n, flags):
    """The fused line pass built without the round-off measurement (OWL_SQ_NO_ROE) gives the same
    words."""
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", OWL_EMU_NO_ROE="1")
    r = subprocess.run([emu, "square", str(E), str(W), str(H), str(n), str(flags), "0"], capture_output=True,
                       text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.array([int(x, 16) for x in r.stdout.strip().split("\n")[1].split()], dtype=np.uint32)
    start = np.zeros((E - 1) // 32 + 1, dtype=np.uint32)
    start[0] = 4 if flags & 2 else 3
    assert np.array_equal(got, oracle.gmp_square(E, start, n, ll=bool(flags & 2)))


@pytest.mark.parametrize("E,W,H,n,variant", [
    (86243, 64, 64, 12, 2),       # 8 values a thread: plan 8 * 2 * 4
    (1300021, 64, 640, 3, 2),     # 8 values a thread: plan 8 * 4 * 5 * 4
    (2500009, 64, 1280, 2, 2),    # 8 values a thread: plan 8 * 8 * 5 * 4
    (4500007, 64, 2048, 2, 2),    # 8 values a thread: plan 8 * 8 * 8 * 4
    (5600027, 64, 2560, 2, 3),    # 16 values a thread, the two-CTA launch bounds
])
def test_emulated_column_variants_match_gmp(emu, oracle, E, W, H, n, variant):
    """The column pass's tile variants (owl_plan_set_column_variant) from a random start."""
    roe, got = run(emu, "square", E, W, H, n, 0, 5, OWL_EMU_COL=str(variant))
    want = oracle.gmp_square(E, splitmix_words(E, 5), n)
    assert np.array_equal(got, want)
    assert roe < 0.1


@pytest.mark.parametrize("E,W,H,n,flags", [
    (1300021, 64, 640, 3, 0),     # 8-thread line-group CTAs
    (1000003, 128, 256, 6, 2),    # 16-thread CTAs, LL
    (1999993, 256, 256, 4, 0),    # 32-thread CTAs
])
def test_emulated_grouped_line_pass(emu, oracle, E, W, H, n, flags):
    """The batch's grouped line-pass kernel (k_pass1_group, here with a group of one plan) from a
    random start."""
    ll = bool(flags & 2)
    roe, got = run(emu, "square", E, W, H, n, flags, 9, OWL_EMU_GROUP="1")
    want = oracle.gmp_square(E, splitmix_words(E, 9), n, ll=ll)
    assert np.array_equal(got, want)
    assert roe < 0.1


@pytest.mark.parametrize("E,W,H,n,flags", [
    (1999993, 1024, 64, 6, 0),    # 128-thread CTAs: all carry words requested at once, then polled
    (4500007, 2048, 64, 4, 2),    # 256-thread CTAs: carry words polled one after another, LL
])
def test_emulated_self_publishing_carry_words(emu, oracle, E, W, H, n, flags):
    """The line passes from W = 1024 up publish their carry rows word by word (never-0 encoded
    words, each consumer thread polling and clearing its own) instead of with a flag."""
    ll = bool(flags & 2)
    roe, got = run(emu, "square", E, W, H, n, flags, 13)
    want = oracle.gmp_square(E, splitmix_words(E, 13), n, ll=ll)
    assert np.array_equal(got, want)
    assert roe < 0.1
