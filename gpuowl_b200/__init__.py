"""gpuowl_b200 -- B200-native engine for the Mersenne PRP/LL squaring x <- x^2 (-2) mod 2^E-1.

The engine is libowl.so (hand-written sm_100a CUDA behind the C ABI in
include/owl.h). This module is a thin ctypes binding over that ABI, used by the
tests and bench.py. There is no CPU path: importing works anywhere, but every
operation needs libowl.so and a CUDA device, and raises OwlError otherwise.

Names follow the reference's Gpu surface (src/Gpu.h): writeIn/readData,
square/squareLoop, modMul, isEqual, bufResidue.
"""
import ctypes
import os

import numpy as np

__all__ = ["OwlError", "load", "Plan", "n_words", "fft_choose", "LIB_PATH", "prp_run", "ll_run",
           "prp_save", "prp_load", "ll_save", "ll_load", "crc32"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libowl.so")

SQ_MUL3 = 1
SQ_LL = 2
SQ_NO_ROE = 4
# column-pass tile variants (include/owl.h OWL_COL_*)
COL_AUTO, COL_V16, COL_V8, COL_V16_OCC2 = 0, 1, 2, 3
COL_NAMES = {COL_V16: "v16", COL_V8: "v8", COL_V16_OCC2: "v16occ2"}
# split-precision form flags (include/owl.h OWL_SPLIT_*)
SPLIT_COLUMNS, SPLIT_LINES = 1, 2


def column_variant_supported(H, variant):
    """Whether the column variant is built for columns of H points."""
    return bool(load().owl_column_variant_supported(int(H), int(variant)))


OK = 0
ERR_TIMEOUT = -4


class OwlError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (status %d)" % (msg, status))
        self.status = status


_lib = None

_P = ctypes.c_void_p
_I32P = ctypes.POINTER(ctypes.c_int32)
_U32P = ctypes.POINTER(ctypes.c_uint32)
_U64P = ctypes.POINTER(ctypes.c_uint64)

class RunOpts(ctypes.Structure):
    """owl_run_opts (include/owl_host.h)."""
    _fields_ = [("block_size", ctypes.c_uint32), ("log_step", ctypes.c_uint32), ("check_step", ctypes.c_uint32),
                ("stop_after", ctypes.c_uint32), ("n_savefiles", ctypes.c_uint32), ("W", ctypes.c_uint32),
                ("H", ctypes.c_uint32), ("save_dir", ctypes.c_char_p), ("inject_fault_k", ctypes.c_uint32),
                ("verbose", ctypes.c_int), ("res_cap", ctypes.c_uint32), ("res_k", ctypes.POINTER(ctypes.c_uint32)),
                ("res_res64", ctypes.POINTER(ctypes.c_uint64)), ("res_n", ctypes.POINTER(ctypes.c_uint32)),
                ("split", ctypes.c_int), ("proof_power", ctypes.c_uint32), ("column_variant", ctypes.c_uint32)]


class RunResult(ctypes.Structure):
    """owl_run_result (include/owl_host.h)."""
    _fields_ = [("is_prime", ctypes.c_int), ("finished", ctypes.c_int), ("k", ctypes.c_uint32),
                ("res64", ctypes.c_uint64), ("n_errors", ctypes.c_uint32), ("res2048", ctypes.c_char * 513),
                ("proof_power", ctypes.c_uint32), ("proof_file", ctypes.c_char * 1024),
                ("roe_n", ctypes.c_uint32), ("roe_max", ctypes.c_float), ("roe_z", ctypes.c_float),
                ("roe_z_avg", ctypes.c_float), ("n_danger_roe", ctypes.c_uint32)]


_SIGS = {
    "owl_abi_version": ([], ctypes.c_int),
    "owl_error_string": ([ctypes.c_int], ctypes.c_char_p),
    "owl_last_error": ([], ctypes.c_char_p),
    "owl_device_count": ([ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "owl_device_info": ([ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                         ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    "owl_fft_choose": ([ctypes.c_uint32, ctypes.c_double, _U32P, _U32P, _U32P], ctypes.c_int),
    "owl_plan_create": ([ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                         ctypes.POINTER(_P)], ctypes.c_int),
    "owl_plan_destroy": ([_P], ctypes.c_int),
    "owl_plan_shape": ([_P, _U32P, _U32P, _U32P], ctypes.c_int),
    "owl_plan_set_timeout": ([_P, ctypes.c_uint64], ctypes.c_int),
    "owl_plan_set_split": ([_P, ctypes.c_int], ctypes.c_int),
    "owl_plan_set_column_variant": ([_P, ctypes.c_uint32], ctypes.c_int),
    "owl_plan_column_variant": ([_P, _U32P], ctypes.c_int),
    "owl_column_variant_supported": ([ctypes.c_uint32, ctypes.c_uint32], ctypes.c_int),
    "owl_buf_alloc": ([_P, ctypes.POINTER(_P)], ctypes.c_int),
    "owl_buf_free": ([_P, _P], ctypes.c_int),
    "owl_buf_copy": ([_P, _P, _P], ctypes.c_int),
    "owl_buf_set": ([_P, _P, ctypes.c_uint32], ctypes.c_int),
    "owl_write_digits": ([_P, _P, _I32P], ctypes.c_int),
    "owl_read_digits": ([_P, _P, _I32P], ctypes.c_int),
    "owl_write_words": ([_P, _P, _U32P], ctypes.c_int),
    "owl_read_words": ([_P, _P, _U32P], ctypes.c_int),
    "owl_square": ([_P, _P, _P, ctypes.c_uint32, ctypes.c_uint32], ctypes.c_int),
    "owl_modmul": ([_P, _P, _P, ctypes.c_int], ctypes.c_int),
    "owl_is_equal": ([_P, _P, _P, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "owl_res64": ([_P, _P, _U64P], ctypes.c_int),
    "owl_sum64": ([_P, _P, _U64P], ctypes.c_int),
    "owl_read_roe": ([_P, ctypes.POINTER(ctypes.c_float), ctypes.c_uint32, _U32P], ctypes.c_int),
    "owl_sync": ([_P], ctypes.c_int),
    "owl_probe_wait_timeout": ([_P], ctypes.c_int),
    "owl_plan_stream": ([_P, ctypes.POINTER(_P)], ctypes.c_int),
    "owl_prp_run": ([ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(RunOpts), ctypes.POINTER(RunResult)], ctypes.c_int),
    "owl_ll_run": ([ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(RunOpts), ctypes.POINTER(RunResult)], ctypes.c_int),
    "owl_prp_save": ([ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _U32P,
                      ctypes.c_uint32, ctypes.c_double], ctypes.c_int),
    "owl_prp_load": ([ctypes.c_char_p, ctypes.c_uint32, _U32P, _U32P, _U64P, _U32P, _U32P,
                      ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "owl_ll_save": ([ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, _U32P, ctypes.c_double], ctypes.c_int),
    "owl_ll_load": ([ctypes.c_char_p, ctypes.c_uint32, _U32P, _U32P, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "owl_crc32": ([ctypes.c_void_p, ctypes.c_size_t], ctypes.c_uint32),
    "owl_sha3_256": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint8)], None),
    "owl_proof_points": ([ctypes.c_uint32, ctypes.c_uint32, _U32P, ctypes.c_uint32, _U32P], ctypes.c_int),
    "owl_proof_verify": ([ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
                         ctypes.c_int),
    "owl_exp_mul": ([_P, _P, ctypes.c_uint64, _P], ctypes.c_int),
    "owl_probe_tc_wait_timeout": ([_P], ctypes.c_int),
    "owl_worktodo_parse": ([ctypes.c_char_p, ctypes.c_void_p], ctypes.c_int),
    "owl_worktodo_get": ([ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p,
                          ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "owl_task_run": ([ctypes.c_int, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                      ctypes.c_size_t], ctypes.c_int),
    "owl_cert_run": ([ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint8),
                      ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "owl_file_md5": ([ctypes.c_char_p, ctypes.c_char_p], ctypes.c_int),
    "owl_batch_create": ([ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(_P), ctypes.POINTER(_P)], ctypes.c_int),
    "owl_batch_square": ([_P, ctypes.POINTER(_P), ctypes.c_uint32, ctypes.c_uint32], ctypes.c_int),
    "owl_batch_sync": ([_P], ctypes.c_int),
    "owl_batch_destroy": ([_P], ctypes.c_int),
    "owl_profile_square": ([_P, _P, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float), _U32P],
                           ctypes.c_int),
}


def load(path=None):
    """Load libowl.so (built by gpuowl_b200/build.py). Raises OwlError if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OwlError(-100, "libowl.so not built (run python -m gpuowl_b200.build): " + p)
    lib = ctypes.CDLL(p)
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.owl_abi_version() != 1:
        raise OwlError(-100, "libowl ABI mismatch")
    if path is None:
        _lib = lib
    return lib


def _check(status):
    if status != OK:
        lib = load()
        raise OwlError(status, lib.owl_last_error().decode(errors="replace") or
                       lib.owl_error_string(status).decode())


def n_words(E):
    """(E-1)/32+1 compact u32 words (reference src/common.h nWords)."""
    return (E - 1) // 32 + 1


def fft_choose(E, max_bpw=0.0, tune=None):
    """(N, W, H) for exponent E (reference FFTConfig::bestFit). With `tune`, a tune.json written by
    gpuowl_b200.tune, the W x H split measured fastest for that N is used."""
    lib = load()
    N, W, H = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib.owl_fft_choose(E, max_bpw, ctypes.byref(N), ctypes.byref(W), ctypes.byref(H)))
    if tune and os.path.exists(tune):
        import json
        with open(tune) as f:
            t = json.load(f)
        # with measured max bits/word (tune --bpw-scan): the smallest FFT whose limit covers E
        # (or max_bpw when given) and that holds at least 8 bits per word (the engine's lower bound)
        scanned = sorted((int(n), v) for n, v in t.items() if len(v) >= 5 and v[4])
        for n, v in scanned:
            if 8 <= E / n <= (max_bpw if max_bpw > 0 else v[4]):
                return n, int(v[0]), int(v[1])
        if str(N.value) in t:
            return N.value, int(t[str(N.value)][0]), int(t[str(N.value)][1])
    return N.value, W.value, H.value


def device_count():
    lib = load()
    n = ctypes.c_int(0)
    _check(lib.owl_device_count(ctypes.byref(n)))
    return n.value


class Plan:
    """One exponent on one device (reference Gpu, src/Gpu.cpp:394-564).

    Word buffers are device pointers (ints) returned by alloc(); they hold N
    balanced int32 digits in natural word order.
    """

    def __init__(self, E, device=0, W=0, H=0, split=False, column_variant=0):
        self.lib = load()
        self.E = int(E)
        self.device = device
        h = _P()
        _check(self.lib.owl_plan_create(device, self.E, W, H, ctypes.byref(h)))
        self.h = h
        N, Wv, Hv = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(self.lib.owl_plan_shape(self.h, ctypes.byref(N), ctypes.byref(Wv), ctypes.byref(Hv)))
        self.N, self.W, self.H = N.value, Wv.value, Hv.value
        self.nwords = n_words(self.E)
        self.split = 0
        if split:
            self.set_split(split)
        if column_variant != COL_AUTO:
            self.set_column_variant(column_variant)

    def close(self):
        if getattr(self, "h", None):
            _check(self.lib.owl_plan_destroy(self.h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- buffers --
    def alloc(self):
        b = _P()
        _check(self.lib.owl_buf_alloc(self.h, ctypes.byref(b)))
        return b.value

    def free(self, buf):
        _check(self.lib.owl_buf_free(self.h, buf))

    def copy(self, dst, src):
        _check(self.lib.owl_buf_copy(self.h, dst, src))

    def set(self, buf, value):
        _check(self.lib.owl_buf_set(self.h, buf, value))

    def set_timeout(self, ns):
        _check(self.lib.owl_plan_set_timeout(self.h, int(ns)))

    def set_split(self, flags=True):
        """Split-precision form: INT8 tensor-core GEMMs for the first and last stages of every
        column FFT (SPLIT_COLUMNS; 32-point at H = 2048, 40-point at H = 2560) and / or of every
        line FFT (SPLIT_LINES; 16-point at W = 2048). True means SPLIT_COLUMNS; a flag whose pass
        has no split form at this shape raises OwlError."""
        _check(self.lib.owl_plan_set_split(self.h, int(flags)))
        self.split = int(flags)

    def set_column_variant(self, variant):
        """Column-pass tile variant: COL_V16, COL_V8, COL_V16_OCC2, or COL_AUTO for the shape's
        default (include/owl.h)."""
        _check(self.lib.owl_plan_set_column_variant(self.h, int(variant)))

    @property
    def column_variant(self):
        v = ctypes.c_uint32(0)
        _check(self.lib.owl_plan_column_variant(self.h, ctypes.byref(v)))
        return v.value

    def write_digits(self, buf, digits):
        d = np.ascontiguousarray(digits, dtype=np.int32)
        assert d.size == self.N
        _check(self.lib.owl_write_digits(self.h, buf, d.ctypes.data_as(_I32P)))

    def read_digits(self, buf):
        d = np.empty(self.N, dtype=np.int32)
        _check(self.lib.owl_read_digits(self.h, buf, d.ctypes.data_as(_I32P)))
        return d

    def writeIn(self, buf, words):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        assert w.size == self.nwords
        _check(self.lib.owl_write_words(self.h, buf, w.ctypes.data_as(_U32P)))

    def readOut(self, buf, out=None):
        """Compact words of a buffer (reference readAndCompress: checked read + compactBits), into
        `out` (a contiguous uint32 array of nwords, e.g. over pinned memory) when given."""
        w = np.empty(self.nwords, dtype=np.uint32) if out is None else out
        assert w.dtype == np.uint32 and w.size == self.nwords and w.flags["C_CONTIGUOUS"]
        _check(self.lib.owl_read_words(self.h, buf, w.ctypes.data_as(_U32P)))
        return w

    # -- engine ops --
    def squareLoop(self, out, inp, n, mul3=False, ll=False, roe=True):
        """n squarings; roe=False skips the round-off measurement (readROE gets no entries for them)."""
        flags = (SQ_MUL3 if mul3 else 0) | (SQ_LL if ll else 0) | (0 if roe else SQ_NO_ROE)
        _check(self.lib.owl_square(self.h, out, inp, int(n), flags))

    def expMul(self, a, h, b):
        """a := a^h * b (reference Gpu::expMul; a and b different buffers)."""
        _check(self.lib.owl_exp_mul(self.h, a, int(h), b))

    def modMul(self, io_a, in_b, mul3=False):
        _check(self.lib.owl_modmul(self.h, io_a, in_b, 1 if mul3 else 0))

    def isEqual(self, a, b):
        r = ctypes.c_int(0)
        _check(self.lib.owl_is_equal(self.h, a, b, ctypes.byref(r)))
        return bool(r.value)

    def bufResidue(self, buf):
        r = ctypes.c_uint64(0)
        _check(self.lib.owl_res64(self.h, buf, ctypes.byref(r)))
        return r.value

    def sum64(self, buf):
        r = ctypes.c_uint64(0)
        _check(self.lib.owl_sum64(self.h, buf, ctypes.byref(r)))
        return r.value

    def readROE(self, cap=1 << 16):
        arr = (ctypes.c_float * cap)()
        n = ctypes.c_uint32(0)
        _check(self.lib.owl_read_roe(self.h, arr, cap, ctypes.byref(n)))
        return np.array(arr[:n.value], dtype=np.float32)

    def sync(self):
        _check(self.lib.owl_sync(self.h))

    def stream(self):
        """The plan's cudaStream_t as an int (wrap with torch.cuda.ExternalStream)."""
        s = _P()
        _check(self.lib.owl_plan_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def profile_square(self, buf, n, roe=True):
        """Per-kernel device time of n squarings: {"pass2": (ms, launches), "pass1": ..., "edge": ...}."""
        ms = (ctypes.c_float * 3)()
        cnt = (ctypes.c_uint32 * 3)()
        _check(self.lib.owl_profile_square(self.h, buf, int(n), 0 if roe else SQ_NO_ROE, ms, cnt))
        return {"pass2": (ms[0], cnt[0]), "pass1": (ms[1], cnt[1]), "edge": (ms[2], cnt[2])}

    def probe_wait_timeout(self):
        """Returns the status of a device wait that must time out (ERR_TIMEOUT)."""
        return self.lib.owl_probe_wait_timeout(self.h)

    def probe_tc_wait_timeout(self):
        """Status of a tensor-core completion wait that must time out (ERR_TIMEOUT)."""
        return self.lib.owl_probe_tc_wait_timeout(self.h)


# ---- host drivers (include/owl_host.h) ----

def _run(fn_name, E, device, block, log_step, check_step, stop_after, save_dir, W, H, inject_fault_k, verbose,
         n_savefiles=4, cap=4096, split=False, proof_power=0, column_variant=0):
    lib = load()
    ks = (ctypes.c_uint32 * cap)()
    rs = (ctypes.c_uint64 * cap)()
    n = ctypes.c_uint32(0)
    o = RunOpts(block, log_step, check_step, stop_after, n_savefiles, W, H,
                save_dir.encode() if save_dir else None, inject_fault_k, 1 if verbose else 0, cap,
                ks, rs, ctypes.pointer(n), int(split), int(proof_power), int(column_variant))
    r = RunResult()
    _check(getattr(lib, fn_name)(device, E, ctypes.byref(o), ctypes.byref(r)))
    return {"is_prime": bool(r.is_prime), "finished": bool(r.finished), "k": r.k, "res64": r.res64,
            "n_errors": r.n_errors, "res2048": r.res2048.decode(),
            "proof_power": r.proof_power, "proof_file": r.proof_file.decode() or None,
            "roe_n": r.roe_n, "roe_max": r.roe_max, "roe_z": r.roe_z, "roe_z_avg": r.roe_z_avg,
            "n_danger_roe": r.n_danger_roe,
            "checkpoints": [(ks[i], rs[i]) for i in range(n.value)]}


def prp_run(E, device=0, block=1000, log_step=20000, check_step=0, stop_after=0, save_dir=None, W=0, H=0,
            inject_fault_k=0, verbose=False, split=False, proof_power=0, column_variant=0):
    """PRP-3 test (the reference's Gpu::isPrimePRP) through owl_prp_run; with proof_power > 0 the
    proof residues go to save_dir/<E>/proof/ and the verified proof to save_dir/proof/<E>-<p>.proof."""
    return _run("owl_prp_run", E, device, block, log_step, check_step, stop_after, save_dir, W, H,
                inject_fault_k, verbose, split=split, proof_power=proof_power, column_variant=column_variant)


class Task(ctypes.Structure):
    """owl_task (include/owl_host.h): one worktodo entry."""
    _fields_ = [("kind", ctypes.c_int), ("exponent", ctypes.c_uint32), ("squarings", ctypes.c_uint32),
                ("aid", ctypes.c_char * 33), ("line", ctypes.c_char * 512)]
    KINDS = {0: "PRP", 1: "LL", 2: "CERT"}

    def as_dict(self):
        return {"kind": self.KINDS.get(self.kind, "?"), "exponent": self.exponent, "squarings": self.squarings,
                "aid": self.aid.decode(), "line": self.line.decode()}


def worktodo_parse(line):
    """The task of one worktodo line (reference Worktodo parse), or None if the line is ignored."""
    t = Task()
    if load().owl_worktodo_parse(line.encode(), ctypes.byref(t)) != 0:
        return None
    return t


def worktodo_get(dir, instance=0, master_dir=None):
    """Next task of worker `instance` from <dir>/worktodo-<instance>.txt or the pooled
    <master_dir>/worktodo.txt, or None."""
    t, found = Task(), ctypes.c_int(0)
    _check(load().owl_worktodo_get(str(dir).encode(), instance, str(master_dir).encode() if master_dir else None,
                                   ctypes.byref(t), ctypes.byref(found)))
    return t if found.value else None


def task_run(task, dir, instance=0, device=0, proof_power=0, block=1000, W=0, H=0, split=False, column_variant=0):
    """Runs one task (reference Task::execute); returns its result JSON line (also appended to
    <dir>/results-<instance>.txt)."""
    o = RunOpts(block, 0, 0, 0, 4, W, H, None, 0, 0, 0, None, None, None, int(split), int(proof_power),
                int(column_variant))
    buf = ctypes.create_string_buffer(8192)
    _check(load().owl_task_run(device, str(dir).encode(), instance, ctypes.byref(task), ctypes.byref(o), buf,
                               len(buf)))
    return buf.value.decode()


def cert_run(E, squarings, cert_file, device=0):
    """(sha3-256 digest bytes, res64) of `squarings` squarings of the start value in cert_file."""
    out = (ctypes.c_uint8 * 32)()
    r = ctypes.c_uint64(0)
    _check(load().owl_cert_run(device, E, squarings, str(cert_file).encode(), out, ctypes.byref(r)))
    return bytes(out), r.value


def file_md5(path):
    out = ctypes.create_string_buffer(33)
    _check(load().owl_file_md5(str(path).encode(), out))
    return out.value.decode()


def sha3_256(data):
    """SHA3-256 digest (bytes) of `data` with the library's proof hash."""
    b = bytes(data)
    out = (ctypes.c_uint8 * 32)()
    load().owl_sha3_256(b, len(b), out)
    return bytes(out)


def proof_points(E, power):
    """Iterations whose residues a power-`power` proof needs (increasing, the last = E)."""
    lib = load()
    n = ctypes.c_uint32(0)
    _check(lib.owl_proof_points(E, power, None, 0, ctypes.byref(n)))
    arr = (ctypes.c_uint32 * n.value)()
    _check(lib.owl_proof_points(E, power, arr, n.value, ctypes.byref(n)))
    return list(arr)


def proof_verify(path, device=0):
    """(valid, is_prime) of a proof file (reference Proof::verify)."""
    v, p = ctypes.c_int(0), ctypes.c_int(0)
    _check(load().owl_proof_verify(device, str(path).encode(), ctypes.byref(v), ctypes.byref(p)))
    return bool(v.value), bool(p.value)


def ll_run(E, device=0, log_step=10000, stop_after=0, save_dir=None, W=0, H=0, verbose=False, split=False,
           column_variant=0):
    """Lucas-Lehmer test (the reference's Gpu::isPrimeLL) through owl_ll_run."""
    return _run("owl_ll_run", E, device, 1000, log_step, 0, stop_after, save_dir, W, H, 0, verbose, split=split,
                column_variant=column_variant)


def prp_save(save_dir, E, k, block, res64, check, n_errors=0, elapsed=0.0):
    c = np.ascontiguousarray(check, dtype=np.uint32)
    _check(load().owl_prp_save(save_dir.encode(), E, k, block, res64, c.ctypes.data_as(_U32P), n_errors, elapsed))


def prp_load(save_dir, E):
    k, b, ne = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    r, el = ctypes.c_uint64(), ctypes.c_double()
    c = np.zeros(n_words(E), dtype=np.uint32)
    _check(load().owl_prp_load(save_dir.encode(), E, ctypes.byref(k), ctypes.byref(b), ctypes.byref(r),
                               c.ctypes.data_as(_U32P), ctypes.byref(ne), ctypes.byref(el)))
    return {"k": k.value, "block": b.value, "res64": r.value, "check": c, "n_errors": ne.value, "elapsed": el.value}


def ll_save(save_dir, E, k, data, elapsed=0.0):
    d = np.ascontiguousarray(data, dtype=np.uint32)
    _check(load().owl_ll_save(save_dir.encode(), E, k, d.ctypes.data_as(_U32P), elapsed))


def ll_load(save_dir, E):
    k, el = ctypes.c_uint32(), ctypes.c_double()
    d = np.zeros(n_words(E), dtype=np.uint32)
    _check(load().owl_ll_load(save_dir.encode(), E, ctypes.byref(k), d.ctypes.data_as(_U32P), ctypes.byref(el)))
    return {"k": k.value, "data": d, "elapsed": el.value}


def crc32(data):
    b = bytes(data)
    return load().owl_crc32(b, len(b))


class Batch:
    """Plans of one device squared together, one CUDA-graph launch per call (owl_batch_*)."""

    def __init__(self, plans, device=0):
        self.lib = load()
        self.plans = list(plans)
        arr = (_P * len(self.plans))(*[p.h for p in self.plans])
        h = _P()
        _check(self.lib.owl_batch_create(device, len(self.plans), arr, ctypes.byref(h)))
        self.h = h

    def square(self, bufs, n, ll=False, roe=True):
        arr = (_P * len(bufs))(*bufs)
        _check(self.lib.owl_batch_square(self.h, arr, int(n), (SQ_LL if ll else 0) | (0 if roe else SQ_NO_ROE)))

    def sync(self):
        _check(self.lib.owl_batch_sync(self.h))

    def close(self):
        if getattr(self, "h", None):
            _check(self.lib.owl_batch_destroy(self.h))
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
