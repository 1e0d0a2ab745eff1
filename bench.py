#!/usr/bin/env python
"""bench.py -- ms per PRP-3 iteration at the 8M FFT on B200 (libowl): the plain FP64 form
(the headline value) and the split-precision tensor-core form ("split_tc"), both bit-exact.

Workload (one "step" = one Gerbicz block of the reference's PRP loop,
src/Gpu.cpp:1461-1483): modMul(check, data) then 1,000 squarings of data,
for E = the seeded prime in [136M, 139M] (136,181,029) at N = 8M words
(W = H = 2048, 16.2 bits/word). Inputs are resident in HBM when the timed region
starts; the L2 is flushed (a 512 MiB write) between timed steps, outside the
timing. After the timed region the res64 at every 1,000 iterations is compared
with the GMP golden table and a full Gerbicz check (B extra squarings) is run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's algorithm on the host cores: the reference's
OpenCL kernels cannot run here, so its CPU restatement (oracle/ibdwt.c, all host
threads) stands in, timed over a fixed sample of CPU_SAMPLE 8M squarings; the other arm
takes the same sample for its cpu_baseline before it touches the GPU. Multi-GPU runs are replicas (one
exponent per GPU, no collective on the data path): value = max-over-ranks time /
all iterations.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20261203
E_8M = 136181029      # oracle_seeded_prime(SEED + 2, 136M, 139M)
W_8M, H_8M = 2048, 2048
N_8M = 2 * W_8M * H_8M
NW_8M = (E_8M - 1) // 32 + 1
BLOCK = 1000
# squarings in the CPU sample (after one untimed squaring), the same in both arms: about 2 s of
# CPU work at 8M on 16 host threads
CPU_SAMPLE = 25


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--block", type=int, default=BLOCK)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision (tensor-core) form")
    ap.add_argument("--batch-shapes", default="default", choices=["default", "tuned"],
                    help="batch64: the library's W x H split per FFT size, or the split and column variant "
                         "that gpuowl_b200/tune_b200.json holds for that size (the FFT size is the same)")
    ap.add_argument("--no-configs", action="store_true",
                    help="prp8m on one GPU: skip the short runs of the other configurations (20M, 256K, "
                         "batch64) whose lines the 8M line carries under \"configs\"")
    ap.add_argument("--workload", default="prp8m", choices=["prp8m", "batch64", "prp20m", "prp256k"],
                    help="prp8m: the headline line; batch64: 64 uneven exponents in one graph per block; "
                         "prp20m / prp256k: PRP-3 at the 20M FFT (5 * 2^22) / the 256K FFT")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [x for x in sm if mx and x > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def load_golden(name):
    path = os.path.join(ROOT, "tests", "golden", name + ".json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_bf16():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def profiled_traffic(name="8m"):
    """Per-launch DRAM bytes of the pass kernels from the committed ncu summary
    (profiles/traffic_<name>.json), if any."""
    path = os.path.join(ROOT, "profiles", "traffic_%s.json" % name)
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def roe_measured(k, n):
    """Whether the block of n squarings from iteration k measures its round-off. The reference's PRP
    loop measures it on a sample only (src/Gpu.cpp:1026, 1459-1464: 2,000 iterations once the first
    30 are past, then 400 after every 20,000-iteration log step; the other iterations run the kernel
    build without it, src/Gpu.cpp:592-596), and so does owl_prp_run. Here a block is measured whole
    when it holds a sampled iteration, and the first sample ends at iteration 2,000 instead of 2,030
    (blocks 0 and 1 of 1,000), so that the third warm-up block already runs, and captures, the graph
    of the blocks without the measurement."""
    if k < 2000 and k + n > 30:
        return True
    start = (k + n - 1) // 20000 * 20000  # the last log step before the block's end
    return start >= 20000 and k < start + 400 and k + n > start


def cpu_port_ms_per_iter(E, N, iters, threads):
    """The reference's IBDWT squaring restated on the CPU (oracle/ibdwt.c), ms per iteration."""
    import ctypes
    import numpy as np
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                   capture_output=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    lib.oracle_ibdwt_create.restype = ctypes.c_void_p
    lib.oracle_ibdwt_create.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int]
    lib.oracle_ibdwt_square.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.c_int,
                                        ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.oracle_ibdwt_destroy.argtypes = [ctypes.c_void_p]
    lib.oracle_expand_bits.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.POINTER(ctypes.c_int32)]
    p = lib.oracle_ibdwt_create(E, N, threads)
    rng = np.random.default_rng(SEED)
    nw = (E - 1) // 32 + 1
    w = rng.integers(0, 2 ** 32, size=nw, dtype=np.uint64).astype(np.uint32)
    if E % 32:
        w[-1] &= (1 << (E % 32)) - 1
    d = np.zeros(N, dtype=np.int32)
    lib.oracle_expand_bits(w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), N, E,
                           d.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    roe = ctypes.c_double()
    dp = d.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    lib.oracle_ibdwt_square(p, dp, 0, 0, ctypes.byref(roe))  # warm
    times = []
    for _ in range(iters):
        t0 = time.perf_counter()
        lib.oracle_ibdwt_square(p, dp, 0, 0, ctypes.byref(roe))
        times.append(time.perf_counter() - t0)
    lib.oracle_ibdwt_destroy(p)
    return 1e3 * sum(times) / len(times), times


def replica_summary(dist, total_ms, e2e_step_ms, steps, block, world, device="cpu"):
    """Replicas (one exponent per GPU, no collective on the data path): the job's time is the
    slowest rank's. Returns (max timed ms, max e2e ms per step, value in ms per iteration over
    all ranks' iterations)."""
    if dist is not None and world > 1:
        import torch
        t = torch.tensor([total_ms, e2e_step_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_step_ms = float(t[0]), float(t[1])
    return total_ms, e2e_step_ms, total_ms / (world * steps * block)


def cpu_sample_line():
    """The CPU baseline: CPU_SAMPLE squarings of the 8M workload with oracle/ibdwt.c on every host
    thread. Both arms take it the same way, in a process that has not touched the GPU yet."""
    threads = os.cpu_count() or 1
    ms, _ = cpu_port_ms_per_iter(E_8M, N_8M, CPU_SAMPLE, threads)
    return {"value": round(ms, 3), "unit": "ms/iter", "cores": threads, "kind": "port",
            "sample": "%d squarings (after 1 untimed) at E=%d, N=8M with oracle/ibdwt.c (OpenMP, all host "
                      "threads), taken before any GPU work; the reference's OpenCL kernels have no CPU "
                      "runtime here" % (CPU_SAMPLE, E_8M)}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cpu = cpu_sample_line()
    ms = cpu["value"]
    line = {
        "impl": "reference",
        "metric": "ms/iter PRP @8M FFT: split-precision TC vs plain FP64, bit-exact res64",
        "value": ms, "unit": "ms/iter", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "PRP-3 squaring, E=136181029 (seeded prime in [136M,139M]), FFT 8M",
                   "E": E_8M, "N": N_8M, "step": "one 8M IBDWT squaring on the host cores",
                   "sample": "%d squarings regardless of --steps/--warmup" % CPU_SAMPLE},
        "cpu_baseline": cpu,
        "e2e": {"value": ms, "unit": "ms/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local):
    # the CPU baseline first, in a process that has not touched the GPU (rank 0 of a 1-GPU run)
    cpu = None
    if not args.no_cpu_baseline and world == 1 and rank == 0:
        cpu = cpu_sample_line()
    import numpy as np
    import torch
    import gpuowl_b200 as owl
    from gpuowl_b200 import build
    build.build()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    B = args.block
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    golden = load_golden("prp_8m")

    def measure(split, steps, warmup, with_e2e):
        """Timed PRP blocks of one form: CUDA-event step times, per-kernel device times from the
        launch stamps, res64 per block against the golden table, a final Gerbicz check and
        (with_e2e) the host-buffer end-to-end loop through the public API."""
        plan = owl.Plan(E_8M, device=local, W=W_8M, H=H_8M, split=split)
        stream = torch.cuda.ExternalStream(plan.stream(), device=torch.device("cuda", local))
        data, check, aux = plan.alloc(), plan.alloc(), plan.alloc()
        plan.writeIn(data, [3] + [0] * (plan.nwords - 1))
        plan.writeIn(check, [1] + [0] * (plan.nwords - 1))
        res = []
        blk = [0]

        def step():
            k = blk[0] * B
            blk[0] += 1
            plan.modMul(check, data)
            return plan.profile_square(data, B, roe=roe_measured(k, B))

        for _ in range(warmup):
            step()
            res.append("%016x" % plan.bufResidue(data))
        roe_warm = plan.readROE()
        step_ms, prof = [], {"pass2": [0.0, 0], "pass1": [0.0, 0], "edge": [0.0, 0]}
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                pr = step()
                e1.record(stream)
                e1.synchronize()
                step_ms.append(e0.elapsed_time(e1))
                for k, (ms, n) in pr.items():
                    prof[k][0] += ms
                    prof[k][1] += n
                res.append("%016x" % plan.bufResidue(data))
        torch.cuda.synchronize()
        barrier()
        roe = np.concatenate([roe_warm, plan.readROE()])
        # Gerbicz check of the final state (reference doCheck, src/Gpu.cpp:767-771)
        plan.squareLoop(aux, check, B, mul3=True)
        plan.modMul(check, data)
        gerbicz_ok = plan.isEqual(check, aux)
        e2e_ms = []
        if with_e2e:
            # e2e through the public API with pinned host buffers: writeIn -> block -> readOut
            pin_in = torch.empty(plan.nwords, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
            pin_out = torch.empty(plan.nwords, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
            plan.readOut(data, out=pin_in)
            # one untimed pass first: squareLoop's graph for this buffer pair is captured on first use.
            # These blocks lie past the round-off sample, so they run, like the timed blocks, the
            # build without the measurement.
            plan.writeIn(data, pin_in)
            plan.modMul(check, data)
            plan.squareLoop(data, data, B, roe=False)
            plan.readOut(data, out=pin_in)
            barrier()
            for _ in range(max(2, steps // 2)):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                plan.writeIn(data, pin_in)
                plan.modMul(check, data)
                plan.squareLoop(data, data, B, roe=False)
                plan.readOut(data, out=pin_out)
                e2e_ms.append(1e3 * (time.perf_counter() - t0))
                pin_in, pin_out = pin_out, pin_in
            barrier()
        plan.close()
        n = min(len(res), len(golden["res64"])) if golden else 0
        return {"total_ms": sum(step_ms), "prof": prof, "roe": float(roe.max()) if roe.size else None,
                "gerbicz_ok": bool(gerbicz_ok), "res_match": (res[:n] == golden["res64"][:n]) if golden else None,
                "res_checked": n, "clocks": clocks.summary(), "e2e_ms": e2e_ms}

    plain = measure(False, args.steps, args.warmup, True)
    split = measure(1, args.steps, args.warmup, False) if not args.no_split else None
    # both passes split (the line pass's 16-point stages on the tensor cores too)
    both = measure(3, args.steps, args.warmup, False) if not args.no_split else None
    total_ms, prof, roe = plain["total_ms"], plain["prof"], plain["roe"]
    e2e_ms = plain["e2e_ms"]
    total_ms, e2e_step, value = replica_summary(dist, total_ms, sum(e2e_ms) / len(e2e_ms), args.steps, B, world,
                                                device="cuda")
    split_line = None
    if split is not None:
        s_total, _, s_value = replica_summary(dist, split["total_ms"], 0.0, args.steps, B, world, device="cuda")
        sp = split["prof"]
        tc_ms = sp["pass2"][0] / max(sp["pass2"][1], 1)
        # INT8 work of one k_pass2_tc launch: W/2 CTAs x 2 directions x 28 digit-plane products of a
        # 128 x 64 (outputs) x 64 (inputs) GEMM (issued as 2 halves x 14 MMAs of N = 32 (7 - i))
        tc_ops = 2.0 * (W_8M // 2) * 2 * 28 * 128 * 64 * 64
        bf16 = measured_bf16()
        b_total, _, b_value = replica_summary(dist, both["total_ms"], 0.0, args.steps, B, world, device="cuda")
        bp = both["prof"]
        l_ms = bp["pass1"][0] / max(bp["pass1"][1], 1)
        # the split line pass (fused): H/2 CTAs x 2 directions x 28 digit-plane products of a
        # 256 x 32 (outputs) x 32 (inputs) GEMM
        line_ops = 2.0 * (H_8M // 2) * 2 * 28 * 256 * 32 * 32
        both_line = {
            "form": "the column pass as above and the 16-point line stages as INT8 tcgen05 GEMMs too",
            "ms_per_iter": round(b_value, 5), "ms_per_step": round(b_total / args.steps, 4),
            "kernel_ms": {k: round(v[0] / max(v[1], 1), 5) for k, v in bp.items()},
            "max_roe": round(both["roe"], 5) if both["roe"] is not None else None,
            "res64_match_golden": both["res_match"], "res64_checked": both["res_checked"],
            "gerbicz_ok": both["gerbicz_ok"],
            "line_tensor_roofline": {"bound": "tensor", "kernel": "k_pass1 (split)",
                                     "achieved": round(line_ops / (l_ms * 1e-3) / 1e12, 2),
                                     "peak": round(2 * bf16[0], 1), "unit": "TOP/s (int8)",
                                     "frac": round(line_ops / (l_ms * 1e-3) / 1e12 / (2 * bf16[0]), 4),
                                     "int8_ops_per_launch": line_ops},
            "clocks": both["clocks"],
            "vs_plain": round(b_value / value, 3),
        }
        split_line = {
            "form": "split-precision: 32-point column stages as INT8 tcgen05 GEMMs on 7 base-256 digit planes",
            "ms_per_iter": round(s_value, 5), "ms_per_step": round(s_total / args.steps, 4),
            "kernel_ms": {k: round(v[0] / max(v[1], 1), 5) for k, v in sp.items()},
            "max_roe": round(split["roe"], 5) if split["roe"] is not None else None,
            "max_roe_plain": round(roe, 5) if roe is not None else None,
            "res64_match_golden": split["res_match"], "res64_checked": split["res_checked"],
            "gerbicz_ok": split["gerbicz_ok"],
            "tensor_roofline": {"bound": "tensor", "kernel": "k_pass2_tc",
                                "achieved": round(tc_ops / (tc_ms * 1e-3) / 1e12, 2),
                                "peak": round(2 * bf16[0], 1), "unit": "TOP/s (int8)",
                                "frac": round(tc_ops / (tc_ms * 1e-3) / 1e12 / (2 * bf16[0]), 4),
                                "peak_kind": "2 x %s bf16 dense (int8 dense rate is twice bf16's)" % bf16[1],
                                "int8_ops_per_launch": tc_ops},
            "gpu_launches": (2 * B + 8) * args.steps,
            "clocks": split["clocks"],
            "vs_plain": round(s_value / value, 3),
            "both_passes": both_line,
        }
    res_match, n, gerbicz_ok, clocks = plain["res_match"], plain["res_checked"], plain["gerbicz_ok"], plain["clocks"]
    roe = np.array([roe]) if roe is not None else np.array([])

    # roofline of the dominant kernel: algorithmic bytes per launch = read + write of the
    # 8N-byte state = 16 N bytes, over its average launch time in the timed region
    dom = "pass2" if prof["pass2"][0] >= prof["pass1"][0] else "pass1"
    avg_ms = prof[dom][0] / max(prof[dom][1], 1)
    alg_bytes = 16 * N_8M
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic().get(dom)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # per timed step: modMul = pass1 IN, pass2 FWD, pass1 IN, pass2 MUL, pass1 OUT, carry fixup (6);
    # the block = pass1 IN, B x pass2, B-1 x pass1 FUSED, pass1 OUT, carry fixup (2B + 2)
    launches_per_step = 2 * B + 8
    line = {
        "metric": "ms/iter PRP @8M FFT: split-precision TC vs plain FP64, bit-exact res64",
        "value": round(value, 5), "unit": "ms/iter", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "PRP-3, E=136181029 (seeded prime in [136M,139M]), FFT 8M (W=H=2048), "
                               "plain FP64 form",
                   "E": E_8M, "N": N_8M, "block": B, "step": "modMul(check,data) + %d squarings" % B,
                   "timed_iterations": args.steps * B, "l2": "flushed (512 MiB write) between timed steps",
                   "timing": "step: CUDA events on the plan's stream around modMul + a graph-launched block; "
                             "kernels: per-launch %globaltimer stamps (first CTA start, last CTA end) in the same steps",
                   "parallelism": "replicas x%d" % world},
        "res64_match_golden": res_match, "res64_checked": n, "gerbicz_ok": bool(gerbicz_ok),
        "max_roe": round(float(roe.max()), 5) if roe.size else None,
        "split_tc": split_line,
        "kernel_ms": {k: round(v[0] / max(v[1], 1), 5) for k, v in prof.items()},
        "roofline": {"bound": "hbm", "kernel": "k_pass2" if dom == "pass2" else "k_pass1",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic, "alg_bytes_per_launch": alg_bytes},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_step / B, 5), "unit": "ms/iter",
                "h2d_bytes_per_step": 4 * NW_8M, "d2h_bytes_per_step": 4 * NW_8M + 16,
                "step": "owl_write_words from pinned host words (expanded on the device) + modMul + %d "
                        "squarings + owl_read_words into pinned host words (compacted on the device, "
                        "checksummed)" % B},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
    }
    if world == 1 and not args.no_configs:
        line["configs"] = other_configs(args, rank, world, local)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _gmp_ms_per_iter(E, iters):
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    lib.oracle_gmp_ms_per_iter.restype = ctypes.c_double
    lib.oracle_gmp_ms_per_iter.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    return lib.oracle_gmp_ms_per_iter(E, iters)


def gmp_batch_baseline(exps, procs=8, iters=3):
    """The CPU baseline of the batch: the GMP squaring loop (mod 2^E - 1) on `procs` processes of
    one core each. Each exponent's ms per iteration is sampled (`iters` squarings after 40 warm-up
    ones); a job of the same number of iterations for every exponent, spread evenly over the
    processes, runs at procs * len(exps) / sum(seconds per iteration) aggregate iterations/s."""
    import multiprocessing as mp
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True, capture_output=True)
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(procs) as pool:
        ms = pool.starmap(_gmp_ms_per_iter, [(E, iters) for E in exps])
    wall = time.perf_counter() - t0
    rate = procs * len(exps) / (sum(ms) * 1e-3)
    return {"value": round(rate, 1), "unit": "iter/s", "cores": procs, "kind": "port",
            "sample": "GMP 6.3 mpz squaring mod 2^E-1 (oracle/gmp_loop.c, the exact oracle; the reference's "
                      "OpenCL kernels have no CPU runtime here): %d squarings of each of the %d exponents after 40 "
                      "warm-up ones, %d processes x 1 core, %.1f s wall; aggregate = %d x %d / sum of s/iter"
                      % (iters, len(exps), procs, wall, procs, len(exps))}


def run_batch64(args, rank, world, local):
    """64 exponents log-uniform in [1M, 20M] (seeded), each at the smallest FFT with <= 19 bits per
    word, squared together as one CUDA-graph launch per 1,000-iteration block; aggregate iter/s and
    per-exponent res64 at every 1,000 iterations against the GMP table."""
    # the exponents and their res64 from the golden fixture (tests/golden/gen_golden.py batch64)
    items = (load_golden("batch64") or {"items": []})["items"]
    exps = [it["E"] for it in items]
    golden = {it["E"]: it["res64"] for it in items}
    # the same exponents to 10,000 iterations where that table is present
    for it in (load_golden("batch64_10k") or {"items": []})["items"]:
        if it["E"] in golden:
            golden[it["E"]] = it["res64"]
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        cpu = gmp_batch_baseline(exps)
    import torch
    import gpuowl_b200 as owl
    from gpuowl_b200 import build
    build.build()
    torch.cuda.set_device(local)
    B = args.block
    plans, bufs = [], []
    table = {}
    if getattr(args, "batch_shapes", "default") == "tuned":
        with open(os.path.join(ROOT, "gpuowl_b200", "tune_b200.json")) as f:
            table = json.load(f)
    for E in exps:
        N, W, H = owl.fft_choose(E, 19.0)
        cv = owl.COL_AUTO
        if str(N) in table:
            W, H = int(table[str(N)][0]), int(table[str(N)][1])
            cv = int(table[str(N)][5]) if len(table[str(N)]) >= 6 and table[str(N)][5] else owl.COL_AUTO
        p = owl.Plan(E, device=local, W=W, H=H, column_variant=cv)
        b = p.alloc()
        p.writeIn(b, [3] + [0] * (p.nwords - 1))
        plans.append(p)
        bufs.append(b)
    batch = owl.Batch(plans, device=local)
    res = {E: [] for E in exps}
    blk = [0]

    def square():
        # round-off measured on the reference's sample of iterations, as in the single-exponent line
        batch.square(bufs, B, roe=roe_measured(blk[0] * B, B))
        blk[0] += 1
        batch.sync()

    for _ in range(args.warmup):
        square()
        for p, b in zip(plans, bufs):
            res[p.E].append("%016x" % p.bufResidue(b))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        square()
        times.append(time.perf_counter() - t0)
        for p, b in zip(plans, bufs):
            res[p.E].append("%016x" % p.bufResidue(b))
    total = sum(times)
    points = sum(p.N for p in plans)
    groups = {}
    for p in plans:
        groups[(p.W, p.H)] = groups.get((p.W, p.H), 0) + 1
    checked = matched = 0
    for E in exps:
        g = golden.get(E, [])
        n = min(len(g), len(res[E]))
        checked += n
        matched += sum(1 for i in range(n) if g[i] == res[E][i])
    shapes = sorted({(p.N) for p in plans})
    line = {"metric": "aggregate iter/s, 64 uneven exponents (batched)", "value": round(len(exps) * B * args.steps / total, 1),
            "unit": "iter/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "64 exponents log-uniform in [1M,20M] (seed 20261203), FFT per exponent at <=19 "
                                   "bits/word, one graph launch per %d-iteration block" % B,
                       "fft_sizes": shapes, "timing": "wall clock around launch + synchronize",
                       "shapes": "W x H split and column variant per FFT size: %s" % (
                           "the tuner's table (gpuowl_b200/tune_b200.json)"
                           if getattr(args, "batch_shapes", "default") == "tuned" else "the library's defaults"),
                       "launches": "plans of one W x H shape (%d shapes) share one launch per pass: %d kernels per "
                                   "iteration for the %d plans" % (len(groups), sum(2 * ((n + 15) // 16)
                                                                                   for n in groups.values()),
                                                                  len(plans))},
            "res64_checked": checked, "res64_matched": matched,
            "points_per_iteration": points,
            "ns_per_mpoint_iter": round(1e9 * total / (args.steps * B) / (points / 1e6), 2),
            "cpu_baseline": cpu}
    batch.close()
    for p in plans:
        p.close()
    return line


# the other PRP configurations: golden table, shape (0 = the library's choice), range of E
PRP_CONFIGS = {
    "prp20m": ("prp_20m", 4096, 2560, "20M (5*2^22)", "[330M,335M]",
               "proof power 8 configured (its first residue point, at E/256, lies beyond the timed "
               "iterations; tests/test_large.py runs the PRP driver with it)"),
    "prp256k": ("prp_256k", 0, 0, "256K", "[4.8M,5.0M]", ""),
}


def run_prp_config(args, rank, world, local):
    """PRP-3 at another configuration (PRP_CONFIGS) for E the seeded prime of its range: the same timed
    steps as the 8M line (modMul(check, data) + one graph-launched block, CUDA events on the plan's
    stream, L2 flushed between steps), res64 at every 1,000 iterations against the GMP golden table
    and a Gerbicz check at the end. At 20M the split-precision form runs the same steps after the
    plain one (the line's split_tc block)."""
    import torch
    import gpuowl_b200 as owl
    from gpuowl_b200 import build
    build.build()
    torch.cuda.set_device(local)
    gname, W, H, label, rng_txt, note = PRP_CONFIGS[args.workload]
    g = load_golden(gname)
    E = g["E"]
    if not W:
        _, W, H = owl.fft_choose(E)
    N = 2 * W * H
    B = args.block
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    import numpy as np

    def measure(split):
        """Warm-up and timed steps of one form of the column pass: (step times, per-kernel sums,
        res64 per block, round-off samples, Gerbicz result, clocks)."""
        plan = owl.Plan(E, device=local, W=W, H=H, split=split)
        stream = torch.cuda.ExternalStream(plan.stream(), device=torch.device("cuda", local))
        data, check, aux = plan.alloc(), plan.alloc(), plan.alloc()
        plan.writeIn(data, [3] + [0] * (plan.nwords - 1))
        plan.writeIn(check, [1] + [0] * (plan.nwords - 1))
        res, step_ms = [], []
        prof = {"pass2": [0.0, 0], "pass1": [0.0, 0], "edge": [0.0, 0]}
        blk = [0]

        def step():
            k = blk[0] * B
            blk[0] += 1
            plan.modMul(check, data)
            return plan.profile_square(data, B, roe=roe_measured(k, B))

        for _ in range(args.warmup):
            step()
            res.append("%016x" % plan.bufResidue(data))
        roe_warm = plan.readROE()
        torch.cuda.synchronize()
        with ClockSampler(local) as clocks:
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                pr = step()
                e1.record(stream)
                e1.synchronize()
                step_ms.append(e0.elapsed_time(e1))
                for k, (ms, n) in pr.items():
                    prof[k][0] += ms
                    prof[k][1] += n
                res.append("%016x" % plan.bufResidue(data))
        roe = np.concatenate([roe_warm, plan.readROE()])
        plan.squareLoop(aux, check, B, mul3=True)
        plan.modMul(check, data)
        gerbicz_ok = plan.isEqual(check, aux)
        plan.close()
        return step_ms, prof, res, roe, gerbicz_ok, clocks.summary()

    step_ms, prof, res, roe, gerbicz_ok, clocks = measure(False)
    split_line = None
    if args.workload == "prp20m" and not args.no_split:
        s_ms, s_prof, s_res, s_roe, s_gerbicz, s_clocks = measure(True)
        s_n = min(len(s_res), len(g["res64"])) if g else 0
        s_value = sum(s_ms) / (args.steps * B)
        tc_ms = s_prof["pass2"][0] / max(s_prof["pass2"][1], 1)
        # INT8 work of one k_pass2_tc launch at H = 2560: W/2 CTAs x 2 directions x 28 digit-plane
        # products of a 128 x 80 (outputs) x 80 (inputs) GEMM; issued with K padded to 96
        tc_ops = 2.0 * (W // 2) * 2 * 28 * 128 * 80 * 80
        bf16 = measured_bf16()
        split_line = {
            "form": "split-precision: 40-point column stages as INT8 tcgen05 GEMMs on 7 base-256 digit planes",
            "ms_per_iter": round(s_value, 5), "ms_per_step": round(sum(s_ms) / args.steps, 4),
            "kernel_ms": {k: round(v[0] / max(v[1], 1), 5) for k, v in s_prof.items()},
            "max_roe": round(float(s_roe.max()), 5) if s_roe.size else None,
            "res64_match_golden": (s_res[:s_n] == g["res64"][:s_n]) if g else None, "res64_checked": s_n,
            "gerbicz_ok": bool(s_gerbicz),
            "tensor_roofline": {"bound": "tensor", "kernel": "k_pass2_tc",
                                "achieved": round(tc_ops / (tc_ms * 1e-3) / 1e12, 2),
                                "peak": round(2 * bf16[0], 1), "unit": "TOP/s (int8)",
                                "frac": round(tc_ops / (tc_ms * 1e-3) / 1e12 / (2 * bf16[0]), 4),
                                "peak_kind": "2 x %s bf16 dense (int8 dense rate is twice bf16's)" % bf16[1],
                                "int8_ops_per_launch": tc_ops},
            "gpu_launches": (2 * B + 8) * args.steps,
            "clocks": s_clocks,
            "vs_plain": round(s_value / (sum(step_ms) / (args.steps * B)), 3),
        }
    n = min(len(res), len(g["res64"])) if g else 0
    total_ms = sum(step_ms)
    dom = "pass2" if prof["pass2"][0] >= prof["pass1"][0] else "pass1"
    avg_ms = prof[dom][0] / max(prof[dom][1], 1)
    achieved = 16 * N / (avg_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    if rank != 0:
        return None
    line = {
        "metric": "ms/iter PRP @%s FFT, bit-exact res64" % label,
        "value": round(total_ms / (args.steps * B), 5), "unit": "ms/iter", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "PRP-3, E=%d (seeded prime in %s), FFT %s (W=%d, H=%d), plain FP64 form"
                               % (E, rng_txt, label, W, H),
                   "E": E, "N": N, "block": B, "step": "modMul(check,data) + %d squarings" % B,
                   "timed_iterations": args.steps * B, "l2": "flushed (512 MiB write) between timed steps",
                   "note": note},
        "res64_match_golden": (res[:n] == g["res64"][:n]) if g else None, "res64_checked": n,
        "gerbicz_ok": bool(gerbicz_ok), "max_roe": round(float(roe.max()), 5) if roe.size else None,
        "kernel_ms": {k: round(v[0] / max(v[1], 1), 5) for k, v in prof.items()},
        "roofline": {"bound": "hbm", "kernel": "k_pass2" if dom == "pass2" else "k_pass1",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": profiled_traffic(args.workload[3:]).get(dom),
                     "alg_bytes_per_launch": 16 * N},
        "gpu_launches": (2 * B + 8) * args.steps,
        "clocks": clocks,
        "split_tc": split_line,
    }
    return line


# the short runs of the other configurations carried by the default (8M, one GPU) line:
# (workload, timed steps, warm-up steps); each is the same code path as --workload <name>
SUB_CONFIGS = (("prp20m", 2, 3), ("prp256k", 5, 3), ("batch64", 3, 3))


def other_configs(args, rank, world, local):
    """The lines of the 20M, 256K and batched configurations, each from a short run of its own
    workload (a few 1,000-iteration blocks, res64 against its golden table), so that one default
    run measures every configuration."""
    out = {}
    for name, steps, warmup in SUB_CONFIGS:
        sub = argparse.Namespace(**vars(args))
        sub.workload, sub.steps, sub.warmup = name, steps, warmup
        run = run_batch64 if name == "batch64" else run_prp_config
        out[name] = run(sub, rank, world, local)
    return out


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.workload == "batch64" or args.workload in PRP_CONFIGS:
        run = run_batch64 if args.workload == "batch64" else run_prp_config
        line = run(args, rank, world, local)
        if line is not None and rank == 0:
            print(json.dumps(line), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
