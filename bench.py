#!/usr/bin/env python
"""AFMM2D matvec benchmark on B200.

One step = one batched matvec Y = K Q over the workload's N points with
--nrhs right-hand sides (default 16) in the mixed-precision path, with the
assembled operators resident in HBM; value = N * nrhs / step time.  The FP64
plain path and the single-RHS mixed path are timed beside it.  The default
workload is the N = 4,194,304 Gaussian-mixture problem (16 components,
sigma 0.02, kernel 1/r, M = 64, TOL_POW = 6); inputs are seeded synthetic
data.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: the path does not shard (one problem per GPU), so N ranks run N
independent replicas; value = total points*RHS per second over all ranks,
timed as the max over ranks.  --impl reference times the reference's own CPU
code (compiled from its sources into oracle/_ref) on a bounded sample of the
same workload on the host cores; under torchrun only rank 0 runs it.
"""
import argparse
import csv
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "points*RHS/s per matvec at N=4M (mixture, 1/r, TOL 6), mixed batched vs FP64 GPU"


def metric_name(workload, N, p, nrhs):
    """The headline metric string for the default workload; for another one
    the same quantity named by that workload's own sizes."""
    if workload == "mixture4m" and N == 1 << 22 and nrhs == 16:
        return METRIC
    return (f"points*RHS/s per matvec at N={N} ({workload}, {p['kernel']}, TOL {p['tol']}), "
            f"mixed batched ({nrhs} RHS) vs FP64 GPU")
UNIT = "points*RHS/s"
CPU_SAMPLE_N = 65536


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixture4m")
    ap.add_argument("--N", type=int, default=None, help="override N (same distribution)")
    ap.add_argument("--nrhs", type=int, default=16, help="right-hand sides of the batched (headline) path")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=CPU_SAMPLE_N,
                    help="points of the reference CPU run (the workload's N: full size, with a parity check of the "
                         "FP64 GPU result against the reference's output)")
    ap.add_argument("--profile-once", action="store_true", help="only run setup + 2 matvecs (for ncu)")
    ap.add_argument("--tuning", default="auto", choices=["auto", "default"],
                    help="auto: run the library's autotuner during setup (default); default: built-in parameters")
    ap.add_argument("--shard", action="store_true",
                    help="under torchrun: one problem split over the ranks by subtrees (strong scaling) instead of "
                         "one replica per rank")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="tuning value applied after --tuning (repeatable; keys as AFMM.tuning(), e.g. p2p_tc=1)")
    return ap.parse_args()


def tuning_overrides(args):
    out = {}
    for kv in args.set:
        k, _, v = kv.partition("=")
        out[k.strip()] = int(v, 0)
    return out


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(values, dist, device):
    """Element-wise max of a list of floats over all ranks (the step time of a
    replicas run is the slowest rank's)."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        rows = [r for r in csv.reader(self.f) if len(r) >= 9]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def scaled_traffic(kernel, algorithmic_bytes):
    """DRAM bytes per launch for `kernel`, scaled from an ncu capture of a
    smaller case of the same workload (profiles/traffic.json holds the
    captured dram__bytes_read.sum + dram__bytes_write.sum and the capture's
    algorithmic bytes); None if no capture is recorded."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f)[kernel]
        return algorithmic_bytes * d["dram_bytes"] / d["algorithmic_bytes"]
    except (OSError, KeyError, ValueError, ZeroDivisionError):
        return None


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, "fallback"


def cpu_reference(name, n, steps, warmup):
    """The reference's own OpenMP path (oracle/_ref) on a bounded sample."""
    from afmm2d_b200 import workloads
    from oracle_lib import RefLib
    if not RefLib.available():
        return None
    pts, q, p = workloads.make(name, N=n)
    if q.ndim > 1:
        q = np.ascontiguousarray(q[:, 0])
    t0 = time.perf_counter()
    r = RefLib(pts, p["M"], p["tol"], p["kernel"])
    r.assemble()
    setup = time.perf_counter() - t0
    for _ in range(warmup):
        r.matvec(q)
    t0 = time.perf_counter()
    for _ in range(steps):
        y = r.matvec(q)
    dt = (time.perf_counter() - t0) / steps
    threads = r.lib.ref_num_threads()
    return {"value": n / dt, "unit": UNIT, "cores": int(threads), "kind": "reference",
            "sample": f"{name} at N={n} (same distribution, kernel, M, TOL), {steps} matvecs after {warmup} "
                      f"warm-up, OpenMP {threads} threads; reference setup {setup:.1f} s",
            "ms_per_step": dt * 1e3, "setup_s": setup, "y": y}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    n = args.N or CPU_SAMPLE_N
    res = cpu_reference(args.workload, n, max(args.steps, 1), max(args.warmup, 1))
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libafmm2d_ref.so was not built"}))
        return
    from afmm2d_b200 import workloads
    wp = workloads.WORKLOADS[args.workload]
    metric = metric_name(args.workload, args.N or wp["N"], wp, getattr(args, "nrhs", 16))
    line = {"impl": "reference", "metric": metric, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": args.workload, "N": n, "sample_of_N": 1 << 22},
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import afmm2d_b200 as A
    from afmm2d_b200 import workloads

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    R = args.nrhs
    pts, q, p = workloads.make(args.workload, N=args.N)
    N = len(pts)
    Q = np.random.Generator(np.random.PCG64(p["seed"] + 1)).standard_normal((N, R))
    if q.ndim == 2:  # workloads with several charge vectors (gauss1m: 64)
        k = min(R, q.shape[1])
        Q[:, :k] = q[:, :k]
    else:
        Q[:, 0] = q
    # warm process: CUDA context and the library's kernels loaded by a small
    # problem of the same kernel first; the cold figure of a fresh process is
    # reported beside it
    t0 = time.perf_counter()
    w_pts, _, w_p = workloads.make(args.workload, N=8192)
    w = A.AFMM(8192, w_p["M"], w_p["tol"], w_pts, kernel=p["kernel"])
    w.assemble()
    w.computeMatVecProduct(np.ones(8192))
    w.close()
    torch.cuda.synchronize()
    warm_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    a = A.AFMM(N, p["M"], p["tol"], pts, kernel=p["kernel"])
    if tuning_overrides(args).get("m2l_tc") == 2:
        a.set_m2l_fixed_point(2)  # the integer tcgen05 M2L applies byte planes kept at assembly
    a.assemble()
    setup_s = time.perf_counter() - t0
    counts = a.counts()
    dev = f"cuda:{local}"
    stream = torch.cuda.ExternalStream(a.stream())
    dQ = torch.from_numpy(np.asfortranarray(Q).T.copy()).to(dev)  # row c = column c (column-major N x R)
    dY = torch.empty_like(dQ)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    paths = {"fp64": ("fp64", 1), "mixed": ("mixed", 1), "batched": ("mixed", R), "fp64_batched": ("fp64_batched", R)}

    def call(name):
        prec, nr = paths[name]
        a.matvec_device(dQ.data_ptr(), dY.data_ptr(), nr, N, prec)

    def timed(name, steps, warm, stage_acc=None):
        """Mean device ms per step (CUDA events on the handle's stream, L2
        flushed before every step).  With stage_acc, the library's per-stage
        events (one pair of marks around every kernel stage, on the same
        stream) are recorded inside the timed steps and summed into it."""
        for _ in range(warm):
            call(name)
        ms = []
        if stage_acc is not None:
            a.set_profiling(True)
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call(name)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            if stage_acc is not None:
                for k, v in a.stage_times().items():
                    stage_acc[k] = stage_acc.get(k, 0.0) + v / steps
        if stage_acc is not None:
            a.set_profiling(False)
        return float(np.mean(ms))

    def serial_stages(name, steps):
        """Stage times of `steps` further (untimed) steps with the near field
        run after the far field on the handle's stream, so that each stage
        is its kernels' own duration (in the timed steps the batched near
        field runs beside the far field on a second stream)."""
        acc = {}
        a.set_profiling(2)
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            call(name)
            stream.synchronize()
            for k, v in a.stage_times().items():
                acc[k] = acc.get(k, 0.0) + v / steps
        a.set_profiling(False)
        return acc

    overrides = tuning_overrides(args)
    if args.profile_once:
        if args.tuning == "auto":
            a.autotune()
        if overrides:
            a.set_tuning(**overrides)
        for name in paths:
            call(name)
        torch.cuda.synchronize()
        return
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    # every path with the built-in launch parameters first, then (setup, not
    # timed) the autotuner on this problem; the reported paths use its choice
    t_default = {name: timed(name, args.steps, args.warmup) for name in paths}
    tuning, tune_s = a.tuning(), 0.0
    if args.tuning == "auto":
        t0 = time.perf_counter()
        tuning, _ = a.autotune()
        tune_s = time.perf_counter() - t0
    if overrides:
        a.set_tuning(**overrides)
        tuning = a.tuning()
    t_dev = {}
    launches = {}
    stages = {}
    stages_serial = {}
    for name in paths:
        l0 = a.launch_count()
        stages[name] = {}
        t_dev[name] = timed(name, args.steps, args.warmup, stages[name])
        launches[name] = (a.launch_count() - l0) // (args.steps + args.warmup)
        if "p2p_kernel" in stages[name]:
            stages_serial[name] = serial_stages(name, args.steps)
    torch.cuda.synchronize()
    clocks = clk.stop()
    # accuracy: the batched and single-RHS mixed paths against the FP64 path
    y64 = np.empty((N, R))
    for c in range(R):
        a.matvec_device(dQ[c].data_ptr(), dY[c].data_ptr(), 1, N, "fp64")
    y64[:] = dY.cpu().numpy().T
    err_dense = a.evaluateError(nsample=16, seed=1234)
    call("batched")
    yb = dY.cpu().numpy().T
    err_batched = float(np.max([np.linalg.norm(yb[:, c] - y64[:, c]) / np.linalg.norm(y64[:, c]) for c in range(R)]))
    call("mixed")
    err_mixed = float(np.linalg.norm(dY[0].cpu().numpy() - y64[:, 0]) / np.linalg.norm(y64[:, 0]))
    call("fp64_batched")
    yb64 = dY.cpu().numpy().T
    err_fp64b = float(np.max([np.linalg.norm(yb64[:, c] - y64[:, c]) / np.linalg.norm(y64[:, c]) for c in range(R)]))
    # end to end through the C ABI with pinned host buffers (the headline workload)
    hQ = torch.from_numpy(np.asfortranarray(Q).T.copy()).pin_memory()
    hY = torch.empty_like(hQ).pin_memory()
    for _ in range(args.warmup):
        a.matvec_host_ptr(hQ.data_ptr(), hY.data_ptr(), R, N, "mixed")
    e2e = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        a.matvec_host_ptr(hQ.data_ptr(), hY.data_ptr(), R, N, "mixed")
        e2e.append(time.perf_counter() - t1)
    t_e2e = float(np.mean(e2e))
    names = list(paths)
    red = max_over_ranks([t_dev[n] for n in names] + [t_e2e], dist, dev)
    t_dev = dict(zip(names, red[:-1]))
    t_e2e = red[-1]
    value = world * N * R / (t_dev["batched"] * 1e-3)
    hbm, bf16, peak_kind = load_peaks()
    fp64_peak, fp32_peak = A.measure_fma_peaks()
    dmma_peak, dfma_peak, both_peak = A.measure_fp64_pipes()
    # roofline of the dominant kernel of the headline (batched) path, its
    # duration averaged over the timed steps (stage events on the launching
    # stream); algorithmic bytes / flops per launch from the assembled counts
    # the near field runs on a second stream beside the far field: in the
    # timed steps its "p2p_kernel" span shares the GPU with the far field and
    # the "p2p" mark on the launching stream is only the far field's wait for
    # it, so its own duration comes from the serial profile
    sb = dict(stages["batched"])
    near_src = "timed steps"
    if "p2p_kernel" in sb:
        sb.pop("p2p_kernel")
        sb["p2p"] = stages_serial["batched"]["p2p"]
        near_src = ("near-field kernel alone: profiled steps with the near field after the far field "
                    "(in the timed steps it runs beside the far field on a second stream)")
    dom = max((k for k in sb if k not in ("end", "h2d", "d2h")), key=lambda k: sb[k])
    rows = counts["sum_rank"]
    fixed = a.m2l_fixed_point()
    nbox = sum(4 ** j for j in range(2, counts["nlevels"] + 1))
    if dom == "m2l" and fixed:
        byts = counts["m2l_entries"] * 4 + nbox * 40 * 16 + 2 * rows * R * 8
        roof = {"bound": "hbm",
                "kernel": "k_m2l_stored_mma<Q32> (32-bit fixed-point M2L blocks, FP64 tensor-core tiles)",
                "unit": "GB/s", "achieved": byts / (sb[dom] * 1e-3) / 1e9, "peak": hbm, "peak_kind": peak_kind,
                "algorithmic_bytes": byts,
                "byte_definition": "4 B per stored M2L entry (read once) + 16 B decode constants per (box, slot) + "
                                   "nrhs*8 B per skeleton row in and out",
                "ms": sb[dom]}
        roof["traffic"] = scaled_traffic("k_m2l_stored_mma_q32", byts)
    elif dom == "m2l":
        byts = counts["m2l_entries"] * 8 + 2 * rows * R * 8
        roof = {"bound": "hbm", "kernel": "k_m2l_stored_mma (stored FP64 M2L blocks, FP64 tensor-core tiles)",
                "unit": "GB/s", "achieved": byts / (sb[dom] * 1e-3) / 1e9, "peak": hbm, "peak_kind": peak_kind,
                "algorithmic_bytes": byts,
                "byte_definition": "8 B per stored M2L entry (read once) + nrhs*8 B per skeleton row in and out",
                "ms": sb[dom]}
        roof["traffic"] = scaled_traffic("k_m2l_stored_mma", byts)
    elif dom == "p2p":
        flops = 2.0 * R * counts["near_evals"]
        roof = {"bound": "fp32", "kernel": "k_p2p_mma (near field, FP32 entries on TF32x3 tensor-core tiles)",
                "unit": "TFLOP/s", "achieved": flops / (sb[dom] * 1e-3) / 1e12, "peak": fp32_peak,
                "peak_kind": "measured live (register-only FP32 FMA loop)", "traffic": None,
                "algorithmic_flops": flops, "flop_definition": "2*nrhs flops per near-field pair", "ms": sb[dom],
                "ms_source": near_src}
    else:
        byts = counts["l2p_entries"] * 8 + 2 * rows * R * 8
        roof = {"bound": "hbm", "kernel": dom, "unit": "GB/s", "achieved": byts / (sb[dom] * 1e-3) / 1e9,
                "peak": hbm, "peak_kind": peak_kind, "traffic": None, "algorithmic_bytes": byts, "ms": sb[dom]}
    roof["frac"] = roof["achieved"] / roof["peak"] if roof.get("peak") else None
    # the FP64 path's stored M2L is HBM-bound
    s64 = stages["fp64"]
    m2l_bytes = counts["m2l_entries"] * 8
    roof64 = {"bound": "hbm", "kernel": "k_m2l_apply_w (stored FP64 M2L, one RHS, warp per row chunk)", "unit": "GB/s",
              "achieved": m2l_bytes / (s64["m2l"] * 1e-3) / 1e9, "peak": hbm, "peak_kind": peak_kind,
              "algorithmic_bytes": m2l_bytes, "ms": s64["m2l"]}
    roof64["frac"] = roof64["achieved"] / hbm
    # the batched stored M2L on FP64 tensor tiles is bound by the FP64
    # datapath, not by HBM: its FP64 flops against the live DMMA peak
    roof_dmma = None
    if dom == "m2l" and not tuning.get("m2l_tc") and not tuning.get("otf_batched"):
        fl = 2.0 * R * counts["m2l_entries"]
        roof_dmma = {"bound": "tensor", "kernel": "k_m2l_stored_mma (FP64 mma.sync m8n8k4 tiles)", "unit": "TFLOP/s",
                     "achieved": fl / (sb[dom] * 1e-3) / 1e12, "peak": dmma_peak,
                     "peak_kind": "measured live (register-only m8n8k4 DMMA loop)", "algorithmic_flops": fl,
                     "flop_definition": "2*nrhs flops per stored M2L entry (tile padding not counted)",
                     "ms": sb[dom]}
        roof_dmma["frac"] = roof_dmma["achieved"] / dmma_peak
    # the headline roofline is the binding one: of the kernel's two floors
    # (algorithmic bytes / HBM peak, FP64 tensor flops / DMMA peak) the longer,
    # i.e. the larger fraction of the same duration; the other stays beside it
    roof_other = None
    if roof_dmma is not None and roof.get("frac") is not None and roof_dmma["frac"] > roof["frac"]:
        roof_dmma["traffic"] = roof.get("traffic")
        roof_dmma["binding"] = (f"FP64 tensor floor {roof_dmma['algorithmic_flops'] / (dmma_peak * 1e12) * 1e3:.2f} ms "
                                f"> HBM floor {roof['algorithmic_bytes'] / (roof['peak'] * 1e9) * 1e3:.2f} ms")
        roof_other, roof = roof, roof_dmma
    line = {"metric": metric_name(args.workload, N, p, R), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_dev["batched"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "N": N, "kernel": p["kernel"], "M": p["M"], "TOL_POW": p["tol"],
                       "nrhs": R, "precision": "mixed, batched", "m2l_blocks": "fixed32" if fixed else "fp64",
                       "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"replicas x{world}"},
            "paths": {name: {"ms_per_step": t_dev[name], "nrhs": paths[name][1],
                             "points_rhs_per_s": world * N * paths[name][1] / (t_dev[name] * 1e-3),
                             "gpu_launches": launches[name]} for name in paths},
            "speedup_batched_vs_fp64": (N * R / t_dev["batched"]) / (N / t_dev["fp64"]),
            "rel_err_batched_vs_fp64_max_col": err_batched, "rel_err_mixed_vs_fp64": err_mixed,
            "rel_err_fp64_batched_vs_fp64_max_col": err_fp64b,
            "rel_err_fp64_vs_dense_16_leaves": err_dense,
            "setup_s": setup_s, "setup_process_warmup_s": warm_s, "setup": a.setup_times(), "stages_ms": stages,
            "stages_serial_ms": stages_serial,
            "tuning": {"mode": args.tuning, "overrides": overrides, "values": tuning, "autotune_s": tune_s,
                       "default_ms_per_step": t_default},
            "counts": counts,
            "roofline": roof, "roofline_fp64_m2l": roof64, "fma_peaks_tflops": {"fp64": fp64_peak, "fp32": fp32_peak},
            "fp64_pipes_tflops": {"dmma": dmma_peak, "dfma": dfma_peak, "dmma_and_dfma_together": both_peak},
            "roofline_dmma_m2l": roof_dmma, "roofline_hbm_m2l": roof_other,
            "clocks": clocks, "gpu_launches": int(launches["batched"]),
            "e2e": {"value": world * N * R / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * N * R,
                    "d2h_bytes_per_step": 8 * N * R, "ms_per_step": t_e2e * 1e3, "nrhs": R}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        full = args.cpu_sample >= N
        # a bounded sample: a few matvecs of the 65,536-point default; one at full size
        cb = cpu_reference(args.workload, min(args.cpu_sample, N), 1 if full else 5, 0 if full else 1)
        if cb:
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            line["cpu_baseline"]["setup_s"] = cb["setup_s"]
            line["fp64_gpu_vs_cpu_reference_matvec"] = (N / (t_dev["fp64"] * 1e-3)) / cb["value"]
            n_s = min(args.cpu_sample, N)
            if n_s < N:
                # the FP64 GPU path on the reference's own sample (equal N)
                s_pts, s_q, s_p = workloads.make(args.workload, N=n_s)
                s_q = s_q[:, 0] if s_q.ndim == 2 else s_q
                sa = A.AFMM(n_s, s_p["M"], s_p["tol"], s_pts, kernel=s_p["kernel"])
                sa.assemble()
                dq_s = torch.from_numpy(np.ascontiguousarray(s_q)).to(dev)
                dy_s = torch.empty_like(dq_s)
                st_s = torch.cuda.ExternalStream(sa.stream())
                for _ in range(3):
                    sa.matvec_device(dq_s.data_ptr(), dy_s.data_ptr(), 1, n_s, "fp64")
                ms_s = []
                for _ in range(10):
                    with torch.cuda.stream(st_s):
                        flush.zero_()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(st_s)
                    sa.matvec_device(dq_s.data_ptr(), dy_s.data_ptr(), 1, n_s, "fp64")
                    e1.record(st_s)
                    e1.synchronize()
                    ms_s.append(e0.elapsed_time(e1))
                t_s = float(np.mean(ms_s))
                line["fp64_gpu_same_n"] = {"N": n_s, "ms_per_step": t_s, "points_per_s": n_s / (t_s * 1e-3),
                                           "vs_cpu_reference": (n_s / (t_s * 1e-3)) / cb["value"]}
                sa.close()
            if full:
                yr = cb["y"]
                line["rel_err_fp64_vs_reference"] = float(np.linalg.norm(y64[:, 0] - yr) / np.linalg.norm(yr))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    a.close()


def run_many(args):
    """The many-problem workload: 256 independent problems (N log-uniform in
    2,048..65,536, uniform points, log, M = 32, TOL 8).  One step = one FP64
    matvec of every problem through AFMMSet (fused launches replayed from one
    CUDA graph); a loop of per-problem FP64 matvecs is timed beside it.  Under
    torchrun the problems are sharded: rank r takes problems r, r + world,
    ... (no communication), so the total work is fixed (strong scaling)."""
    import torch
    import afmm2d_b200 as A
    from afmm2d_b200 import workloads

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    probs_all, p = workloads.many_problems()
    total_all = int(sum(len(pts) for pts, _ in probs_all))
    probs = [probs_all[k] for k in range(rank, len(probs_all), world)]
    t0 = time.perf_counter()
    hs = []
    for pts, _ in probs:
        h = A.AFMM(len(pts), p["M"], p["tol"], pts, kernel=p["kernel"])
        h.assemble()
        hs.append(h)
    st = A.AFMMSet(hs)
    setup_s = time.perf_counter() - t0
    total = st.total
    dev = f"cuda:{local}"
    q = torch.from_numpy(np.concatenate([qk for _, qk in probs])).to(dev)
    y = torch.empty_like(q)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.ExternalStream(st.stream())

    def timed(fn, s):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(s):
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.mean(ms))

    if dist:
        dist.barrier()
    clk = ClockSampler(local)
    clk.start()
    stages = {}

    def set_step():
        st.matvec_device(q.data_ptr(), y.data_ptr())
        for k, v in st.stage_times().items():
            stages[k] = stages.get(k, 0.0) + v

    t_set = timed(set_step, stream)
    nst = args.warmup + args.steps
    stages = {k: v / nst for k, v in stages.items()}
    # per-problem loop: each handle's own FP64 matvec through the C ABI (each
    # call runs on its handle's stream and returns when done: wall clock)
    offs = st.offsets
    esz = q.element_size()

    def loop():
        for k, h in enumerate(hs):
            h.matvec_device(q.data_ptr() + esz * int(offs[k]), y.data_ptr() + esz * int(offs[k]), 1, h.N, "fp64")

    for _ in range(args.warmup):
        loop()
    torch.cuda.synchronize()
    tl = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loop()
        tl.append(time.perf_counter() - t1)
    t_loop = float(np.mean(tl)) * 1e3
    torch.cuda.synchronize()
    clocks = clk.stop()
    hq = q.cpu().pin_memory()
    hy = torch.empty_like(hq).pin_memory()
    for _ in range(args.warmup):
        st._call("afmm_set_matvec", ctypes.c_void_p(hq.data_ptr()), ctypes.c_void_p(hy.data_ptr()), 0)
    e2e = []
    for _ in range(max(args.steps, 1)):
        t1 = time.perf_counter()
        st._call("afmm_set_matvec", ctypes.c_void_p(hq.data_ptr()), ctypes.c_void_p(hy.data_ptr()), 0)
        e2e.append(time.perf_counter() - t1)
    t_e2e = float(np.mean(e2e))
    # one problem's set output against its own FP64 matvec
    yk = hs[0].computeMatVecProduct(probs[0][1], "fp64")
    same = bool(np.array_equal(hy.numpy()[offs[0]:offs[1]], yk))
    red = max_over_ranks([t_set, t_loop, t_e2e], dist, dev)
    t_set, t_loop, t_e2e = red
    per, _ = st.launches()
    cnt = {k: int(np.sum([h.counts()[k] for h in hs])) for k in ("m2l_entries", "l2p_entries", "near_evals")}
    hbm, _, peak_kind = load_peaks()
    fp64_peak, _ = A.measure_fma_peaks()
    dom = max(stages, key=lambda k: stages[k])
    if dom == "p2p":
        flops = 8.0 * cnt["near_evals"]
        roof = {"bound": "fp64", "kernel": "k_set_p2p64 (near field, FP64 kernel entries)", "unit": "TFLOP/s",
                "achieved": flops / (stages[dom] * 1e-3) / 1e12, "peak": fp64_peak,
                "peak_kind": "measured live (register-only FP64 FMA loop)", "algorithmic_flops": flops,
                "flop_definition": "8 FP64 flops per pair (2 differences, R2, multiply-add; the log counted as 1)",
                "traffic": None, "ms": stages[dom]}
    else:
        byts = float(cnt["m2l_entries"] * 8 if dom == "m2l" else cnt["l2p_entries"] * 8)
        roof = {"bound": "hbm", "kernel": "k_set_" + dom, "unit": "GB/s", "achieved": byts / (stages[dom] * 1e-3) / 1e9,
                "peak": hbm, "peak_kind": peak_kind, "algorithmic_bytes": byts, "traffic": None, "ms": stages[dom]}
    roof["frac"] = roof["achieved"] / roof["peak"]
    line = {"metric": "points/s per FP64 matvec of 256 independent problems (N 2,048..65,536, log, TOL 8)",
            "value": total_all / (t_set * 1e-3), "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_set, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "many", "problems": len(probs_all), "points": total_all, "kernel": p["kernel"],
                       "M": p["M"], "TOL_POW": p["tol"], "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"problems sharded over {world} GPU(s)", "problems_per_rank0": len(hs)},
            "loop_ms_per_step": t_loop, "loop_timing": "wall clock of 256 afmm_matvec FP64 calls",
            "speedup_set_vs_loop": t_loop / t_set,
            "set_output_equals_own_fp64_matvec": same, "setup_s": setup_s,
            "gpu_launches": per, "graph_launches_per_step": 1, "stages_ms": stages, "counts": cnt,
            "roofline": roof,
            "clocks": clocks,
            "e2e": {"value": total_all / t_e2e, "unit": "points/s", "h2d_bytes_per_step": 8 * total_all,
                    "d2h_bytes_per_step": 8 * total_all, "ms_per_step": t_e2e * 1e3}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle_lib import RefLib
        if RefLib.available():
            done, spent, tm = 0, 0.0, 0.0
            for pts, qk in probs:
                t1 = time.perf_counter()
                r = RefLib(pts, p["M"], p["tol"], p["kernel"])
                r.assemble()
                t2 = time.perf_counter()
                r.matvec(qk)
                t3 = time.perf_counter()
                tm += t3 - t2
                spent += t3 - t1
                done += len(pts)
                if spent > 15.0:
                    break
            line["cpu_baseline"] = {"value": done / tm, "unit": "points/s", "cores": int(r.lib.ref_num_threads()),
                                    "kind": "reference",
                                    "sample": f"the first problems of the set ({done} points), one matvec each"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    st.close()


def run_sharded(args):
    """--shard: one problem over all ranks.  Every rank builds the whole
    problem, computes its subtrees' share of each 16-RHS mixed matvec
    (afmm_set_shard) and one NCCL all-reduce sums the shards; value = N * nrhs
    / the max over ranks of the step time (strong scaling: the work is the
    problem's whatever the rank count).  e2e adds the host copies of the
    charges (every rank) and of the result."""
    import datetime

    import torch
    import torch.distributed as dist

    import afmm2d_b200 as A
    from afmm2d_b200 import shard, workloads

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:  # one shard: the whole problem through the same code
        dist.init_process_group("gloo", init_method="file://" + tempfile.mktemp(), rank=0, world_size=1)
    R = args.nrhs
    pts, q, p = workloads.make(args.workload, N=args.N)
    N = len(pts)
    Q = np.random.Generator(np.random.PCG64(p["seed"] + 1)).standard_normal((N, R))
    t0 = time.perf_counter()
    a = A.AFMM(N, p["M"], p["tol"], pts, kernel=p["kernel"])
    a.assemble()
    setup_s = time.perf_counter() - t0
    if args.tuning == "auto":
        a.autotune()
    overrides = tuning_overrides(args)
    if overrides:
        a.set_tuning(**overrides)
    sm = shard.ShardedMatvec(a)
    dev = f"cuda:{local}"
    hQ = torch.from_numpy(np.asfortranarray(Q).T.copy()).pin_memory()
    hY = torch.empty_like(hQ).pin_memory()
    dQ = hQ.to(dev)
    dY = torch.empty_like(dQ)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        dist.barrier()
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.mean(ms))

    clk = ClockSampler(local)
    clk.start()
    t_dev = timed(lambda: sm.matvec_device(dQ, dY, R, "mixed"))

    def e2e_step():
        dQ.copy_(hQ, non_blocking=True)
        sm.matvec_device(dQ, dY, R, "mixed")
        hY.copy_(dY, non_blocking=True)

    t_e2e = timed(e2e_step)
    clocks = clk.stop()
    t_dev, t_e2e = max_over_ranks([t_dev, t_e2e], dist if world > 1 else None, dev)
    # the sharded product against this rank's whole one (rank 0 checks)
    err = None
    if rank == 0:
        a.set_shard(0, 1)
        whole = torch.empty_like(dQ)
        a.matvec_device(dQ.data_ptr(), whole.data_ptr(), R, N, "mixed")
        err = float(torch.max(torch.abs(whole - dY)).item())
    lev = A.shard_range(a.nLevels, rank, world)[0]
    line = {"metric": metric_name(args.workload, N, p, R), "value": N * R / (t_dev * 1e-3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "N": N, "kernel": p["kernel"], "M": p["M"], "TOL_POW": p["tol"],
                       "nrhs": R, "precision": "mixed, batched", "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"one problem in {world} subtree shards (level {lev}) + all-reduce"},
            "max_abs_diff_sharded_vs_whole": err, "setup_s": setup_s, "clocks": clocks, "roofline": None,
            "gpu_launches": None,
            "e2e": {"value": N * R / (t_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 8 * N * R,
                    "d2h_bytes_per_step": 8 * N * R, "ms_per_step": t_e2e}}
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    a.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "many":
        run_many(args)
    elif args.shard:
        run_sharded(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
