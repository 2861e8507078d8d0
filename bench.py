#!/usr/bin/env python
"""Benchmark of the 3D stratified ray fan (ray-steps/s) on B200.

One step = the large 3D fan workload: four seeded synthetic atmospheres,
each traced with inclinations 0.5..60 deg every 0.1 deg (596, FP64-accumulated
as the reference CLI does) x azimuths 0..357 deg every 3 deg (120) = 71,520
rays, 10 bounces, 2000 km range, amplitude on (18 equations), FP64 --
286,080 rays per step, the four fans running concurrently on four CUDA
streams.  ray-steps = accepted RK4 steps (the sum of prop_rk4's returned k
in the reference).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU, each tracing its own fans (weak scaling, no
data-path collective); value = all ranks' ray-steps / max over ranks of the
device time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "ray-steps/s"
UNIT = "ray-steps/s"
SEEDS = (1, 2, 3, 4)
FAN = dict(incl=(0.5, 60.01, 0.1), az=(0.0, 357.0, 3.0), bounces=10, rng_max=2000.0)
# Algorithmic work per accepted RK4 ray-step (FLOP-equivalents: add/sub/mul 1,
# div/sqrt 4, exp/log/pow/trig 20), counted by running the reference algorithm
# (the oracle restatement) with an operation-counting scalar; roofline.json
# holds the counts, the weights and the sample they came from.
with open(os.path.join(ROOT, "roofline.json")) as _f:
    ROOFLINE = json.load(_f)
FLOPS_PER_STEP = {"fp64": ROOFLINE["variants"]["fp64_amp"], "fp32c": ROOFLINE["variants"]["fp32c_amp"],
                  "fp32c_flagged": ROOFLINE["variants"]["fp32c_amp"]}
# The FP32C kernel runs two classes of work on two pipes: the ray equations
# (the no-amplitude count) in FP64 and the Jacobian auxiliaries (the rest) in
# FP32, issued from the same schedulers, so its peak is the serial mix of the
# measured FP64 and FP32 rates.
FP32C_SPLIT = {"fp64": ROOFLINE["variants"]["fp32c_noamp"],
               "fp32": ROOFLINE["variants"]["fp32c_amp"] - ROOFLINE["variants"]["fp32c_noamp"]}


def mixed_peak(p64, p32):
    if not p64 or not p32:
        return None
    return FLOPS_PER_STEP["fp32c"] / (FP32C_SPLIT["fp64"] / p64 + FP32C_SPLIT["fp32"] / p32)


L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) per fan launch of the dominant kernel, from the ncu
# captures of the full 71,520-ray fan cut to one bounce (bench.py --profile-case
# fan3d_fp32c / fan3d_fp64, summarised in profiles/): the tables, launch angles
# and code are read once per launch and the state stays in registers, so the
# bytes do not grow with the steps of the 10-bounce launch, whose extra
# arrival rows (<= 76 MB) are written into the 126 MB L2.
TRAFFIC = {"fp64": 1453568 + 414720, "fp32c": 2059264 + 278784, "fp32c_flagged": 2059264 + 278784}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, 71,520-ray fan at 1 bounce "
                  "(profiles/fan3d_*_ncu_full_71520rays_1bnc.md)")


def config_dict(extra=None):
    n = n_fan_rays()
    d = {"workload": f"3d-strat-fan-4x{n}rays-10bnc-2000km-fp64-amp",
         "rays_per_step": 4 * n, "rays_per_fan": n, "incl_deg": list(FAN["incl"]), "az_deg": list(FAN["az"]),
         "bounces": FAN["bounces"], "max_rng_km": FAN["rng_max"], "calc_amp": True,
         "profiles": "seeded synthetic zTuvdp, 751 levels 0-150 km, seeds 1-4 (one fan each per step)",
         "l2": "flushed (256 MiB write) between timed steps"}
    if extra:
        d.update(extra)
    return d


def write_profiles(d):
    from infraga_b200 import synth
    return [synth.write_met(os.path.join(d, f"gen{s}.met"), s) for s in SEEDS]


def fan_angles():
    from infraga_b200 import synth
    return synth.fan_angles(*FAN["incl"], *FAN["az"])


def n_fan_rays():
    return fan_angles()[0].size


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU legs
_REF_PROBED = {}


def _ref_build(stem):
    """The fastest build of a reference driver (oracle/_ref) that runs on this
    host: -O3 -march=sapphirerapids (the GPU host's CPU) when it starts here,
    else the portable -O3 build.  Returns (path, flags) or (None, None)."""
    if stem in _REF_PROBED:
        return _REF_PROBED[stem]
    out = (None, None)
    for suffix, flags in (("_native", "-O3 -march=sapphirerapids"), ("_fast", "-O3")):
        exe = os.path.join(ROOT, "oracle", "_ref", stem + suffix)
        if not os.path.exists(exe):
            continue
        try:   # one short ray through the solver on the committed config-0 profile
            met = os.path.join(ROOT, "tests", "golden", "profiles", "gen0.met")
            args = ([met, "inclination=10", "azimuth=90", "bounces=0", "max_rng=100", "write_rays=false"]
                    if stem == "iga_ref_3d" else [])
            r = subprocess.run([exe, "prop", *args] if args else [exe], stdout=subprocess.DEVNULL,
                               stderr=subprocess.DEVNULL, timeout=60)
            if r.returncode == (0 if args else 2):
                out = (exe, flags)
                break
        except (OSError, subprocess.TimeoutExpired):
            continue
    _REF_PROBED[stem] = out
    return out


def ref_binary():
    return _ref_build("iga_ref_3d")[0]


def parse_ref_steps(text):
    for line in text.splitlines():
        if line.startswith("# rays"):
            parts = line.split()
            return int(parts[4]), float(parts[6])
    raise RuntimeError("reference driver output without a summary line")


def cpu_sample_reference(met, az_list, incl_step, procs):
    """Run the reference solver (oracle/_ref, compiled from the reference
    sources) as `procs` concurrent single-threaded processes, one azimuth each.
    Returns (ray-steps, wall seconds)."""
    exe = ref_binary()
    cmds = [[exe, "prop", met, "incl_min=0.5", f"incl_max={FAN['incl'][1]}", f"incl_step={incl_step}",
             f"azimuth={az}", f"bounces={FAN['bounces']}", f"max_rng={FAN['rng_max']}", "write_rays=false"]
            for az in az_list[:procs]]
    t0 = time.perf_counter()
    ps = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for c in cmds]
    outs = [p.communicate()[0] for p in ps]
    wall = time.perf_counter() - t0
    steps = sum(parse_ref_steps(o)[0] for o in outs)
    return steps, wall


def cpu_sample_port(met, az_list, incl_step, threads):
    from infraga_b200 import synth
    from oracle import oracle
    th, ph = [], []
    for az in az_list:
        a, b = synth.fan_angles(0.5, FAN["incl"][1], incl_step, az, az, 1.0)
        th.append(a); ph.append(b)
    th, ph = np.concatenate(th), np.concatenate(ph)
    t0 = time.perf_counter()
    _, steps = oracle.fan_3d(met, th, ph, bounces=FAN["bounces"], rng_max=FAN["rng_max"], write_rays=0,
                             n_threads=threads)
    return int(steps.sum()), time.perf_counter() - t0


def cpu_baseline(met):
    """Bounded single-core sample: one azimuth (90 deg), every 20th inclination
    (30 rays), same fan settings."""
    if ref_binary():
        steps, wall = cpu_sample_reference(met, [90.0], 2.0, 1)
        kind = "reference"
    else:
        steps, wall = cpu_sample_port(met, [90.0], 2.0, 1)
        kind = "port"
    return {"value": steps / wall, "unit": UNIT, "cores": 1, "kind": kind,
            "flags": _ref_build("iga_ref_3d")[1] if kind == "reference" else None,
            "sample": f"1 azimuth (90 deg) x 30 inclinations (0.5..60 step 2), seed {SEEDS[0]}, "
                      f"{steps} ray-steps in {wall:.1f} s"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    tmp = tempfile.mkdtemp(prefix="iga_bench_")
    mets = write_profiles(tmp)
    az_all = [float(a) for a in np.arange(0.0, 360.0, 3.0)]
    kind = "reference" if ref_binary() else "port"
    per_step = []
    for i in range(args.warmup + args.steps):
        met = mets[i % len(mets)]
        az = [az_all[(i * cores + j) % len(az_all)] for j in range(cores)]
        if kind == "reference":
            steps, wall = cpu_sample_reference(met, az, 2.0, cores)
        else:
            steps, wall = cpu_sample_port(met, az, 2.0, cores)
        if i >= args.warmup:
            per_step.append((steps, wall))
    tot_steps = sum(s for s, _ in per_step)
    tot_t = sum(w for _, w in per_step)
    value = tot_steps / tot_t
    sample = (f"{cores} concurrent single-threaded processes, one azimuth each, 30 inclinations "
              f"(0.5..60 step 2) per azimuth, same fan settings; {tot_steps} ray-steps over {args.steps} steps")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict({"reference_sample": sample}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
                             "flags": _ref_build("iga_ref_3d")[1] if kind == "reference" else None},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def fp64_peak_tflops(torch):
    """Measured FP64 throughput of cuBLAS DGEMM (torch.matmul, 8192^3), best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(); torch.matmul(a, b); e.record(); e.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def fp32_peak_tflops(torch):
    """Measured FP32 (non-tensor-core: TF32 off) SGEMM throughput, 8192^3, best of 5."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(); torch.matmul(a, b); e.record(); e.synchronize()
            best = min(best, s.elapsed_time(e) * 1e-3)
        del a, b
        return 2.0 * n ** 3 / best / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def run_ours(args):
    import torch
    import torch.distributed as dist
    import infraga_b200 as ig

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)

    tmp = tempfile.mkdtemp(prefix=f"iga_bench_{rank}_")
    mets = write_profiles(tmp)
    atmos = [ig.Atmosphere.load(m) for m in mets]
    th, ph = fan_angles()
    n = th.size
    precs = {"fp64": ig.FP64, "fp32c": ig.FP32C, "fp32c_flagged": ig.FP32C_FLAGGED}
    head = "fp32c" if args.precision in ("fp32c", "both") else "fp64"
    legs = [p_ for p_ in ("fp32c", "fp64") if args.precision in (p_, "both")]
    if args.precision == "both":   # the fan kernel without the re-trace pass (focusing rays flagged)
        legs.append("fp32c_flagged")
    all_params = {k: [a.default_params(bounces=FAN["bounces"], rng_max=FAN["rng_max"], write_rays=0,
                                       precision=precs[k]) for a in atmos] for k in legs}
    nb = FAN["bounces"] + 1
    d_th = torch.tensor(th, dtype=torch.float64, device=dev)
    d_ph = torch.tensor(ph, dtype=torch.float64, device=dev)
    bufs = [dict(arr=torch.empty((n, nb, 12), dtype=torch.float64, device=dev),
                 n=torch.empty(n, dtype=torch.int32, device=dev),
                 st=torch.empty(n, dtype=torch.int64, device=dev),
                 stat=torch.empty(n, dtype=torch.int32, device=dev),
                 ws=torch.zeros(ig.fan_workspace_bytes(), dtype=torch.uint8, device=dev)) for _ in atmos]
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    main = torch.cuda.current_stream()
    side = [torch.cuda.Stream(device=dev) for _ in atmos]

    def step(params):
        # the four seed fans of the workload, concurrently on four streams
        for k, a in enumerate(atmos):
            side[k].wait_stream(main)
            b = bufs[k]
            ig.fan_run_device(a, params[k], d_th.data_ptr(), d_ph.data_ptr(), n, b["arr"].data_ptr(),
                              b["n"].data_ptr(), b["st"].data_ptr(), b["stat"].data_ptr(), b["ws"].data_ptr(),
                              side[k].cuda_stream)
        for k in range(len(atmos)):
            main.wait_stream(side[k])

    peaks, gemm = {}, {}
    if not args.no_peak:
        gemm = {"fp64": fp64_peak_tflops(torch), "fp32": fp32_peak_tflops(torch)}
        peaks = {"fp64": gemm["fp64"], "fp32c": mixed_peak(gemm["fp64"], gemm["fp32"])}
        peaks["fp32c_flagged"] = peaks["fp32c"]

    props = torch.cuda.get_device_properties(dev)
    gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local)

    def measure(params):
        for _ in range(args.warmup):
            step(params)
        torch.cuda.synchronize()
        sampler = ClockSampler(gpu_id)
        sampler.start()
        steps_acc = torch.zeros((), dtype=torch.int64, device=dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t_wall0 = time.perf_counter()
        for i in range(args.steps):
            flush.zero_()
            evs[i][0].record(main)
            step(params)
            evs[i][1].record(main)
            for b in bufs:
                steps_acc += b["st"].sum()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        wall = time.perf_counter() - t_wall0
        clocks = sampler.stop()
        kern_s = sum(s_.elapsed_time(e_) for s_, e_ in evs) * 1e-3
        my_steps = int(steps_acc.item())
        tot_steps, max_t = my_steps, kern_s
        if world > 1:
            t = torch.tensor([float(my_steps), kern_s], dtype=torch.float64, device=dev)
            s2 = t.clone()
            dist.all_reduce(s2[:1], op=dist.ReduceOp.SUM)
            dist.all_reduce(t[1:], op=dist.ReduceOp.MAX)
            tot_steps, max_t = int(s2[0].item()), float(t[1].item())
        return {"value": tot_steps / max_t, "ms_per_step": 1e3 * max_t / args.steps, "my_steps": my_steps,
                "kern_s": kern_s, "tot_steps": tot_steps, "wall": wall, "clocks": clocks}

    res = {k: measure(all_params[k]) for k in legs}
    params = all_params[head]
    value = res[head]["value"]
    tot_steps, max_t = res[head]["tot_steps"], res[head]["ms_per_step"] * args.steps * 1e-3
    my_steps, kern_s, wall, clocks = res[head]["my_steps"], res[head]["kern_s"], res[head]["wall"], res[head]["clocks"]

    # e2e: the public host-buffer C ABI (iga_fan_run: H2D of the launch angles
    # from pinned memory, kernel, D2H of the arrival records), one host thread
    # per seed fan so the four calls overlap on the GPU, wall-clocked per step;
    # the max over ranks of the wall time.  Run for every precision leg.
    th_p = torch.from_numpy(th).pin_memory().numpy()
    ph_p = torch.from_numpy(ph).pin_memory().numpy()

    def measure_e2e(params):
        e2e_steps, e2e_t = 0, 0.0
        for k, a in enumerate(atmos):
            ig.fan_run(a, params[k], th_p, ph_p)   # size the handles' device buffers
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            out = [None] * len(atmos)

            def work(k):
                out[k] = ig.fan_run(atmos[k], params[k], th_p, ph_p)
            ths = [threading.Thread(target=work, args=(k,)) for k in range(len(atmos))]
            t0 = time.perf_counter()
            for t_ in ths:
                t_.start()
            for t_ in ths:
                t_.join()
            e2e_t += time.perf_counter() - t0
            e2e_steps += sum(r["total_steps"] for r in out)
        if world > 1:
            t = torch.tensor([float(e2e_steps), e2e_t], dtype=torch.float64, device=dev)
            s_ = t.clone()
            dist.all_reduce(s_[:1], op=dist.ReduceOp.SUM)
            dist.all_reduce(t[1:], op=dist.ReduceOp.MAX)
            e2e_steps, e2e_t = int(s_[0].item()), float(t[1].item())
        # bytes iga_fan_run copies per call: the launch angles in; the arrival
        # slots [n][bounces+1][12], per-ray counts, status and step counts out
        return {"value": e2e_steps / e2e_t if e2e_t > 0 else None, "unit": UNIT,
                "h2d_bytes_per_step": 2 * 8 * n * len(atmos),
                "d2h_bytes_per_step": len(atmos) * (n * nb * 12 * 8 + n * (4 + 4 + 8))}

    e2e = {k: measure_e2e(all_params[k]) for k in legs} if not args.no_e2e else {}

    result = None
    if rank == 0:
        fps = FLOPS_PER_STEP[head]
        achieved = fps * my_steps / kern_s / 1e12
        peak = peaks.get(head)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * max_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32c (fp64 ray equations, fp32 Jacobian auxiliaries with compensated sums)" if head == "fp32c" else "f64",
            "data": "synthetic",
            "config": config_dict({"parallelism": f"independent fans per GPU x{world}", "precision": head,
                                   "ray_steps_per_step": tot_steps / args.steps / world}),
            "e2e": e2e.get(head, {"value": None, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}),
            # FP32C: the fan kernel and the FP64-auxiliary re-trace kernel per fan
            "gpu_launches": args.steps * len(atmos) * (2 if head == "fp32c" else 1),
            "roofline": {"bound": "fp64+fp32" if head == "fp32c" else "fp64", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak else None, "traffic": TRAFFIC.get(head), "traffic_source": TRAFFIC_SOURCE,
                         "peak_source": ("measured in this run: cuBLAS DGEMM and SGEMM (TF32 off) 8192^3 via "
                                         "torch.matmul, best of 5; FP32C peak = flops_per_step / (fp64 part / DGEMM "
                                         "+ fp32 part / SGEMM)" if head == "fp32c" else
                                         "measured in this run: cuBLAS DGEMM 8192^3 via torch.matmul, best of 5"),
                         "gemm_tflops": gemm or None,
                         "flops_per_step": fps,
                         "flops_split": FP32C_SPLIT if head == "fp32c" else None},
            "legs": {k: {"value": v["value"], "ms_per_step": v["ms_per_step"], "clocks": v["clocks"],
                         "roofline_frac": (FLOPS_PER_STEP[k] * v["my_steps"] / v["kern_s"] / 1e12 / peaks[k])
                         if peaks.get(k) else None, "e2e": e2e.get(k)}
                     for k, v in res.items()},
            "clocks": clocks,
            "wall_s_timed_region": wall,
        }
        if "fp32c" in res and "fp64" in res:
            line["fp32c_over_fp64"] = res["fp32c"]["value"] / res["fp64"]["value"]
        if "fp32c_flagged" in res and "fp64" in res:
            line["fp32c_flagged_over_fp64"] = res["fp32c_flagged"]["value"] / res["fp64"]["value"]
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline(mets[0])
        if world == 1 and not args.no_extra:
            line.update(extra_configs(gpu_id))
        result = line
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    for a in atmos:
        a.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return 0 if result is not None or rank != 0 else 1


# ---------------------------------------------------------------- serving
SERVE = dict(rate=200.0, requests=60, fan_rays=(100, 100_000), eig_pairs=(1, 64), eig_frac=0.25,
             n_strat=56, n_rngdep=8, seed=11)


def serving_workload(tmp, args):
    """Config-4 request stream: Poisson arrivals (rate/s) of ray-fan requests
    (log-uniform 100..100,000 rays) and eigenray requests (1..64 pairs) over
    64 resident synthetic atmospheres (56 stratified, 8 spherical 11x11
    range-dependent grids)."""
    from infraga_b200 import synth
    g = np.random.default_rng(SERVE["seed"])
    strat = [synth.write_met(os.path.join(tmp, f"s{i}.met"), 100 + i) for i in range(SERVE["n_strat"])]
    grids = []
    for i in range(SERVE["n_rngdep"]):
        d = os.path.join(tmp, f"g{i}")
        grids.append(synth.write_rngdep_grid(d, 200 + i, n_lat=11, n_lon=11, lat0=30.0 + i, lon0=-110.0 + 2 * i,
                                             dlat=1.0, dlon=1.0, prefix="node"))
    th_all, ph_all = synth.fan_angles(0.5, 60.01, 0.1, 0.0, 357.0, 3.0)
    t = 0.0
    reqs = []
    for _ in range(args.serve_requests):
        t += g.exponential(1.0 / args.serve_rate)
        if g.random() < SERVE["eig_frac"]:
            n = int(g.integers(SERVE["eig_pairs"][0], SERVE["eig_pairs"][1] + 1))
            rng_km = g.uniform(50.0, 500.0, n)
            az = g.uniform(0.0, 2 * np.pi, n)
            pairs = [((0.0, 0.0, 0.0), (float(r * np.cos(a)), float(r * np.sin(a)))) for r, a in zip(rng_km, az)]
            reqs.append(dict(t=t, kind="eig", atmo=int(g.integers(0, SERVE["n_strat"])), pairs=pairs))
        else:
            n = int(np.exp(g.uniform(np.log(SERVE["fan_rays"][0]), np.log(SERVE["fan_rays"][1]))))
            pick = np.sort(g.choice(th_all.size, size=min(n, th_all.size), replace=False))
            a = int(g.integers(0, SERVE["n_strat"] + SERVE["n_rngdep"]))
            reqs.append(dict(t=t, kind="fan", atmo=a, th=th_all[pick], ph=ph_all[pick]))
    return strat, grids, reqs


def run_serving(args):
    """p50/p99 request latency and throughput of the request server under the
    config-4 stream, beside the one-request-at-a-time FP64 path."""
    import torch
    import infraga_b200 as ig
    torch.cuda.set_device(0)
    tmp = tempfile.mkdtemp(prefix="iga_serve_")
    strat_files, grid_files, reqs = serving_workload(tmp, args)
    strat = [ig.Atmosphere.load(m) for m in strat_files]
    grids = [ig.Atmosphere.load_rngdep(*g_) for g_ in grid_files]
    eigp = ig.eig_params(strat[0], bnc_min=0, bnc_max=1)   # FP64 traces: the one-at-a-time comparator
    eigp32 = ig.eig_params(strat[0], bnc_min=0, bnc_max=1)  # FP32-compensated traces: the served stream
    eigp32.fan.precision = ig.FP32C

    def params_for(r, precision):
        if r["atmo"] < len(strat):
            a = strat[r["atmo"]]
            return a, a.default_params(bounces=5, rng_max=1000.0, write_rays=0, precision=precision)
        a = grids[r["atmo"] - len(strat)]
        return a, a.default_params(geometry=ig.GEOM_SPH, bounces=2, write_rays=0)

    # warm the kernels and the absorption tables once
    for r in reqs[:8]:
        if r["kind"] == "fan":
            a, p = params_for(r, ig.FP32C)
            ig.fan_run(a, p, r["th"][:64], r["ph"][:64])
    torch.cuda.synchronize()
    sampler = ClockSampler("0")
    sampler.start()
    with ig.Server(max_inflight=8, eig_workers=2, hbm_budget=64 << 30) as srv:
        t0 = time.perf_counter()
        ids = []
        for r in reqs:
            dt = r["t"] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            if r["kind"] == "fan":
                a, p = params_for(r, ig.FP32C)
                ids.append(srv.submit_fan(a, p, r["th"], r["ph"]))
            else:
                ids.append(srv.submit_eig(strat[r["atmo"]], eigp32, r["pairs"]))
        for k, i in enumerate(ids):
            srv.wait(i, -1.0)
            srv.fetch(i)
            print(f"serving: request {k} done at {time.perf_counter() - t0:.2f} s", file=sys.stderr, flush=True)
        wall = time.perf_counter() - t0
        st = srv.stats()
    clocks = sampler.stop()

    # comparator: the same stream served one request at a time, FP64
    lat, steps64 = [], 0
    t_start = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t_start
        if now < r["t"]:
            time.sleep(r["t"] - now)
        if r["kind"] == "fan":
            a, p = params_for(r, ig.FP64)
            steps64 += ig.fan_run(a, p, r["th"], r["ph"])["total_steps"]
        else:
            steps64 += ig.eig_run(strat[r["atmo"]], eigp, r["pairs"])["total_steps"]
        lat.append(time.perf_counter() - t_start - r["t"])
        print(f"one-at-a-time: {r['kind']} done at {time.perf_counter() - t_start:.2f} s", file=sys.stderr, flush=True)
    serial_wall = time.perf_counter() - t_start
    n_fan = sum(r["kind"] == "fan" for r in reqs)
    line = {"metric": "serving latency p50/p99 [s] and ray-steps/s", "value": st["ray_steps"] / st["wall_s"],
            "unit": "ray-steps/s", "impl": "ours-serving", "n_gpus": 1, "higher_is_better": True,
            "scaling": "none", "vs_baseline": None,
            "dtype": "f32c 3D stratified fans and eigen searches, f64 range-dependent fans",
            "data": "synthetic",
            "config": {"workload": f"poisson {args.serve_rate:g}/s, {len(reqs)} requests ({n_fan} fans of "
                                   f"100..100000 rays log-uniform, {len(reqs) - n_fan} eigen of 1..64 pairs), "
                                   f"{len(strat)} stratified + {len(grids)} 11x11 range-dependent atmospheres",
                       "fan_settings": "3D stratified: 5 bounces, 1000 km, FP32C; sph range-dependent: 2 bounces, FP64",
                       "eigen_settings": "bnc 0..1, FP32-compensated traces (FP64 in the one-at-a-time comparator)"},
            "p50_s": st["p50_s"], "p99_s": st["p99_s"], "fan_p50_s": st["fan_p50_s"], "fan_p99_s": st["fan_p99_s"],
            "eig_p50_s": st["eig_p50_s"], "eig_p99_s": st["eig_p99_s"], "completed": st["completed"],
            "rays": st["rays"], "eigenrays": st["eigenrays"], "wall_s": wall,
            "one_at_a_time_fp64": {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                                   "ray_steps_per_s": steps64 / serial_wall, "wall_s": serial_wall},
            "clocks": clocks}
    print(json.dumps(line), flush=True)
    for a in strat + grids:
        a.close()
    shutil.rmtree(tmp, ignore_errors=True)
    return 0


# ---------------------------------------------------------------- config 2
def ref_sphr_binary():
    return _ref_build("iga_ref_sphr")[0]


def cpu_baseline_sphr(files):
    """The reference's spherical range-dependent solver (oracle/_ref) on a
    bounded sample: azimuth 90 deg, `procs` inclinations spread over the
    fan's range, one single-threaded process each, all 20 bounces."""
    exe = ref_sphr_binary()
    if not exe:
        return None
    from infraga_b200 import workloads as wl
    procs = max(1, min(8, os.cpu_count() or 1))
    incls = np.linspace(5.0, 45.0, procs)
    prefix, lat_f, lon_f, topo = files
    f = wl.SPHR_FAN
    cmds = [[exe, "prop", prefix, lat_f, lon_f, f"topo_file={topo}", f"inclination={x:.2f}", "azimuth=90",
             f"bounces={f['bounces']}", f"max_rng={f['rng_max']}", "write_rays=false"] for x in incls]
    t0 = time.perf_counter()
    ps = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for c in cmds]
    outs = [p.communicate(timeout=600)[0] for p in ps]
    wall = time.perf_counter() - t0
    steps = sum(parse_ref_steps(o)[0] for o in outs)
    return {"value": steps / wall, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"azimuth 90 deg x {procs} inclinations 5..45 deg, 20 bounces, one process each; "
                      f"{steps} ray-steps in {wall:.1f} s"}


def sphr_measure(steps, warmup, shapes=((1, None, "fp64"), (0, None, "fp64"), (1, 0, "fp64"), (1, None, "fp32c"),
                                       (1, None, "fp32c_flagged"), (0, None, "fp32c"))):
    """Config 2: spherical range-dependent fan over a 21x21 node grid with
    0.05-deg fractal terrain (workloads.py), FP64 and FP32-compensated.  The
    autotuner (iga_fan_tune) picks the CTA size first (on the FP64 kernel);
    each (calc_amp, block, precision) in `shapes` (block None = the tuned
    one, 0 = the kernel's default) is timed over `steps` launches with CUDA
    events after `warmup`, L2 flushed between.  Returns (legs, tuned block,
    seconds per tuning candidate, rays, files)."""
    import torch
    import infraga_b200 as ig
    from infraga_b200 import workloads as wl
    dev = torch.device("cuda", torch.cuda.current_device())
    files = wl.sphr_files()
    atmo = ig.Atmosphere.load_rngdep(files[0], files[1], files[2], topo_file=files[3], geometry=ig.GEOM_SPH)
    th, ph = wl.sphr_angles()
    n = th.size
    f = wl.SPHR_FAN
    nb = f["bounces"] + 1
    d_th = torch.tensor(th, dtype=torch.float64, device=dev)
    d_ph = torch.tensor(ph, dtype=torch.float64, device=dev)
    arr = torch.empty((n, nb, 12), dtype=torch.float64, device=dev)
    na = torch.empty(n, dtype=torch.int32, device=dev)
    st = torch.empty(n, dtype=torch.int64, device=dev)
    ws = torch.zeros(ig.fan_workspace_bytes(), dtype=torch.uint8, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    tp = atmo.default_params(geometry=ig.GEOM_SPH, bounces=f["bounces"], rng_max=f["rng_max"], write_rays=0)
    best, tune_s = ig.fan_tune(atmo, tp, th, ph)
    legs = {}
    for amp, block, prec in shapes:
        block = best if block is None else block
        params = atmo.default_params(geometry=ig.GEOM_SPH, bounces=f["bounces"], rng_max=f["rng_max"],
                                     write_rays=0, calc_amp=amp,
                                     precision={"fp64": ig.FP64, "fp32c": ig.FP32C, "fp32c_flagged": ig.FP32C_FLAGGED}[prec])
        params.block = block
        times, n_steps = [], 0
        for i in range(warmup + steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ig.fan_run_device(atmo, params, d_th.data_ptr(), d_ph.data_ptr(), n, arr.data_ptr(), na.data_ptr(),
                              st.data_ptr(), 0, ws.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            if i >= warmup:
                times.append(e0.elapsed_time(e1) * 1e-3)
                n_steps = int(st.sum().item())
        t = sum(times) / len(times)
        name = ("" if prec == "fp64" else prec + "_") + ("amp" if amp else "noamp") + \
            ("" if block == best else f"_block{block or 128}")
        legs[name] = {"ray_steps": n_steps, "s_per_fan": t, "value": n_steps / t, "block": block or 128,
                      "precision": prec}
    atmo.close()
    return legs, best, tune_s, n, files


def run_sphr(args):
    """Config 2 on its own line (``--sphr``): tuned and default launch shapes,
    with and without amplitude, and the reference's CPU rate."""
    legs, best, tune_s, n, files = sphr_measure(args.steps, args.warmup)
    cpu = None if args.no_cpu else cpu_baseline_sphr(files)
    head = legs["amp"]
    line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * head["s_per_fan"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"sph-rngdep-fan-{n}rays-21x21grid-401x401terrain-20bnc-3000km-fp64",
                       "rays": n, "l2": "flushed (256 MiB write) between timed steps"},
            "legs": legs, "autotune": {"block": best, "seconds_per_candidate": tune_s}, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- config 3
def cpu_baseline_eig(mets, pairs_by_seed, bnc_max):
    """The reference eigenray search (oracle/_ref iga_ref_3d_fast eig mode) on a
    bounded sample: up to 8 pairs of the first seed, one process per pair,
    bounce counts 0..bnc_max (the caller bounds it: the reference spends
    minutes per pair on 0..8)."""
    exe = ref_binary()
    if not exe:
        return None
    procs = max(1, min(8, os.cpu_count() or 1))
    cmds = []
    for k, (src, rcv) in enumerate(pairs_by_seed[0][:procs]):
        cmds.append([exe, "eig", mets[0], f"rcvr_x={rcv[0]:.6f}", f"rcvr_y={rcv[1]:.6f}", "bnc_min=0",
                     f"bnc_max={bnc_max}", f"out=/tmp/iga_eig_cpu_{os.getpid()}_{k}.dat",
                     f"out_id=/tmp/iga_eig_cpu_{os.getpid()}_{k}"])
    t0 = time.perf_counter()
    ps = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for c in cmds]
    outs = [p.communicate(timeout=1200)[0] for p in ps]
    wall = time.perf_counter() - t0
    n_eig = 0
    for o in outs:
        for line in o.splitlines():
            if line.startswith("# eigenrays"):
                n_eig += int(line.split()[2])
    return {"value": n_eig / wall, "unit": "eigenrays/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} pairs of seed 1, bounces 0..{bnc_max}, one process per pair; "
                      f"{n_eig} eigenrays in {wall:.1f} s"}


def eigen_measure(seeds):
    """Config 3: batched 3D eigenray search, 128 pairs per seed, bounces
    0..8, FP64 and FP32-compensated traces; eigenrays/s over the wall time of
    iga_eig_run, and the FP32C eigenrays against the FP64 ones.  Returns
    (legs, comparison, profile paths, pairs per seed)."""
    import infraga_b200 as ig
    from infraga_b200 import workloads as wl
    bmax = wl.EIG["bnc_max"]
    mets = [wl.profile_met(sd) for sd in seeds]
    atmos = [ig.Atmosphere.load(m) for m in mets]
    pairs = [wl.eig_pairs(sd) for sd in seeds]
    # warm-up: a small search per precision (kernel loading, allocator)
    for prec in (ig.FP64, ig.FP32C):
        p = ig.eig_params(atmos[0], bnc_min=0, bnc_max=1)
        p.fan.precision = prec
        ig.eig_run(atmos[0], p, pairs[0][:4])
    legs, rows = {}, {}
    for name, prec in (("fp64", ig.FP64), ("fp32c", ig.FP32C)):
        n_eig, steps, t_tot = 0, 0, 0.0
        rows[name] = []
        for a, pr in zip(atmos, pairs):
            p = ig.eig_params(a, bnc_min=0, bnc_max=bmax)
            p.fan.precision = prec
            t0 = time.perf_counter()
            r = ig.eig_run(a, p, pr)
            t_tot += time.perf_counter() - t0
            n_eig += r["eigenrays"].shape[0]
            steps += r["total_steps"]
            rows[name].append((r["eigenrays"], r["pair_index"]))
        legs[name] = {"eigenrays": n_eig, "seconds": t_tot, "value": n_eig / t_tot, "ray_steps": steps}
    # FP32C eigenrays against the FP64 ones: matched by pair, bounce count and
    # launch inclination (within 0.05 deg)
    d_pos, d_t, n_match = [], [], 0
    for (r64, i64), (r32, i32) in zip(rows["fp64"], rows["fp32c"]):
        for k in range(r64.shape[0]):
            cand = np.where((i32 == i64[k]) & (r32[:, 2] == r64[k, 2]) & (np.abs(r32[:, 0] - r64[k, 0]) < 0.05))[0]
            if cand.size:
                j = cand[np.argmin(np.abs(r32[cand, 0] - r64[k, 0]))]
                n_match += 1
                d_pos.append(np.hypot(r32[j, 3] - r64[k, 3], r32[j, 4] - r64[k, 4]))
                d_t.append(abs(r32[j, 5] - r64[k, 5]))

    def pct(v, q):
        v = np.asarray(v, dtype=np.float64)
        v = v[np.isfinite(v)]
        return float(np.percentile(v, q)) if v.size else None

    nonfinite = {k: int(sum(int((~np.isfinite(r[:, :12])).any(axis=1).sum()) for r, _ in rows[k])) for k in rows}
    err = {"matched": n_match, "fp64_eigenrays": legs["fp64"]["eigenrays"],
           "fp32c_eigenrays": legs["fp32c"]["eigenrays"],
           "landing_km_p50": pct(d_pos, 50), "landing_km_p99": pct(d_pos, 99),
           "time_s_p50": pct(d_t, 50), "time_s_p99": pct(d_t, 99),
           "rows_with_nonfinite_columns": nonfinite}
    for a in atmos:
        a.close()
    return legs, err, mets, pairs


def run_eigen(args):
    """Config 3 on its own line (``--eigen``): 8 seeds x 128 pairs, 0..8
    bounces, and the reference's CPU rate on a bounded sample."""
    from infraga_b200 import workloads as wl
    legs, err, mets, pairs = eigen_measure(list(range(1, 9)))
    cpu = None if args.no_cpu else cpu_baseline_eig(mets, pairs, 1)
    head = legs["fp32c"]
    line = {"metric": "eigenrays/s", "value": head["value"], "unit": "eigenrays/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": 1e3 * head["seconds"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-compensated (f64 Newton)", "data": "synthetic",
            "config": {"workload": f"3d-strat-eigen-8seeds-x-{wl.EIG['pairs']}pairs-bnc0-{wl.EIG['bnc_max']}",
                       "timing": "wall clock of iga_eig_run over all seeds (host-driven search)"},
            "legs": legs, "fp32c_vs_fp64": err, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)
    return 0


def extra_configs(gpu_id):
    """Compact measurements of configs 2 and 3 and of the waveform mode carried
    in the default line, each with the clocks sampled during it: the config-2
    fan at the tuned CTA size (2 timed launches after 1 warm-up), one config-3
    seed (128 pairs, bounces 0..8) at both precisions, and the -wnl_wvfrm fan
    (576 rays, 2 timed calls after 1 warm-up)."""
    from infraga_b200 import workloads as wl
    out = {}
    sampler = ClockSampler(gpu_id)
    sampler.start()
    legs, best, tune_s, n, _ = sphr_measure(2, 1, shapes=((1, None, "fp64"), (1, None, "fp32c"),
                                                          (1, None, "fp32c_flagged")))
    out["config2"] = {"metric": METRIC, "unit": UNIT, "value": legs["amp"]["value"], "dtype": "f64",
                      "fp32c_value": legs["fp32c_amp"]["value"],
                      "fp32c_over_fp64": legs["fp32c_amp"]["value"] / legs["amp"]["value"],
                      "workload": f"sph-rngdep-fan-{n}rays-21x21grid-401x401terrain-20bnc-3000km",
                      "timing": "CUDA events, mean of 2 launches after 1 warm-up, L2 flushed",
                      "block": best, "s_per_fan": legs["amp"]["s_per_fan"],
                      "fp32c_s_per_fan": legs["fp32c_amp"]["s_per_fan"],
                      "fp32c_flagged_value": legs["fp32c_flagged_amp"]["value"], "clocks": sampler.stop()}
    sampler = ClockSampler(gpu_id)
    sampler.start()
    legs3, err, _, _ = eigen_measure([1])
    out["config3"] = {"metric": "eigenrays/s", "unit": "eigenrays/s",
                      "workload": f"3d-strat-eigen-1seed-x-{wl.EIG['pairs']}pairs-bnc0-{wl.EIG['bnc_max']}",
                      "timing": "wall clock of iga_eig_run", "legs": legs3, "fp32c_vs_fp64": err,
                      "clocks": sampler.stop()}
    sampler = ClockSampler(gpu_id)
    sampler.start()
    w = wnl_measure(2)
    w["clocks"] = sampler.stop()
    out["wnl"] = w
    return out


# ---------------------------------------------------------------- weakly non-linear waveforms
# -wnl_wvfrm over a fan: 16 inclinations x 36 azimuths (576 rays, about four
# per SM), the reference's default 8192-sample impulse, one bounce.
WNL = dict(incl=(4.0, 34.0, 16), az=(0.0, 350.0, 36), bounces=1, len=8192, seed=1, ref_rays=2)


def wnl_waveform(n):
    """wvfrm::build_wvfrm's built-in impulse with its defaults (p0 10 Pa, t0 0.1 s,
    alpha 4, N_rise 10, N_period 40; waveforms.cpp:67-84)."""
    import math
    p0, t0, alpha = 10.0, 0.1, 4.0
    dur = t0 * n * max(((1.0 + alpha) - math.sqrt(1.0 + alpha)) / 10, 2.0 * 3.14159 * math.sqrt(1 + alpha) / 40)
    t = np.array([-dur / 2.0 + dur * i / n for i in range(n)])
    xp = (alpha + 1.0) - math.sqrt(alpha + 1.0)
    norm = xp ** alpha * (1.0 - xp / (1.0 + alpha)) * math.exp(-xp)
    x = np.where(t >= 0, t / t0, 0.0)
    pw = np.where(t >= 0, p0 * (x ** alpha * (1.0 - x / (1.0 + alpha)) * np.exp(-x)) / norm, 0.0)
    return t, pw


def wnl_fan():
    th = np.repeat(np.linspace(*WNL["incl"]), WNL["az"][2])
    ph = np.tile(np.linspace(*WNL["az"]), WNL["incl"][2])
    return th, ph


def wnl_cpu_reference(met, th, ph):
    """The reference's waveform mode (oracle/_ref/infraga-3d-wnl, built from its
    sources over oracle/fftshim) on one host core for a few rays of the fan:
    seconds per waveform."""
    exe = os.path.join(ROOT, "oracle", "_ref", "infraga-3d-wnl")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/infraga-3d-wnl not built"}
    tot = 0.0
    n = WNL["ref_rays"]
    idx = np.linspace(0, th.size - 1, n).astype(int)
    with tempfile.TemporaryDirectory() as d:
        shutil.copy(met, os.path.join(d, "atmo.met"))
        for i in idx:
            t0 = time.perf_counter()
            subprocess.run([exe, "-wnl_wvfrm", "atmo.met", f"inclination={th[i]!r}", f"azimuth={ph[i]!r}",
                            f"bounces={WNL['bounces']}"], cwd=d, stdout=subprocess.DEVNULL, check=True, timeout=600)
            tot += time.perf_counter() - t0
    return {"value": n / tot, "unit": "waveforms/s", "cores": 1, "kind": "reference",
            "sample": f"{n} rays of the fan (indices {idx.tolist()}), one process each, wall clock"}


def wnl_measure(reps=2, cpu=True):
    """Waveforms per second through iga_wnl_run (host buffers in and out: the
    trace, the step-count pass and the waveform kernel), with the Heun steps
    per second of the waveform kernel's work, and the reference on the host."""
    import infraga_b200 as ig
    from infraga_b200 import workloads as wl
    met = wl.profile_met(WNL["seed"])
    atmo = ig.Atmosphere.load(met)
    p = ig.wnl_params(atmo, bounces=WNL["bounces"])
    th, ph = wnl_fan()
    t, pw = wnl_waveform(WNL["len"])
    ig.wnl_run(atmo, p, th[:8], ph[:8], t, pw)   # warm-up (kernel loading, allocator)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        r = ig.wnl_run(atmo, p, th, ph, t, pw)
        times.append(time.perf_counter() - t0)
    sec = statistics.mean(times)
    steps = float(np.sum(r["steps"]))
    out = {"metric": "waveforms/s", "unit": "waveforms/s", "value": th.size / sec, "dtype": "f64",
           "workload": f"3d-strat-wnl-{th.size}rays-{WNL['len']}samples-{WNL['bounces']}bnc-impulse",
           "timing": f"wall clock of iga_wnl_run, mean of {reps} calls after 1 warm-up",
           "s_per_call": sec, "heun_steps": steps, "heun_steps_per_s": steps / sec,
           "rays_ok": int(np.sum(r["status"] == 0))}
    if cpu:
        out["cpu_reference"] = wnl_cpu_reference(met, th, ph)
    atmo.close()
    return out


def run_wnl(args):
    import torch
    torch.cuda.set_device(0)
    sampler = ClockSampler("0")
    sampler.start()
    out = wnl_measure(max(args.steps, 1), cpu=not args.no_cpu)
    out["clocks"] = sampler.stop()
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------- profiling cases
# Small, self-contained runs of each kernel for ncu captures (summaries under
# profiles/): each case traces one modest workload once per repetition, so a
# capture with ``-k regex:<kernel> -c 1`` sees a representative launch of a few
# hundred milliseconds at most.  ``python bench.py --profile-case <case>``.
def _profile_case(name):
    import infraga_b200 as ig
    from infraga_b200 import synth
    from infraga_b200 import workloads as wl
    golden = os.path.join(ROOT, "tests", "golden")
    if name in ("fan3d_fp32c", "fan3d_fp64"):
        # the full 71,520-ray fan of the benchmark (every persistent block
        # resident, as in the timed run) cut to one bounce within 600 km, so
        # one launch takes tens of milliseconds
        atmo = ig.Atmosphere.load(wl.profile_met(1))
        th, ph = synth.fan_angles(*FAN["incl"], *FAN["az"])
        prec = ig.FP32C if name.endswith("fp32c") else ig.FP64
        p = atmo.default_params(bounces=1, rng_max=600.0, write_rays=0, precision=prec)
        return lambda: ig.fan_run(atmo, p, th, ph)
    if name in ("config2_fp32c", "config2_fp64"):
        # the config-2 fan itself (14,328 rays, 21x21 grid with terrain, 20
        # bounces, 3000 km): one launch of several seconds, for launch lists
        # (gpu__time_duration only) of the fan and re-trace kernels
        f = wl.sphr_files()
        atmo = ig.Atmosphere.load_rngdep(f[0], f[1], f[2], topo_file=f[3], geometry=ig.GEOM_SPH)
        th, ph = wl.sphr_angles()
        s = wl.SPHR_FAN
        p = atmo.default_params(geometry=ig.GEOM_SPH, bounces=s["bounces"], rng_max=s["rng_max"], write_rays=0,
                                precision=ig.FP32C if name.endswith("fp32c") else ig.FP64)
        return lambda: ig.fan_run(atmo, p, th, ph)
    if name == "fansph":       # spherical stratified fan (fansph_fp64_kernel): 1,440 rays
        atmo = ig.Atmosphere.load(wl.profile_met(1))
        th, ph = synth.fan_angles(0.5, 60.0, 0.5, 0.0, 330.0, 30.0)
        p = atmo.default_params(geometry=ig.GEOM_SPH, bounces=5, rng_max=2000.0, src=(30.0, 0.0, 0.0))
        return lambda: ig.fan_run(atmo, p, th, ph)
    if name in ("fansphr", "fansphr_fp32c"):   # 21x21 grid with terrain: 408 rays, 1 bounce, 600 km
        f = wl.sphr_files()
        atmo = ig.Atmosphere.load_rngdep(f[0], f[1], f[2], topo_file=f[3], geometry=ig.GEOM_SPH)
        th, ph = synth.fan_angles(0.5, 50.0, 3.0, 0.0, 345.0, 15.0)
        p = atmo.default_params(geometry=ig.GEOM_SPH, bounces=1, rng_max=600.0,
                                precision=ig.FP32C if name.endswith("fp32c") else ig.FP64)
        return lambda: ig.fan_run(atmo, p, th, ph)
    if name == "fan3dr":       # committed 5x5 grid with terrain (fan3dr_fp64_kernel): 1,080 rays
        d = os.path.join(golden, "rngdep3d")
        atmo = ig.Atmosphere.load_rngdep(os.path.join(d, "node"), os.path.join(d, "node_x.dat"),
                                         os.path.join(d, "node_y.dat"), topo_file=os.path.join(d, "topo.dat"),
                                         geometry=ig.GEOM_3D)
        th, ph = synth.fan_angles(0.5, 45.0, 0.5, 0.0, 330.0, 30.0)
        p = atmo.default_params(bounces=2, rng_max=600.0)
        return lambda: ig.fan_run(atmo, p, th, ph)
    if name == "paths":        # 3D stratified fan with sampled ray paths (PATHS instantiation)
        atmo = ig.Atmosphere.load(wl.profile_met(1))
        th, ph = synth.fan_angles(1.0, 45.0, 1.0, 0.0, 330.0, 30.0)
        p = atmo.default_params(bounces=3, rng_max=1000.0, write_rays=1)
        steps = ig.fan_run(atmo, p, th, ph)["ray_steps"]
        return lambda: ig.fan_paths(atmo, p, th, ph, caustics=True, ray_steps=steps)
    if name == "wnl3d":        # waveforms of 148 rays, 8192 samples, no bounce (wnl3d_kernel: one CTA per ray)
        atmo = ig.Atmosphere.load(wl.profile_met(1))
        th = np.repeat(np.linspace(4.0, 34.0, 4), 37)
        ph = np.tile(np.linspace(0.0, 360.0, 37), 4)
        p = ig.wnl_params(atmo, bounces=0)
        t, pw = wnl_waveform(8192)
        return lambda: ig.wnl_run(atmo, p, th, ph, t, pw)
    if name == "eig3d":        # 3D eigenray search, 16 pairs (trace3d_fp64_kernel)
        atmo = ig.Atmosphere.load(wl.profile_met(1))
        pairs = wl.eig_pairs(1, 16)
        p = ig.eig_params(atmo, bnc_min=0, bnc_max=2, streams=1)
        return lambda: ig.eig_run(atmo, p, pairs)
    if name == "eigsph":       # spherical eigenray search, 8 pairs (tracesph_fp64_kernel)
        atmo = ig.Atmosphere.load(wl.profile_met(1))
        pairs = [((30.0, 0.0, 0.0), (30.0 + 2.0 * k / 8.0, 2.5 + 0.25 * k)) for k in range(8)]
        p = ig.eig_params(atmo, geometry=ig.GEOM_SPH, bnc_min=0, bnc_max=1, streams=1)
        return lambda: ig.eig_run(atmo, p, pairs)
    raise SystemExit(f"unknown profiling case {name!r} (one of {', '.join(PROFILE_CASES)})")


PROFILE_CASES = ("fan3d_fp32c", "fan3d_fp64", "config2_fp32c", "config2_fp64", "fansph", "fansphr_fp32c", "fansphr",
                 "fan3dr", "paths", "wnl3d", "eig3d", "eigsph")


def run_profile_case(args):
    run = _profile_case(args.profile_case)
    for _ in range(args.reps):
        run()
    print(f"{args.profile_case}: ok")
    return 0


def launch_ranks(n):
    """`--gpus N` without an external launcher: start N ranks (one process per
    GPU, RANK / LOCAL_RANK / WORLD_SIZE set by torch.distributed.run on
    127.0.0.1) running this script with the same arguments; exit with the
    launcher's status."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end host-API leg")
    ap.add_argument("--no-peak", action="store_true", help="skip the GEMM peak measurements")
    ap.add_argument("--no-extra", action="store_true",
                    help="leave the compact config-2 / config-3 measurements out of the default line")
    ap.add_argument("--precision", choices=["both", "fp32c", "fp64"], default="both",
                    help="fan precision(s) to time; the headline is fp32c unless only fp64 is run")
    ap.add_argument("--az-step", type=float, default=FAN["az"][2],
                    help="azimuth spacing in degrees (a larger value gives a smaller fan, for profiling)")
    ap.add_argument("--serving", action="store_true",
                    help="run the request-server benchmark (Poisson stream of fan and eigen requests) instead")
    ap.add_argument("--serve-rate", type=float, default=SERVE["rate"], help="request arrival rate [1/s]")
    ap.add_argument("--serve-requests", type=int, default=SERVE["requests"], help="requests in the stream")
    ap.add_argument("--sphr", action="store_true",
                    help="time the spherical range-dependent fan with terrain (config 2) instead")
    ap.add_argument("--eigen", action="store_true",
                    help="time the batched 3D eigenray search (config 3, FP64 and FP32C) instead")
    ap.add_argument("--wnl", action="store_true",
                    help="time the weakly non-linear waveform mode over a 576-ray fan instead")
    ap.add_argument("--profile-case", choices=PROFILE_CASES,
                    help="run one small profiling workload of a single kernel (for ncu captures) instead")
    ap.add_argument("--reps", type=int, default=1, help="repetitions of --profile-case")
    args = ap.parse_args()
    if args.profile_case:
        return run_profile_case(args)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus)
    if args.serving:
        return run_serving(args)
    if args.sphr:
        return run_sphr(args)
    if args.eigen:
        return run_eigen(args)
    if args.wnl:
        return run_wnl(args)
    if args.az_step != FAN["az"][2]:
        FAN["az"] = (FAN["az"][0], FAN["az"][1], args.az_step)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
