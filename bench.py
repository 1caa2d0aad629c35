"""Benchmark: conditional-block sampling of the synthetic 64-qubit ring workload on B200.

One step = one sample of the hot path: the 2^20 conditional block of one 44-bit prefix
(complex64 contraction over all parity slices, complex128 coherent sum + tail) and the FP64
CDF draw of its 20 free bits.  Workload: 64-qubit ring, depth 73, 314 T gates (378-vertex
injected graph), 2 parity slices (4 slices, rmax 34: one 128 GiB complex64 table), PCG64
prefixes/uniforms from make_protocol.  Inputs and tables are far larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]
                    [--mode fused|device|plain] [--no-plain] [--no-cpu] [--no-audit] [--no-configs]
    python bench.py --serve [--graphs] ...        the serving mix alone
    python bench.py --profile-case ...            the small profiling case of profiles/

Multi-GPU (torchrun, one rank per GPU): independent replicas, each rank samples its own
prefixes (weak scaling); the elapsed time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "samples/s (64q, 2^20 block) served vs plain at c_y≥0.9999; p50/p99 ms"
# DRAM traffic / algorithmic bytes of one launch of the dominant kernel, measured by ncu on a
# group of the same plan whose tables are 2^27-2^28 entries (profiles/dcs_g_ring64_prefix_group21_bytes_low3.md,
# profiles/k_runs_ring64_prefix_group21.md, profiles/k_fused_ring64_prefix_group23.md): full-size launches cannot be captured with all
# counters, and the traffic of a group scales with the entries it touches.
TRAFFIC_RATIO = {"k_runs": 0.9823, "k_fused": 0.9635, "dcs_g (plan-specialised k_runs)": 0.9780}
FALLBACK_HBM = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="ring64_d73_t314_k20")
    ap.add_argument("--mode", default="fused", choices=["fused", "device", "plain"])
    ap.add_argument("--storage", default=None, choices=["float16"],
                    help="binary16 table storage (the approximate half-storage tier; --mode device or plain)")
    ap.add_argument("--plain-samples", type=int, default=1)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-audit", action="store_true")
    ap.add_argument("--audits", type=int, default=64,
                    help="generation samples audited in complex128 (ids from an independent PCG64 stream)")
    ap.add_argument("--audit-seed", type=int, default=24521)
    ap.add_argument("--audit-mode", default="fused", choices=["fused", "device"],
                    help="complex128 executor of the audits (fused: plan-specialised kernels in FP64)")
    ap.add_argument("--no-configs", action="store_true", help="skip the small workloads (16q, 40q) sub-report")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--seed", type=int, default=24520)
    ap.add_argument("--tune", action="store_true", help="autotune the fused tile shape before timing")
    ap.add_argument("--no-jit", action="store_true",
                    help="run the library's register-run kernel instead of the plan-specialised group kernels")
    ap.add_argument("--prefetch-kb", type=int, default=None,
                    help="generated kernels: KiB per CTA staging the next tile's first-run entries "
                         "(default: the tuned configuration)")
    ap.add_argument("--tune-groups", action="store_true",
                    help="choose the generated kernel variant per group (autotune.tune_groups) before timing")
    ap.add_argument("--serve", action="store_true", help="run the serving mix (32q/48q/64q) instead")
    ap.add_argument("--serve-seconds", type=float, default=12.0, help="arrival window of the serving run")
    ap.add_argument("--serve-rate", type=float, default=1.0, help="Poisson request rate (1/s)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving mix in the default run")
    ap.add_argument("--plain-64q-seconds", type=float, default=None,
                    help="serving comparator: per-sample plain-path time of the 64q circuit (default: measured)")
    ap.add_argument("--serve-max-samples", type=int, default=64)
    ap.add_argument("--hbm-budget-gib", type=float, default=170.0)
    ap.add_argument("--graphs", action="store_true",
                    help="serving: replay each runner's batch as a CUDA graph (captured per batch size)")
    return ap.parse_args()


def dist_init():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def peaks():
    """HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json (`hbm_gbs`, at the top level or under
    a per-GPU entry), else the fallback figure."""
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            v = d.get("hbm_gbs") if isinstance(d, dict) else None
            if v is None and isinstance(d, dict):
                v = next((x["hbm_gbs"] for x in d.values() if isinstance(x, dict) and "hbm_gbs" in x), None)
            if v is not None and float(v) > 0:
                return float(v), "measured"
        except (ValueError, TypeError, KeyError, StopIteration):
            pass
    return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[0]) for r in self.rows if len(r) >= 8 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 8:
                for nm, v in zip(names, r[4:8]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------------------------------------
def cpu_baseline(workload, seconds, rank0=True):
    """The oracle's C/OpenMP executor (complex128) on a bounded sample of the same plan.

    The 2^34-entry complex128 table of the 64-qubit plan does not fit host memory, so the
    sample is the longest prefix of the first slice's steps whose table stays <= 2^24 entries
    (256 MiB); the measured algorithmic bytes/s is converted to samples/s with the full
    per-sample algorithmic bytes (complex128, all slices): an extrapolation, not a measured
    64-qubit sample."""
    from dcs245_classical_sampling_b200 import plan as P
    from dcs245_classical_sampling_b200.engine import SliceParams
    from dcs245_classical_sampling_b200.sampling import make_protocol
    from dcs245_classical_sampling_b200.workloads import build_workload
    from oracle import c as oc
    lib = oc.load()
    w = build_workload(workload)
    bp = P.build_block_plan(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                            w["open_vertices"])
    proto = make_protocol(7, 1, w["n"], w["open_vertices"])
    x = np.array([int(c) for c in proto["records"][0]["input_data_bits"]], np.uint8)
    _, items = SliceParams(bp).items(x)
    params = oc.encode_params(items[0][1])
    steps = oc.encode(bp.steps)
    cap = 24
    last = 0
    for j, st in enumerate(bp.steps):
        if max(len(st.active_in), len(st.active_out)) > cap or max(st.active_in + st.active_out + (0,)) >= cap + 2:
            break
        last = j + 1
    sample_steps = bp.steps[:last]
    slots = max([0] + [max(s.active_in + s.active_out + (0,)) + 1 for s in sample_steps])
    E = np.zeros(1 << slots, np.complex128)
    alg_sample = sum(((1 << len(s.active_in)) + (1 << len(s.active_out))) * 16 for s in sample_steps)
    per_sample = P.step_bytes(bp, 16) * len(items)
    t0 = time.perf_counter()
    reps = 0
    while True:
        E[:] = 0
        E[0] = 1
        oc.run_steps(lib, steps, params, E, 0, last)
        reps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    bps = alg_sample * reps / dt
    return {"value": bps / per_sample, "unit": "samples/s", "cores": int(lib.oracle_threads()), "kind": "port",
            "sample": (f"extrapolated: C/OpenMP complex128 executor over the first {last} of {len(bp.steps)} steps "
                       f"of one slice (tables <= 2^{cap}), {reps} reps in {dt:.1f} s = {bps / 1e9:.2f} GB/s "
                       f"algorithmic; samples/s = that rate / {per_sample / 2**40:.2f} TiB per sample (all "
                       f"{len(items)} slices); a complete 64-qubit sample needs a 256 GiB complex128 table"),
            "seconds": dt, "algorithmic_gbs": bps / 1e9, "steps_sampled": last, "steps_total": len(bp.steps)}


# The small workloads, measured completely on the CPU and the GPU (no extrapolation): the
# 16-qubit case (all 256 samples, as its configuration asks) and the 40-qubit case (a fixed
# subset of its 1,000 samples on the CPU, all of them on the GPU).
SMALL_CONFIGS = {"ring16_d20_t24_k8": {"samples": 256, "cpu_samples": 256, "mode": "device"},
                 "ring40_d45_t190_k16": {"samples": 1000, "cpu_samples": 8, "mode": "fused"}}


def cpu_small_configs(seed):
    """Complete CPU samples (block + draw) of the small workloads: the oracle engine with the
    C/OpenMP executor (oracle.c.CpuSampler), timed sample by sample."""
    from dcs245_classical_sampling_b200.sampling import make_protocol
    from dcs245_classical_sampling_b200.workloads import build_workload
    from oracle import block_ref
    from oracle import c as oc
    lib = oc.load()
    out = {}
    for name, cfg in SMALL_CONFIGS.items():
        w = build_workload(name)
        eng = block_ref.OracleEngine(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                                     w["open_vertices"])
        cs = oc.CpuSampler(eng, lib)
        recs = make_protocol(seed, cfg["cpu_samples"], w["n"], w["open_vertices"])["records"]
        t0 = time.perf_counter()
        idx = []
        for r in recs:
            x = np.array([int(c) for c in r["input_data_bits"]], np.uint8)
            idx.append(cs.sample(x, r["draw_uniform"])["A_index"])
        dt = time.perf_counter() - t0
        out[name] = {"value": len(recs) / dt, "unit": "samples/s", "samples": len(recs), "seconds": dt,
                     "cores": int(lib.oracle_threads()), "kind": "port",
                     "what": "complete samples: oracle engine + C/OpenMP complex128 executor + NumPy draw",
                     "indices_head": idx[:8]}
    return out


def reference_arm(args):
    """The reference's CPU path for this workload, timed on the host cores.  The reference is
    Python and cannot run on a GPU machine, so its restatement in C (the oracle's executor) runs
    instead.  Each step is one bounded sample of the 64-qubit plan (cpu_baseline), whose measured
    duration is ms_per_step; value is the samples/s that rate extrapolates to."""
    rank, world, _ = dist_init()
    if rank != 0:
        return
    samples, secs = [], []
    cb = None
    per_step = max(1.0, args.cpu_seconds / 8)
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        cb = cpu_baseline(args.workload, per_step)
        if i >= args.warmup:
            samples.append(cb["value"])
            secs.append(time.perf_counter() - t0)
    value = float(np.mean(samples))
    configs = None if args.no_configs else cpu_small_configs(args.seed)
    line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(secs)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded ring circuit, PCG64 prefixes)",
            "config": {"workload": args.workload, "block": "2^20", "precision": "complex128 CPU executor",
                       "kind": (f"extrapolated from {cb['steps_sampled']} of {cb['steps_total']} steps of one "
                                "slice: one step of this line is one bounded sample, not one 64-qubit sample"),
                       "step_seconds": per_step},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "configs": configs}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
GEN_COUNT = 2048  # samples of the 64-qubit generation protocol (the batched configuration's output)


def gpu_arm(args):
    import torch
    rank, world, local = dist_init()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from dcs245_classical_sampling_b200 import _lib
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    from dcs245_classical_sampling_b200.sampling import (draw_many, make_audit_ids, make_protocol, sample_checked,
                                                         straddle_margin)
    from dcs245_classical_sampling_b200.workloads import build_workload

    w = build_workload(args.workload)
    t0 = time.perf_counter()
    eng = InplaceConditionalBlockGPU(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                                     w["open_vertices"])
    eng.alloc(np.complex64, device=local, mode=args.mode, storage=args.storage)
    tune_report = None
    if args.mode == "fused" and args.tune:
        tune_report = eng.autotune(jit=not args.no_jit)
    if args.mode == "fused" and eng.fplan.tile_runs is not None and eng.jit == args.no_jit:
        eng.set_fused_config(jit=not args.no_jit)  # plan-specialised group kernels (NVRTC, cached cubins)
    if args.mode == "fused" and args.prefetch_kb is not None:
        eng.set_fused_config(prefetch_kb=args.prefetch_kb)
    group_report = None
    if args.mode == "fused" and args.tune_groups:
        group_report = eng.tune_groups()
    setup_s = time.perf_counter() - t0
    k = eng.k
    total = args.warmup + args.steps
    count = max(GEN_COUNT, total + args.plain_samples + 2)
    # generation protocol (PCG64 prefixes and uniforms) and, from a separate PCG64 stream chosen
    # before any sample is drawn, the audited sample ids (production/protocol_common.py:22-31)
    proto = make_protocol(args.seed + 1000 * rank, count, w["n"], w["open_vertices"])
    recs = proto["records"]
    xs = [np.array([int(c) for c in r["input_data_bits"]], np.uint8) for r in recs]
    us = [r["draw_uniform"] for r in recs]
    audit_ids = (make_audit_ids(args.audit_seed + 1000 * rank, count, 1, args.audits)[0]
                 if args.audits > 0 and not args.no_audit else [])
    stream = torch.cuda.current_stream(dev)

    # ---- device-resident throughput (value): inputs prepared and uploaded before timing
    preps = [eng.prepare([x]) for x in xs[:total]]
    d_us = torch.tensor(us[:total], dtype=torch.float64, device=dev)
    outs = torch.zeros((total, 1 << k), dtype=torch.complex128, device=dev)
    res = torch.empty((total, _lib.DRAW_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    lib = _lib.load()
    scratch = torch.empty(lib.dcs_draw_scratch_bytes(k, 1), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)

    def one(i, record=False):
        ev0 = torch.cuda.Event(enable_timing=True) if record else None
        if record:
            ev0.record(stream)
        launches = eng.enqueue(preps[i], outs[i:i + 1])
        _lib.check(lib.dcs_draw(_lib.ptr(outs[i]), k, 1, _lib.ptr(d_us[i:i + 1]), _lib.ptr(scratch),
                                _lib.ptr(res[i]), stream.cuda_stream))
        ev1 = None
        if record:
            ev1 = torch.cuda.Event(enable_timing=True)
            ev1.record(stream)
        return launches + 6, (ev0, ev1)

    for i in range(args.warmup):
        one(i)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    launches = 0
    lat_events = []
    for i in range(args.warmup, total):
        n, evs = one(i, record=True)
        launches += n
        lat_events.append(evs)
    stop.record(stream)
    torch.cuda.synchronize(dev)
    elapsed = start.elapsed_time(stop) / 1000.0
    clk = clocks.stop()
    if world > 1:
        t = torch.tensor([elapsed], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        elapsed = float(t.item())
    lat = sorted(a.elapsed_time(b) for a, b in lat_events)
    draws = res.cpu().numpy().view(_lib.DRAW_DTYPE).reshape(-1)
    value = args.steps * world / elapsed

    # ---- dominant kernel: time the contraction passes of one extra sample on their own
    dom = kernel_roofline(eng, preps[args.warmup], outs[args.warmup:args.warmup + 1], stream)

    # ---- end to end through the public API: host prefixes in; per sample the block, its host
    # copy, the checked draw with NumPy's exact CDF values and the SHA-256 of the weights and
    # amplitudes out (the reference worker's per-sample record, production/worker.py:105-113)
    sample_checked(eng, xs[:2], us[:2], hashes=True, exact_cdf=True)
    torch.cuda.synchronize(dev)
    ea = torch.cuda.Event(enable_timing=True)
    eb = torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    e2e_recs = sample_checked(eng, xs[args.warmup:total], us[args.warmup:total], hashes=True, exact_cdf=True)
    eb.record(stream)
    torch.cuda.synchronize(dev)
    e2e_elapsed = ea.elapsed_time(eb) / 1000.0
    h2d = preps[args.warmup]["h2d_bytes"] + 8  # params/coefs/xors/begin blob + the uniform
    d2h = (1 << k) * 16 + _lib.DRAW_DTYPE.itemsize + 8 * eng.items  # block + draw record + scale flags
    e2e_same = all(int(r["A_index"]) == int(d["index"]) for r, d in zip(e2e_recs, draws[args.warmup:total]))
    if world > 1:
        t = torch.tensor([e2e_elapsed], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_elapsed = float(t.item())

    # ---- precision audit, part 1: the audited samples' complex64 blocks with the timed executor
    audit_c64 = None
    if audit_ids and rank == 0:
        ta = time.perf_counter()
        xa = [xs[i] for i in audit_ids]
        ua = [us[i] for i in audit_ids]
        blocks_a = torch.empty((len(xa), 1 << k), dtype=torch.complex128, device=dev)
        for j, x in enumerate(xa):
            blocks_a[j] = eng.blocks([x])[0]
        draws_a = draw_many(blocks_a, ua)
        torch.cuda.synchronize(dev)
        audit_c64 = {"ids": audit_ids, "x": xa, "u": ua, "blocks": blocks_a, "draws": draws_a,
                     "seconds": time.perf_counter() - ta}

    fused_cfg = getattr(eng, "fused_config", None)
    if fused_cfg is not None:
        fused_cfg = {**fused_cfg, "jit": bool(getattr(eng.fplan, "jit", None)),
                     "group_cfg": {str(g): list(c) for g, c in (getattr(eng, "jit_group_cfg", None) or {}).items()}}
    del eng, preps, outs  # release the 128 GiB table before the other engines allocate theirs
    import gc
    gc.collect()
    torch.cuda.empty_cache()
    # ---- plain per-sample path (one launch + one host max read per step), same workload
    plain = None
    if not args.no_plain and args.plain_samples > 0 and rank == 0:
        from dcs245_classical_sampling_b200.sampling import draw_checked
        peng = InplaceConditionalBlockGPU(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                                          w["open_vertices"])
        peng.alloc(np.complex64, device=local, mode="plain")
        v, _ = peng.block(xs[total])
        torch.cuda.synchronize(dev)
        pa = torch.cuda.Event(enable_timing=True)
        pb = torch.cuda.Event(enable_timing=True)
        pa.record(stream)
        for i in range(args.plain_samples):
            v, _ = peng.block(xs[total + 1 + i])
            draw_checked(v, us[total + 1 + i], hashes=False)
        pb.record(stream)
        torch.cuda.synchronize(dev)
        plain_s = pa.elapsed_time(pb) / 1000.0 / args.plain_samples
        plain = {"value": 1.0 / plain_s, "unit": "samples/s", "samples": args.plain_samples,
                 "path": "one launch + one host max read per vertex step (reference control flow)"}
        del peng
        gc.collect()
        torch.cuda.empty_cache()

    # ---- precision audit, part 2: independent complex128 recontractions of the audited samples
    audit = None
    if audit_c64 is not None:
        audit = run_audit(args, audit_c64, local)
        del audit_c64

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = gpu_small_configs(args, local)

    serve = None
    if rank == 0 and world == 1 and not args.no_serve and args.workload == "ring64_d73_t314_k20":
        if plain is not None:
            args.plain_64q_seconds = 1.0 / plain["value"]
        serve = run_serving(args, local)

    if rank == 0:
        peak, how = peaks()
        cb = None
        if not args.no_cpu and world == 1:
            cb = cpu_baseline(args.workload, args.cpu_seconds)
            cb = {k2: cb[k2] for k2 in ("value", "unit", "cores", "kind", "sample")}
            if configs is not None:
                for name, c in cpu_small_configs(args.seed).items():
                    configs[name]["cpu"] = c
                    configs[name]["gpu_over_cpu"] = configs[name]["value"] / c["value"]
                    configs[name]["e2e_over_cpu"] = configs[name]["e2e"]["value"] / c["value"]
        ach = dom["alg_bytes_per_launch"] / dom["avg_launch_s"] / 1e9
        near = [bool(min(d["uniform"] - d["cdf_lower_exact"], d["cdf_upper_exact"] - d["uniform"])
                     < straddle_margin(float(d["weight_l2"]))) for d in draws[args.warmup:total]]
        line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f16 storage, f64 arithmetic" if args.storage else "c64",
                "data": "synthetic (seeded 64q ring circuit, PCG64 prefixes and uniforms)",
                "config": {"workload": args.workload, "block": f"2^{k}", "mode": args.mode,
                           "slices": 1 << len(w["parity_operations"]), "rmax": eng_rmax(w),
                           "table_bytes": (1 << eng_maxslots(w)) * (4 if args.storage else 8), "batch_per_step": 1,
                           "storage": args.storage or "complex64",
                           "l2": "inputs larger than L2 (128 GiB table per slice pass)",
                           "parallelism": f"replicas x{world}"},
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
                "e2e": {"value": args.steps * world / e2e_elapsed, "unit": "samples/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h,
                        "api": "sampling.sample_checked: engine blocks, host copy, checked draw with NumPy's exact "
                               "CDF values and both SHA-256 hashes per sample",
                        "same_indices_as_value": e2e_same},
                "gpu_launches": launches,
                "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                             "traffic": (TRAFFIC_RATIO[dom["kernel"]] * dom["alg_bytes_per_launch"]
                                         if dom["kernel"] in TRAFFIC_RATIO else None),
                             "traffic_note": "ncu dram bytes / algorithmic bytes of a smaller launch of the same "
                                             "kernel and plan, times this launch's algorithmic bytes",
                             "kernel": dom["kernel"],
                             "peak_source": f"{how} (MEASURED_PEAKS.json hbm_gbs)" if how == "measured" else
                             "fallback 6650 GB/s", "launches": dom["launches"],
                             "alg_bytes_per_launch": dom["alg_bytes_per_launch"],
                             "avg_launch_ms": dom["avg_launch_s"] * 1e3,
                             "per_launch": [[b, round(t, 4), round(b / t / 1e6 / peak, 4)]
                                            for b, t in zip(dom["launch_bytes"], dom["launch_ms"])],
                             "per_launch_fields": ["algorithmic bytes", "ms (CUDA events)", "fraction of peak"]},
                "compute": compute_view(dom, torch.cuda.get_device_properties(dev).multi_processor_count,
                                        float(clk.get("sm_mhz") or 1965.0) if isinstance(clk, dict) else 1965.0),
                "plain": plain, "speedup_vs_plain": (value / plain["value"]) if plain else None,
                "draws": {"indices": [int(d["index"]) for d in draws[args.warmup:total]],
                          "ties": int(sum(int(d["tie"]) for d in draws[args.warmup:total])),
                          "near_cdf_edge": int(sum(near)),
                          "near_cdf_edge_margin": "sampling.straddle_margin: 6 sigma of the CDF shift of a block "
                                                  "at relative L2 1e-5 with independent per-entry errors",
                          "straddles_audited": audit["straddles"] if audit else None},
                "clocks": clk, "setup_s": setup_s, "cpu_baseline": cb, "audit": audit,
                "configs": configs, "serve": serve,
                "fused_config": fused_cfg,
                "autotune": tune_report, "tune_groups": group_report}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_audit(args, a64, local):
    """Config 4: the audited samples' complex64 blocks (contracted by the timed executor) against
    independent complex128 recontractions with a different slicing (one more parity slice: rmax
    33, a 128 GiB complex128 table), as the reference's audits use inplace_k3_fp64 next to
    inplace_k2_fp32 (production/worker.py:137-170).  Per sample: c_y (the normalised overlap,
    review/full_vector_audit_certificate.py:36), relative L2 error, and the indices both blocks
    select with the sample's uniform; a differing index is a straddle of a CDF edge and must lie
    within the complex64 margin of it."""
    import gc
    import torch
    from dcs245_classical_sampling_b200.audit import audit_vector_pair, relative_l2
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    from dcs245_classical_sampling_b200.sampling import CDF_SHIFT_BOUND, draw_many
    from dcs245_classical_sampling_b200.workloads import WORKLOADS, build_workload
    gc.collect()
    torch.cuda.empty_cache()
    name = args.workload + "_audit" if args.workload + "_audit" in WORKLOADS else args.workload
    wa = build_workload(name)
    t0 = time.perf_counter()
    ref = InplaceConditionalBlockGPU(wa["graph"], wa["unitaries"], wa["n"], wa["order"], wa["parity_operations"],
                                     wa["open_vertices"])
    ref.alloc(np.complex128, device=local, mode=args.audit_mode)
    setup = time.perf_counter() - t0
    rows, secs = [], []
    straddles, bad = 0, 0
    for j, sid in enumerate(a64["ids"]):
        ts = time.perf_counter()
        v, meta = ref.block(a64["x"][j])
        secs.append(time.perf_counter() - ts)
        ap = a64["blocks"][j]
        rec = audit_vector_pair(v, ap, sid)
        i128 = int(draw_many(v.unsqueeze(0), [a64["u"][j]])[0]["index"])
        d64 = a64["draws"][j]
        i64 = int(d64["index"])
        if i64 != i128:
            straddles += 1
            near = min(d64["uniform"] - d64["cdf_lower_exact"], d64["cdf_upper_exact"] - d64["uniform"])
            bad += int(not near < CDF_SHIFT_BOUND)
        rows.append([int(sid), rec["normalized_conditional_overlap_abs"], relative_l2(v, ap), i64, i128])
    rmax = ref.inplace_rmax
    del ref
    gc.collect()
    torch.cuda.empty_cache()
    cy = [r[1] for r in rows]
    rl = [r[2] for r in rows]
    return {"plan": wa["name"], "rmax": rmax, "audited": len(rows), "mode": args.audit_mode,
            "ids": "64 of the 2048 generation samples, chosen before generation by an independent PCG64 stream "
                   f"(seed {args.audit_seed}, protocol_common.py:22-31)",
            "min_c_y": min(cy) if cy else None, "mean_c_y": float(np.mean(cy)) if cy else None,
            "max_rel_l2": max(rl) if rl else None, "mean_rel_l2": float(np.mean(rl)) if rl else None,
            "all_c_y_ge_0.9999": all(c >= 0.9999 for c in cy), "all_rel_l2_lt_1e-5": all(x < 1e-5 for x in rl),
            "straddles": straddles, "straddles_outside_margin": bad,
            "complex128_seconds_per_block": float(np.mean(secs)) if secs else None, "complex128_setup_s": setup,
            "complex64_seconds": a64["seconds"],
            "rows_fields": ["sample id", "c_y", "rel L2", "index (complex64)", "index (complex128)"],
            "rows": rows}


def gpu_small_configs(args, local):
    """The small workloads measured completely on the GPU: device-resident samples/s (inputs
    prepared and uploaded first), end to end through sampling.sample_checked, and c_y of a few
    samples against complex128 recontractions."""
    import gc
    import torch
    from dcs245_classical_sampling_b200 import _lib
    from dcs245_classical_sampling_b200.audit import audit_vector_pair
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    from dcs245_classical_sampling_b200.sampling import make_protocol, sample_checked
    from dcs245_classical_sampling_b200.workloads import build_workload
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    out = {}
    for name, cfg in SMALL_CONFIGS.items():
        w = build_workload(name)
        args6 = (w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"], w["open_vertices"])
        eng = InplaceConditionalBlockGPU(*args6)
        eng.alloc(np.complex64, device=local, mode=cfg["mode"])
        if cfg["mode"] == "fused":
            eng.set_fused_config(variant=12, low=3, grouping="bytes", jit=True)
        recs = make_protocol(args.seed, cfg["samples"], w["n"], w["open_vertices"])["records"]
        xs = [np.array([int(c) for c in r["input_data_bits"]], np.uint8) for r in recs]
        us = [r["draw_uniform"] for r in recs]
        k = eng.k
        preps = [eng.prepare([x]) for x in xs]
        outs = torch.empty((len(xs), 1 << k), dtype=torch.complex128, device=dev)
        d_us = torch.tensor(us, dtype=torch.float64, device=dev)
        res = torch.empty((len(xs), _lib.DRAW_DTYPE.itemsize), dtype=torch.uint8, device=dev)
        lib = _lib.load()
        scratch = torch.empty(lib.dcs_draw_scratch_bytes(k, 1), dtype=torch.uint8, device=dev)
        for i in range(min(3, len(xs))):
            eng.enqueue(preps[i], outs[i:i + 1])
        torch.cuda.synchronize(dev)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for i in range(len(xs)):
            eng.enqueue(preps[i], outs[i:i + 1])
            _lib.check(lib.dcs_draw(_lib.ptr(outs[i]), k, 1, _lib.ptr(d_us[i:i + 1]), _lib.ptr(scratch),
                                    _lib.ptr(res[i]), stream.cuda_stream))
        b.record(stream)
        torch.cuda.synchronize(dev)
        value = len(xs) / (a.elapsed_time(b) / 1000.0)
        sample_checked(eng, xs[:3], us[:3], hashes=True, exact_cdf=True)
        torch.cuda.synchronize(dev)
        a.record(stream)
        e2e_recs = sample_checked(eng, xs, us, hashes=True, exact_cdf=True)
        b.record(stream)
        torch.cuda.synchronize(dev)
        e2e = len(xs) / (a.elapsed_time(b) / 1000.0)
        idx = [int(d["index"]) for d in res.cpu().numpy().view(_lib.DRAW_DTYPE).reshape(-1)]
        same = idx == [r["A_index"] for r in e2e_recs]
        ref = InplaceConditionalBlockGPU(*args6)
        ref.alloc(np.complex128, device=local, mode="device")
        cy = []
        for i in range(4):
            v128, _ = ref.block(xs[i])
            cy.append(audit_vector_pair(v128, outs[i], i)["normalized_conditional_overlap_abs"])
        out[name] = {"value": value, "unit": "samples/s", "samples": len(xs), "mode": cfg["mode"],
                     "e2e": {"value": e2e, "unit": "samples/s", "h2d_bytes_per_step": preps[0]["h2d_bytes"] + 8,
                             "d2h_bytes_per_step": (1 << k) * 16 + _lib.DRAW_DTYPE.itemsize + 8 * eng.items},
                     "e2e_same_indices": same, "min_c_y_4_audits": min(cy), "indices_head": idx[:8]}
        del eng, ref, preps, outs
        gc.collect()
        torch.cuda.empty_cache()
    return out


def eng_rmax(w):
    from dcs245_classical_sampling_b200 import plan as P
    bp = P.build_block_plan(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                            w["open_vertices"])
    return bp.inplace_rmax


def eng_maxslots(w):
    return eng_rmax(w)


def kernel_roofline(eng, prep, out, stream):
    """Average duration and algorithmic bytes of the dominant contraction kernel, from CUDA
    events around each of its launches (one slice of one sample)."""
    import torch
    from dcs245_classical_sampling_b200 import _lib
    lib = eng.lib
    plan = eng.plan
    c0, cn, b0, nb, boff = prep["chunks"][0]
    eng._reset_items(cn)
    evs = []
    params_ptr = _lib.ptr(prep["params"])
    if eng.mode == "fused":
        f = eng.fplan
        for g in range(len(f.groups)):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib.check(f.launch(lib, _lib.ptr(eng.table), params_ptr, g, 1, _lib.ptr(eng.maxbits),
                                _lib.ptr(eng.scale), stream.cuda_stream))
            b.record(stream)
            first, count = f.spans[g]
            alg = ((1 << len(plan.steps[first].active_in)) + (1 << len(plan.steps[first + count - 1].active_out))) * 8
            evs.append((a, b, alg))
        kernel = ("dcs_g (plan-specialised k_runs)" if f.jit is not None else "k_runs") \
            if f.tile_runs is not None and bool((f.groups["variant"] & 4).any()) else "k_fused"
    else:
        for s in range(eng.nsteps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib.check(lib.dcs_slice_steps_batched(eng.dcode, _lib.ptr(eng.table), eng.table_stride,
                                                   eng.dsteps.ctypes.data, params_ptr, eng.nsteps, eng.nsteps, s, 1,
                                                   _lib.ptr(eng.maxbits), _lib.ptr(eng.scale), cn,
                                                   stream.cuda_stream))
            b.record(stream)
            st = plan.steps[s]
            entry = 16 if eng.use_fp64 else (4 if eng.half else 8)
            evs.append((a, b, ((1 << len(st.active_in)) + (1 << len(st.active_out))) * entry))
        kernel = "k_step"
    torch.cuda.synchronize()
    tot_t = sum(a.elapsed_time(b) for a, b, _ in evs) / 1000.0
    tot_b = sum(x for _, _, x in evs)
    n = len(evs)
    # entry-steps of each launch: every vertex step touches 2^max(|in|, |out|) table entries
    spans = eng.fplan.spans if eng.mode == "fused" else [(s, 1) for s in range(eng.nsteps)]
    entry_steps = [sum(1 << max(len(st.active_in), len(st.active_out)) for st in plan.steps[f0:f0 + c])
                   for f0, c in spans]
    prm = prep["params"][:eng.nsteps * _lib.PARAM_DTYPE.itemsize // 8].cpu().numpy().view(_lib.PARAM_DTYPE)
    ops = [sum(step_fp32_ops(st, int(prm[f0 + i]["y"])) for i, st in enumerate(plan.steps[f0:f0 + c]))
           for f0, c in spans]
    return {"kernel": kernel, "launches": n, "avg_launch_s": tot_t / n, "alg_bytes_per_launch": tot_b / n,
            "launch_ms": [a.elapsed_time(b) for a, b, _ in evs], "launch_bytes": [x for _, _, x in evs],
            "launch_entry_steps": entry_steps, "launch_fp32_ops": ops}


def step_fp32_ops(st, y):
    """FP32 operations (add, multiply or fused multiply-add, one each) of one vertex step in the
    unit-weight form the generated kernels evaluate (each free step's f0 divided out, f = f1/f0,
    signs chosen, not multiplied), per the n = 2^|in| input entries.  A grow multiplies each new
    entry by f (4n); a mix forms both entries of an orbit as x + f y (4n); a diagonal mix or a
    fixed step with y = 1 multiplies (4n), a fixed step with y = 0 copies (0).  A replace, a
    two-entry shrink and a four-entry shrink need a + b, and a - b only where the partner sign
    parity(K & beta) is odd (else a + b is reused): 3n, or 4n with the odd sign; a fixed shrink
    adds (n) or adds and multiplies (3n)."""
    from dcs245_classical_sampling_b200.plan import orbit_kind
    kind = orbit_kind(st)[0]
    n = 1 << len(st.active_in)
    if kind == 4:
        return 4 * n if y else 0
    if kind == 5:
        return 3 * n if y else n
    if kind in (3, 6, 7):
        return (4 if bin(st.K & st.beta).count("1") & 1 else 3) * n
    return 4 * n


def compute_view(dom, sms, sm_mhz):
    """The contraction's other bound: entry-steps (one table entry through one vertex step) per
    second.  Inside a fused group the tables grow well beyond the group's input and output (up
    to 2^34 entries on the 64-qubit plan while the pass reads 2^32 and writes 2^30), so the large
    groups are bound by the arithmetic and shared-memory work per entry-step, not by HBM."""
    t = sum(dom["launch_ms"]) / 1000.0
    es = dom["launch_entry_steps"]
    big = sorted(range(len(es)), key=lambda i: -dom["launch_ms"][i])[:3]
    ops = dom["launch_fp32_ops"]
    peak = sms * 128 * sm_mhz * 1e6 / 1e12  # FP32 pipe: 128 lanes per SM per clock (FFMA or FFMA2)
    return {"bound": "fp32", "unit": "TFLOP/s (FP32 operations of the unit-weight step formulas)",
            "achieved": sum(ops) / t / 1e12, "peak": peak, "frac": sum(ops) / t / 1e12 / peak,
            "peak_source": f"{sms} SMs x 128 FP32 lanes x {sm_mhz:.0f} MHz (median SM clock of the timed "
                           "region); a register-resident FFMA / FFMA2 loop measured 127-130 per SM per clock",
            "entry_steps_per_s": sum(es) / t, "entry_steps_per_slice": sum(es), "fp32_ops_per_slice": sum(ops),
            "ps_per_entry_step": 1e12 * t / sum(es),
            "slowest_launches": [[i, es[i], round(dom["launch_ms"][i], 4),
                                  round(ops[i] / dom["launch_ms"][i] / 1e9 / peak, 4)] for i in big],
            "slowest_launches_fields": ["launch", "entry-steps", "ms", "fraction of the FP32 peak"]}


SERVE_MIX = {"ring32_d37_t79_k14": 50, "ring48_d55_t177_k17": 30, "ring64_d73_t314_k20": 20}


def run_serving(args, local):
    """Serving mix: Poisson requests against the three circuits (32q 2^14, 48q 2^17, 64q 2^20 blocks;
    50/30/20 by request count, 1-64 samples each), continuous batching with round-robin batches,
    and admission by HBM budget (one table pool granted per batch; graphs=True keeps fixed
    per-runner tables instead, captured as CUDA graphs).  Compared with plain per-request
    execution: every request alone, in arrival order, one sample at a time on the plain path (one
    launch and one host read per vertex step), whose per-sample times are measured here."""
    import gc
    import torch
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    from dcs245_classical_sampling_b200.sampling import draw_checked, make_protocol
    from dcs245_classical_sampling_b200.serve import (CircuitRunner, Request, Server, TablePool, latency_stats,
                                                      poisson_requests)
    from dcs245_classical_sampling_b200.workloads import build_workload
    dev = torch.device("cuda", local)
    gc.collect()
    torch.cuda.empty_cache()
    budget = int(args.hbm_budget_gib * 2 ** 30)
    t0 = time.perf_counter()
    pool = None if args.graphs else TablePool(budget, dev)
    runners = {}
    for i, name in enumerate(SERVE_MIX):
        w = build_workload(name)
        big = name.startswith("ring64")
        kw = {"pool": pool} if pool is not None else (
            {} if big else {"hbm_budget": (budget - (8 << 34)) * (0.8 if name.startswith("ring48") else 0.2),
                            "graphs": True})
        runners[name] = CircuitRunner(name, w, key=args.seed + 64 + i, max_samples=1 if big else 64,
                                      device=local, **kw)
    for r in runners.values():  # every batch size captured before the arrivals start
        r.precapture(range(1, r.max_samples + 1))
    setup = time.perf_counter() - t0
    Server(runners, pool).run([Request(10 ** 6 + i, c, 1, 0.0) for i, c in enumerate(runners)], realtime=False)
    reqs = poisson_requests(args.serve_rate, args.serve_seconds, SERVE_MIX, seed=args.seed,
                            max_samples=args.serve_max_samples)
    clocks = ClockSampler(local)
    clocks.start()
    ta = time.perf_counter()
    done = Server(runners, pool).run(reqs, realtime=True)
    span = time.perf_counter() - ta
    clk = clocks.stop()
    per = {}
    for r in done:
        d = per.setdefault(r.circuit, {"requests": 0, "samples": 0, "lat_ms": []})
        d["requests"] += 1
        d["samples"] += r.nsamples
        d["lat_ms"].append((r.finish - r.arrival) * 1e3)
    for d in per.values():
        lat = d.pop("lat_ms")
        d["p50_ms"], d["p99_ms"] = float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
    tot = sum(r.nsamples for r in done)
    ties = sum(int(rec["tie"]) for r in done for rec, _ in r.records.values())
    bad = sum(int(rec["status"] != 0) for r in done for rec, _ in r.records.values())
    slots = {c: {"samples_per_launch": r.max_samples, "table_item_gib": r.item_bytes / 2 ** 30, "mode": r.mode}
             for c, r in runners.items()}
    pool_free_after = None if pool is None else pool.free == [(0, pool.nbytes)]
    del runners, pool, kw
    gc.collect()
    torch.cuda.empty_cache()
    # plain per-request execution: measured per-sample times of the plain path per circuit
    plain_s = {}
    for name in SERVE_MIX:
        if name.startswith("ring64") and args.plain_64q_seconds:
            plain_s[name] = args.plain_64q_seconds
            continue
        w = build_workload(name)
        eng = InplaceConditionalBlockGPU(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                                         w["open_vertices"])
        eng.alloc(np.complex64, device=local, mode="plain")
        recs = make_protocol(args.seed, 4, w["n"], w["open_vertices"])["records"]
        xs = [np.array([int(c) for c in r["input_data_bits"]], np.uint8) for r in recs]
        v, _ = eng.block(xs[0])
        n = 1 if name.startswith("ring64") else 3
        tp = time.perf_counter()
        for i in range(n):
            v, _ = eng.block(xs[1 + i])
            draw_checked(v, recs[1 + i]["draw_uniform"], hashes=False)
        plain_s[name] = (time.perf_counter() - tp) / n
        del eng
        gc.collect()
        torch.cuda.empty_cache()
    # the same arrivals served one request at a time, first come first served (a single queue)
    tfree, plain_lat = 0.0, []
    for r in sorted(reqs, key=lambda q: q.arrival):
        start = max(tfree, r.arrival)
        tfree = start + r.nsamples * plain_s[r.circuit]
        plain_lat.append((tfree - r.arrival) * 1e3)
    plain_span = tfree - min(r.arrival for r in reqs) if reqs else 0.0
    plain_busy = sum(r.nsamples * plain_s[r.circuit] for r in reqs)
    return {"metric": "serving mix: samples/s and request p50/p99 ms (32q 2^14, 48q 2^17, 64q 2^20; 50/30/20)",
            "value": tot / span, "unit": "samples/s", "higher_is_better": True,
            "latency": latency_stats(done), "per_circuit": per, "requests": len(done), "samples": tot,
            "span_s": span, "arrival_window_s": args.serve_seconds, "rate_hz": args.serve_rate,
            "hbm_budget_gib": args.hbm_budget_gib,
            "admission": "per-batch table grants from one HBM pool" if not args.graphs else
                         "fixed per-runner tables (CUDA graphs)",
            "pool_returned_every_region": pool_free_after,
            "slots": slots, "ties": ties, "failed_draws": bad, "cuda_graphs": bool(args.graphs), "setup_s": setup,
            "clocks": clk,
            "plain_per_request": {
                "seconds_per_sample": plain_s,
                "value": tot / plain_busy if plain_busy else None, "unit": "samples/s",
                "p50_ms": float(np.percentile(plain_lat, 50)) if plain_lat else None,
                "p99_ms": float(np.percentile(plain_lat, 99)) if plain_lat else None,
                "span_s": plain_span,
                "how": "measured per-sample plain-path times; requests served alone in arrival order "
                       "(single FIFO queue computed from those times)"},
            "speedup_vs_plain": (tot / span) / (tot / plain_busy) if plain_busy else None,
            "data": "synthetic (seeded ring circuits, Philox4x32-10 prefixes and uniforms on the device)"}


def serve_arm(args):
    """`bench.py --serve`: the serving mix alone, as its own JSON line."""
    import torch
    rank, world, local = dist_init()
    torch.cuda.set_device(local)
    line = run_serving(args, local)
    line["n_gpus"] = 1
    print(json.dumps(line), flush=True)


def profile_case(argv):
    """Small, self-contained profiling case for the contraction kernels (the cases the ncu
    summaries under profiles/ capture).

    Runs the first vertex steps of a workload's plan whose table stays within 2^max_slots
    entries (default 2^28 complex64 = 2 GiB: larger than L2, small enough for a full ncu
    capture), for one prefix and one slice, `iters` times, with either the fused kernels or the
    per-step kernel.  Prints one JSON line with the per-launch CUDA-event timings.

        python bench.py --profile-case [--mode fused|device] [--max-slots 28] [--storage float16] ..."""
    import torch

    from dcs245_classical_sampling_b200 import _lib
    from dcs245_classical_sampling_b200 import plan as P
    from dcs245_classical_sampling_b200.engine import SliceParams, device_steps
    from dcs245_classical_sampling_b200.fused import build_fused_plan
    from dcs245_classical_sampling_b200.sampling import make_protocol
    from dcs245_classical_sampling_b200.workloads import build_workload

    ap = argparse.ArgumentParser(prog="bench.py --profile-case")
    ap.add_argument("--workload", default="ring64_d73_t314_k20")
    ap.add_argument("--mode", default="fused", choices=["fused", "device"])
    ap.add_argument("--max-slots", type=int, default=28)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--max-dim", type=int, default=13)
    ap.add_argument("--low", type=int, default=4)
    ap.add_argument("--variant", type=int, default=0)
    ap.add_argument("--pairs", action="store_true", help="two steps per shared-memory round trip")
    ap.add_argument("--jit", action="store_true", help="plan-specialised group kernels (register-run variants)")
    ap.add_argument("--grouping", default="greedy", choices=["greedy", "bytes"],
                    help="fused groups: greedy spans or fewest table bytes")
    ap.add_argument("--prefetch-kb", type=int, default=0,
                    help="generated kernels: KiB per CTA staging the next tile's first-run entries")
    ap.add_argument("--minb", type=int, default=None, help="generated kernels: CTAs per SM for the registers")
    ap.add_argument("--fp64", action="store_true", help="complex128 table, FP64 generated kernels (the audits)")
    ap.add_argument("--kernel-cfg", default=None,
                    help="generated kernels of every group as MINB/STAGING_KB/RUN_DIM[/THREADS], e.g. 2/16/5; "
                         "RUN_DIM 4t or 5t: run bases that may touch other roles")
    ap.add_argument("--storage", default=None, choices=["float16"],
                    help="binary16 tables with FP64 arithmetic (device mode)")
    a = ap.parse_args(argv)
    lib = _lib.load()
    w = build_workload(a.workload)
    bp = P.build_block_plan(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                            w["open_vertices"])
    last = 0
    for j, st in enumerate(bp.steps):
        top = max(st.active_in + st.active_out + (0,)) + 1
        if st.kind == "grow":
            top = max(top, st.pivot + 1)
        if top > a.max_slots:
            break
        last = j + 1
    steps = bp.steps[:last]
    proto = make_protocol(5, 1, w["n"], w["open_vertices"])
    x = np.array([int(c) for c in proto["records"][0]["input_data_bits"]], np.uint8)
    _, items = SliceParams(bp).items(x)
    params = torch.from_numpy(items[0][1][:last].copy().view(np.int64)).cuda()
    dev = torch.device("cuda", 0)
    half = a.storage == "float16"
    if half and a.mode != "device":
        raise SystemExit("--storage float16 takes --mode device")
    if a.fp64 and (a.mode != "fused" or not a.jit or half):
        raise SystemExit("--fp64 takes --mode fused --jit (the complex128 generated kernels)")
    entry = 4 if half else (16 if a.fp64 else 8)
    if half:
        table = torch.zeros(2 << a.max_slots, dtype=torch.float16, device=dev)
    else:
        table = torch.zeros(1 << a.max_slots, dtype=torch.complex128 if a.fp64 else torch.complex64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sub = P.BlockPlan(**{**bp.__dict__, "steps": steps})
    if a.mode == "fused":
        variant, minb, kb = a.variant, a.minb, a.prefetch_kb
        threads = 256
        if a.kernel_cfg:
            parts = a.kernel_cfg.split("/")
            minb, kb = int(parts[0]), int(parts[1])
            rdim = parts[2]
            variant = (variant | 16) if rdim.startswith("5") else (variant & ~16)
            variant = (variant | 64) if rdim.endswith("t") else (variant & ~64)
            if len(parts) > 3:
                threads = int(parts[3])
        fp = build_fused_plan(sub, max_dim=a.max_dim, low=a.low, variant=variant, pairs=a.pairs,
                              grouping=a.grouping, fp64=a.fp64, prefetch_kb=kb)
        if a.jit:
            from dcs245_classical_sampling_b200.jit import JitPlan
            fp.jit = JitPlan(sub, fp, lib, minb=minb, threads=threads)
        nmax = len(fp.groups)
    else:
        dsteps = device_steps(steps)
        nmax = last
    maxbits = torch.zeros(nmax + 1, dtype=torch.int64, device=dev)
    scale = torch.zeros(_lib.SCALE_DTYPE.itemsize // 8, dtype=torch.int64, device=dev)
    one = (int(np.array([1.0], np.float64).view(np.int64)[0]) if half or a.fp64
           else int(np.array([1.0], np.float32).view(np.uint32)[0]))
    per_launch = []
    for it in range(a.iters):
        maxbits.zero_()
        maxbits[0] = one
        scale.zero_()
        if half:
            table[0], table[1] = 1, 0
        else:
            table[0] = 1
        evs = []
        for g in range(nmax):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if a.mode == "fused":
                _lib.check(fp.launch(lib, _lib.ptr(table), _lib.ptr(params), g, 1, _lib.ptr(maxbits),
                                     _lib.ptr(scale), stream.cuda_stream))
                first, count = fp.spans[g]
                alg = ((1 << len(steps[first].active_in)) + (1 << len(steps[first + count - 1].active_out))) * entry
            else:
                _lib.check(lib.dcs_slice_steps(_lib.H16 if half else _lib.C64, _lib.ptr(table), dsteps.ctypes.data,
                                               _lib.ptr(params), last, g, 1, _lib.ptr(maxbits), _lib.ptr(scale),
                                               stream.cuda_stream))
                alg = ((1 << len(steps[g].active_in)) + (1 << len(steps[g].active_out))) * entry
            e1.record(stream)
            evs.append((e0, e1, alg))
        torch.cuda.synchronize(dev)
        if it == a.iters - 1:
            per_launch = [(x0.elapsed_time(x1), alg) for x0, x1, alg in evs]
    tot_ms = sum(t for t, _ in per_launch)
    tot_b = sum(b for _, b in per_launch)
    big = [(t, b) for t, b in per_launch if b >= (1 << 27) * entry]
    # integer sum of the table's words: equal for variants that compute the same values bit for bit
    checksum = int(torch.sum(table.view(torch.int32), dtype=torch.int64).item())
    print(json.dumps({"mode": a.mode, "storage": a.storage or ("complex128" if a.fp64 else "complex64"),
                      "prefetch_kb": a.prefetch_kb, "checksum": checksum, "steps": last, "launches": len(per_launch), "total_ms": tot_ms,
                      "alg_gb": tot_b / 1e9, "alg_gbs": tot_b / tot_ms / 1e6,
                      "big_launch_gbs": (sum(b for _, b in big) / sum(t for t, _ in big) / 1e6) if big else None,
                      "per_launch_ms": [round(t, 3) for t, _ in per_launch]}))


def main():
    if "--profile-case" in sys.argv[1:]:
        profile_case([x for x in sys.argv[1:] if x != "--profile-case"])
        return
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.serve:
        serve_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
