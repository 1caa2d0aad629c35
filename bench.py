"""Benchmark: conditional-block sampling of the synthetic 64-qubit ring workload on B200.

One step = one sample of the hot path: the 2^20 conditional block of one 44-bit prefix
(complex64 contraction over all parity slices, complex128 coherent sum + tail) and the FP64
CDF draw of its 20 free bits.  Workload: 64-qubit ring, depth 73, 314 T gates (378-vertex
injected graph), 2 parity slices (4 slices, rmax 34: one 128 GiB complex64 table), PCG64
prefixes/uniforms from make_protocol.  Inputs and tables are far larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]
                    [--mode fused|device|plain] [--no-plain] [--no-cpu]

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
    ap.add_argument("--audits", type=int, default=2, help="timed samples audited in complex128")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--seed", type=int, default=24520)
    ap.add_argument("--tune", action="store_true", help="autotune the fused tile shape before timing")
    ap.add_argument("--no-jit", action="store_true",
                    help="run the library's register-run kernel instead of the plan-specialised group kernels")
    ap.add_argument("--serve", action="store_true", help="run the serving mix (32q/48q/64q) instead")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="arrival window of the serving run")
    ap.add_argument("--serve-rate", type=float, default=1.0, help="Poisson request rate (1/s)")
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
    per-sample algorithmic bytes (complex128, all slices)."""
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
            "sample": (f"C/OpenMP complex128 executor over the first {last} of {len(bp.steps)} steps of one slice "
                       f"(tables <= 2^{cap}), {reps} reps in {dt:.1f} s = {bps / 1e9:.2f} GB/s algorithmic; "
                       f"samples/s = that rate / {per_sample / 2**40:.2f} TiB per sample (all {len(items)} slices)"),
            "seconds": dt, "algorithmic_gbs": bps / 1e9}


def reference_arm(args):
    rank, world, _ = dist_init()
    if rank != 0:
        return
    samples = []
    cb = None
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(args.workload, max(2.0, args.cpu_seconds / 3))
        if i >= args.warmup:
            samples.append(cb["value"])
    value = float(np.mean(samples))
    line = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded ring circuit, PCG64 prefixes)",
            "config": {"workload": args.workload, "block": "2^20", "precision": "complex128 CPU executor"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
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
    from dcs245_classical_sampling_b200 import plan as P
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    from dcs245_classical_sampling_b200.sampling import make_protocol
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
    setup_s = time.perf_counter() - t0
    k = eng.k
    total = args.warmup + args.steps
    proto = make_protocol(args.seed + 1000 * rank, total + args.plain_samples + 2, w["n"], w["open_vertices"])
    recs = proto["records"]
    xs = [np.array([int(c) for c in r["input_data_bits"]], np.uint8) for r in recs]
    us = [r["draw_uniform"] for r in recs]
    stream = torch.cuda.current_stream(dev)

    # ---- device-resident throughput (value): inputs prepared and uploaded before timing
    preps = [eng.prepare([x]) for x in xs[:total]]
    d_us = torch.tensor(us[:total], dtype=torch.float64, device=dev)
    outs = torch.zeros((total, 1 << k), dtype=torch.complex128, device=dev)
    res = torch.empty((total, _lib.DRAW_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    lib = _lib.load()
    scratch = torch.empty(lib.dcs_draw_scratch_bytes(k, 1), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)

    group_events = []

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

    # ---- end to end through the public API (host prefixes in, host record out)
    from dcs245_classical_sampling_b200.sampling import draw_checked
    e2e_x = xs[:total]
    for i in range(min(2, args.warmup)):
        v, _ = eng.block(e2e_x[i])
        draw_checked(v, us[i], hashes=False)
    torch.cuda.synchronize(dev)
    ea = torch.cuda.Event(enable_timing=True)
    eb = torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    h2d = 0
    for i in range(args.warmup, total):
        v, _ = eng.block(e2e_x[i])
        d = draw_checked(v, us[i], hashes=False)
    eb.record(stream)
    torch.cuda.synchronize(dev)
    e2e_elapsed = ea.elapsed_time(eb) / 1000.0
    h2d = preps[args.warmup]["h2d_bytes"] + 8  # params/coefs/xors/begin blob + the uniform
    d2h = _lib.DRAW_DTYPE.itemsize + 8  # draw record + the scale-flag word
    if world > 1:
        t = torch.tensor([e2e_elapsed], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_elapsed = float(t.item())

    fused_cfg = getattr(eng, "fused_config", None)
    if fused_cfg is not None:
        fused_cfg = {**fused_cfg, "jit": bool(getattr(eng.fplan, "jit", None))}
    eng_items = eng.items
    blocks64 = outs[args.warmup:total].clone()
    del eng, preps, outs  # release the 128 GiB table before the other engines allocate theirs
    import gc
    gc.collect()
    torch.cuda.empty_cache()
    # ---- plain per-sample path (one launch + one host max read per step), same workload
    plain = None
    if not args.no_plain and args.plain_samples > 0 and rank == 0:
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
        torch.cuda.empty_cache()

    # ---- precision audit: independent complex128 recontraction (3-slice plan) of timed samples
    audit = None
    if not args.no_audit and rank == 0:
        audit = run_audit(args, xs, blocks64, local)

    if rank == 0:
        peak, how = peaks()
        cb = None
        if not args.no_cpu and world == 1:
            cb = cpu_baseline(args.workload, args.cpu_seconds)
            cb = {k2: cb[k2] for k2 in ("value", "unit", "cores", "kind", "sample")}
        ach = dom["alg_bytes_per_launch"] / dom["avg_launch_s"] / 1e9
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
                        "d2h_bytes_per_step": d2h},
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
                             "avg_launch_ms": dom["avg_launch_s"] * 1e3, "launch_ms": dom["launch_ms"]},
                "plain": plain, "speedup_vs_plain": (value / plain["value"]) if plain else None,
                "draws": {"indices": [int(d["index"]) for d in draws[args.warmup:total]],
                          "ties": int(sum(int(d["tie"]) for d in draws[args.warmup:total]))},
                "clocks": clk, "setup_s": setup_s, "cpu_baseline": cb, "audit": audit,
                "fused_config": fused_cfg,
                "autotune": tune_report}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_audit(args, xs, blocks64, local):
    """c_y of the timed complex64 blocks against an independent complex128 recontraction with a
    different slicing (one more parity slice: rmax 33, 128 GiB complex128), as the reference's
    audits use inplace_k3_fp64 next to inplace_k2_fp32."""
    import gc
    import torch
    from dcs245_classical_sampling_b200.audit import audit_vector_pair, relative_l2
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    from dcs245_classical_sampling_b200.workloads import build_workload
    gc.collect()
    torch.cuda.empty_cache()
    wa = build_workload(args.workload + "_audit") if args.workload + "_audit" in __import__(
        "dcs245_classical_sampling_b200.workloads", fromlist=["WORKLOADS"]).WORKLOADS else build_workload(args.workload)
    ref = InplaceConditionalBlockGPU(wa["graph"], wa["unitaries"], wa["n"], wa["order"], wa["parity_operations"],
                                     wa["open_vertices"])
    ref.alloc(np.complex128, device=local, mode="device")
    rows = []
    n = min(args.audits, blocks64.shape[0])
    for i in range(n):
        x = xs[args.warmup + i]
        t0 = time.perf_counter()
        v, meta = ref.block(x)
        sec = time.perf_counter() - t0
        rec = audit_vector_pair(v, blocks64[i], args.warmup + i)
        rows.append({"sample": args.warmup + i, "c_y": rec["normalized_conditional_overlap_abs"],
                     "rel_l2": relative_l2(v, blocks64[i]), "ref_seconds": sec})
    del ref
    gc.collect()
    torch.cuda.empty_cache()
    cy = [r["c_y"] for r in rows]
    return {"plan": wa["name"], "rmax": None, "audited": rows, "min_c_y": min(cy) if cy else None,
            "mean_c_y": float(np.mean(cy)) if cy else None, "all_c_y_ge_0.9999": all(c >= 0.9999 for c in cy)}


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
    return {"kernel": kernel, "launches": n, "avg_launch_s": tot_t / n, "alg_bytes_per_launch": tot_b / n,
            "launch_ms": [round(a.elapsed_time(b), 3) for a, b, _ in evs]}


def serve_arm(args):
    """Serving mix: Poisson requests against three circuits, continuous batching, p50/p99."""
    import torch
    from dcs245_classical_sampling_b200.serve import CircuitRunner, Server, latency_stats, poisson_requests
    from dcs245_classical_sampling_b200.workloads import build_workload
    rank, world, local = dist_init()
    torch.cuda.set_device(local)
    mix = {"ring32_d37_t79_k14": 50, "ring48_d55_t177_k17": 30, "ring64_d73_t314_k20": 20}
    budget = args.hbm_budget_gib * 2 ** 30
    t0 = time.perf_counter()
    runners = {}
    big = CircuitRunner("ring64_d73_t314_k20", build_workload("ring64_d73_t314_k20"), key=args.seed + 64,
                        max_samples=1, device=local)
    runners[big.name] = big
    left = budget - big.table_bytes()
    for name, share in (("ring48_d55_t177_k17", 0.8), ("ring32_d37_t79_k14", 0.2)):
        runners[name] = CircuitRunner(name, build_workload(name), key=args.seed + len(runners), max_samples=64,
                                      device=local, hbm_budget=left * share, graphs=args.graphs)
    for r in runners.values():  # every batch size captured before the arrivals start
        r.precapture(range(1, r.max_samples + 1))
    setup = time.perf_counter() - t0
    # warm every runner once
    from dcs245_classical_sampling_b200.serve import Request
    Server(runners).run([Request(10 ** 6 + i, c, 1, 0.0) for i, c in enumerate(runners)], realtime=False)
    reqs = poisson_requests(args.serve_rate, args.serve_seconds, mix, seed=args.seed,
                            max_samples=args.serve_max_samples)
    clocks = ClockSampler(local)
    clocks.start()
    ta = time.perf_counter()
    done = Server(runners).run(reqs, realtime=True)
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
    line = {"metric": "serving mix: samples/s and request p50/p99 ms (32q 2^14, 48q 2^17, 64q 2^20; 50/30/20)",
            "value": tot / span, "unit": "samples/s", "n_gpus": 1, "higher_is_better": True,
            "latency": latency_stats(done), "per_circuit": per, "requests": len(done), "samples": tot,
            "span_s": span, "arrival_window_s": args.serve_seconds, "rate_hz": args.serve_rate,
            "hbm_budget_gib": args.hbm_budget_gib,
            "slots": {c: {"samples_per_launch": r.max_samples, "table_items": r.engine.items,
                          "table_gib": r.table_bytes() / 2 ** 30, "mode": r.mode} for c, r in runners.items()},
            "ties": ties, "failed_draws": bad, "cuda_graphs": bool(args.graphs), "setup_s": setup, "clocks": clk,
            "data": "synthetic (seeded ring circuits, Philox4x32-10 prefixes and uniforms on the device)"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    elif args.serve:
        serve_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
