"""Small, self-contained profiling case for the contraction kernels.

Runs the first vertex steps of a workload's plan whose table stays within 2^max_slots
entries (default 2^28 complex64 = 2 GiB: larger than L2, small enough for a full ncu
capture), for one prefix and one slice, `iters` times, with either the fused kernel or the
per-step kernel.  Prints one JSON line with the per-launch CUDA-event timings.

    python -m dcs245_classical_sampling_b200.profile_case [--mode fused|device] [--max-slots 28]
        [--storage float16]
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main():
    import torch

    from . import _lib
    from . import plan as P
    from .engine import SliceParams, device_steps
    from .fused import build_fused_plan
    from .sampling import make_protocol
    from .workloads import build_workload

    ap = argparse.ArgumentParser()
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
    ap.add_argument("--storage", default=None, choices=["float16"],
                    help="binary16 tables with FP64 arithmetic (device mode)")
    a = ap.parse_args()
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
    entry = 4 if half else 8
    if half:
        table = torch.empty(2 << a.max_slots, dtype=torch.float16, device=dev)
    else:
        table = torch.empty(1 << a.max_slots, dtype=torch.complex64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sub = P.BlockPlan(**{**bp.__dict__, "steps": steps})
    if a.mode == "fused":
        fp = build_fused_plan(sub, max_dim=a.max_dim, low=a.low, variant=a.variant, pairs=a.pairs,
                              grouping=a.grouping)
        if a.jit:
            from .jit import JitPlan
            fp.jit = JitPlan(sub, fp, lib)
        nmax = len(fp.groups)
    else:
        dsteps = device_steps(steps)
        nmax = last
    maxbits = torch.zeros(nmax + 1, dtype=torch.int64, device=dev)
    scale = torch.zeros(_lib.SCALE_DTYPE.itemsize // 8, dtype=torch.int64, device=dev)
    one = (int(np.array([1.0], np.float64).view(np.int64)[0]) if half
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
                alg = ((1 << len(steps[first].active_in)) + (1 << len(steps[first + count - 1].active_out))) * 8
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
    print(json.dumps({"mode": a.mode, "storage": a.storage or "complex64", "steps": last, "launches": len(per_launch), "total_ms": tot_ms,
                      "alg_gb": tot_b / 1e9, "alg_gbs": tot_b / tot_ms / 1e6,
                      "big_launch_gbs": (sum(b for _, b in big) / sum(t for t, _ in big) / 1e6) if big else None,
                      "per_launch_ms": [round(t, 3) for t, _ in per_launch]}))


if __name__ == "__main__":
    main()
