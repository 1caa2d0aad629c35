"""Autotuner for the fused executor's tile shape.

For a plan, each candidate (max tile dimension, contiguous low bits, max steps per group)
gives a different grouping of the vertex steps (``fused.group_steps``).  The tuner times one
slice contraction per candidate with CUDA events on the engine's own table and keeps the
fastest; results are cached per plan fingerprint in ``autotune_cache.json`` next to this file.
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

from . import _lib

CACHE = Path(__file__).resolve().parent / "autotune_cache.json"
# (max tile dim, contiguous low bits, max steps per group, kernel variant, step pairs); variant
# bit 0 = two CTAs per SM, bit 1 = paired tile layout with packed FP32x2 arithmetic, bit 2 =
# register runs (bit 3: of local dimension 4, else 3)
CANDIDATES = [(13, 3, 24, 0, True), (13, 3, 24, 12, False), (13, 4, 24, 12, False), (13, 3, 24, 6, False),
              (13, 4, 24, 6, False), (13, 3, 24, 7, False), (13, 3, 24, 15, False), (13, 5, 24, 6, False),
              (12, 3, 24, 6, False), (13, 3, 12, 6, False)]


def fingerprint(plan):
    h = hashlib.sha256()
    for st in plan.steps:
        h.update(repr((st.kind, st.active_in, st.active_out, st.beta, st.K, st.Ka, st.pivot, st.pivot_a)).encode())
    return h.hexdigest()[:20]


def _load():
    if CACHE.exists():
        try:
            return json.loads(CACHE.read_text())
        except ValueError:
            return {}
    return {}


def cached(plan, device_name):
    return _load().get(f"{fingerprint(plan)}|{device_name}")


# with plan-specialised group kernels (jit.py; scalar register runs, so no packed variants)
# (pairs=True with register runs: two cosets per loop iteration in the generated kernels)
# variant bit 1 with register runs: packed FP32x2 groups where tile bit 0 stays free
JIT_CANDIDATES = [(13, 3, 24, 12, False, None, 256, "bytes"), (13, 4, 24, 12, False, None, 256, "bytes"),
                  (13, 2, 24, 12, False, None, 256, "bytes"), (13, 3, 24, 4, False, None, 256, "bytes"),
                  (13, 4, 24, 12, False), (13, 3, 24, 12, False), (13, 4, 24, 4, False), (13, 4, 24, 4, True),
                  (13, 4, 24, 6, False), (13, 4, 24, 14, False), (13, 4, 24, 15, False)]


KEYS = ("max_dim", "low", "max_steps", "variant", "pairs", "minb", "threads", "grouping", "group_cost", "max_extra",
        "prefetch_kb")
PLAN_KEYS = ("max_dim", "low", "max_steps", "variant", "pairs", "grouping", "group_cost", "max_extra", "prefetch_kb")
DEFAULTS = {"minb": None, "threads": 256, "grouping": "greedy", "group_cost": 1 << 30, "max_extra": 1,
            "prefetch_kb": 0}


def candidate(c):
    """A candidate as a dict of KEYS: a dict, or a tuple in KEYS order (missing tail = defaults)."""
    d = dict(c) if isinstance(c, dict) else dict(zip(KEYS, c))
    return {**DEFAULTS, **d}


def tune(engine, params_dev, candidates=None, repeats=1, save=True, jit=False):
    """Time each candidate on the engine (mode "fused", already allocated) and install the best.

    params_dev: device params of one work item (nsteps dcs_param).  jit: time the candidates
    as plan-specialised group kernels.  Returns the report."""
    if candidates is None:
        candidates = JIT_CANDIDATES if jit else CANDIDATES
    import torch
    from .fused import build_fused_plan
    lib = engine.lib
    stream = torch.cuda.current_stream(engine.device)
    report = []
    best = None
    for cand in map(candidate, candidates):
        try:
            fp = build_fused_plan(engine.plan, **{k: cand[k] for k in PLAN_KEYS})
        except ValueError:
            continue
        if jit and fp.tile_runs is not None:
            from .jit import JitPlan
            fp.jit = JitPlan(engine.plan, fp, lib, minb=cand["minb"], threads=cand["threads"])
            cand = {**cand, "minb": fp.jit.minb}
        need = len(fp.groups) + 1
        if engine.maxbits.numel() < need:
            engine.maxbits = torch.zeros(need, dtype=torch.int64, device=engine.device)
        times = []
        for _ in range(repeats + 1):
            mb = engine.maxbits
            mb.zero_()
            mb[0] = engine.one_bits
            engine.scale.zero_()
            engine.table.view(engine.items, engine.table_stride)[:1, 0] = 1
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib.check(fp.launch(lib, _lib.ptr(engine.table), _lib.ptr(params_dev), 0, len(fp.groups), _lib.ptr(mb),
                                 _lib.ptr(engine.scale), stream.cuda_stream))
            b.record(stream)
            torch.cuda.synchronize(engine.device)
            times.append(a.elapsed_time(b) / 1000.0)
        t = min(times[1:]) if len(times) > 1 else times[0]
        report.append({**cand, "jit": fp.jit is not None, "groups": len(fp.groups), "seconds": t})
        if best is None or t < best[0]:
            if best is not None and best[2].jit is not None:
                best[2].jit.close()
            best = (t, cand, fp)
        elif fp.jit is not None:
            fp.jit.close()
    engine.fplan = best[2]
    nm = len(best[2].groups) + 1
    engine.maxbits = torch.zeros(engine.items * nm, dtype=torch.int64, device=engine.device)
    chosen = {**{k: best[1][k] for k in PLAN_KEYS}, "jit": best[2].jit is not None,
              "minb": best[1]["minb"] if best[2].jit is not None else None,
              "threads": best[1]["threads"] if best[2].jit is not None else None, "seconds": best[0]}
    if save:
        data = _load()
        data[f"{fingerprint(engine.plan)}|{torch.cuda.get_device_name(engine.device)}"] = chosen
        try:
            CACHE.write_text(json.dumps(data, indent=1) + "\n")
        except OSError:
            pass
    return {"best": chosen, "candidates": report}


# per-group kernel choices: (CTAs per SM the registers are sized for, KiB staging the next
# tile's first-run entries (jit.prefetch_layout), local dimension of the register runs).  A third
# entry "4p" selects dimension 4 in the packed FP32x2 form where the group's runs leave tile bit 0
# free; on the 64-qubit plan it was slower on every large group (22: 8.1 against 6.0 ms, 24: 27.2
# against 24.4 ms) and its FP32x2 instructions can round differently from the scalar form, so it
# is not among the defaults.  An optional fourth entry is the CTA size (default: the plan's, 256):
# 128 threads at 3 CTAs per SM hold three tiles per SM instead of two (registers for dimension-5
# runs still fit: 3 x 128 x 128 <= 65536), each thread taking two cosets of the 256-coset runs.
# "4t" / "5t": dimension 4 / 5 with run bases that may touch other roles (variant bit 6: fewer
# register runs, so fewer shared-memory round trips per tile).
GROUP_CANDIDATES = ((3, 0, 4), (3, 8, 4), (2, 0, 4), (2, 16, 4), (2, 32, 4), (2, 0, 5), (2, 16, 5), (2, 32, 5),
                    (3, 0, 4, 128), (3, 0, 5, 128), (3, 8, 5, 128),
                    (3, 8, "4t"), (2, 32, "4t"), (2, 16, "5t"), (2, 32, "5t"), (3, 8, "5t", 128))


def _time_groups(engine, fp, jp, params_dev, repeats):
    """Per-group CUDA-event times (min over repeats) of one slice with the kernels of `jp`."""
    import torch
    lib = engine.lib
    stream = torch.cuda.current_stream(engine.device)
    ng = len(fp.groups)
    best = [float("inf")] * ng
    for _ in range(repeats + 1):
        mb = engine.maxbits
        mb.zero_()
        mb[0] = engine.one_bits
        engine.scale.zero_()
        engine.table.view(engine.items, engine.table_stride)[:1, 0] = 1
        evs = []
        for gi in range(ng):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib.check(jp.launch(_lib.ptr(engine.table), _lib.ptr(params_dev), gi, 1, _lib.ptr(mb),
                                 _lib.ptr(engine.scale), stream.cuda_stream))
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize(engine.device)
        for gi, (a, b) in enumerate(evs):
            best[gi] = min(best[gi], a.elapsed_time(b) / 1000.0)
    return best


def tune_groups(engine, params_dev, candidates=GROUP_CANDIDATES, repeats=2, save=True):
    """Choose, per group of the engine's fused plan (plan-specialised kernels), the kernel variant
    of `candidates` (CTAs per SM, staging KiB, register-run dimension 4 or 5, optionally threads
    per CTA) with the shortest
    launch, timed with CUDA events on the engine's own table; install the mix and return the
    report.  Every variant computes the same values bit for bit (the same operations in the same
    order on each entry), so groups can mix them."""
    import torch
    from .fused import build_fused_plan
    from .jit import JitPlan
    if engine.fplan.jit is None:
        raise ValueError("tune_groups needs the plan-specialised kernels (jit)")
    lib = engine.lib
    threads = engine.fplan.jit.threads
    from .jit import packable
    base = {k: v for k, v in engine.fused_config.items() if k != "group_variant"}
    v4 = (int(base["variant"]) & ~82) | 12
    variants = {4: v4, 5: v4 | 16, "4p": v4 | 2, "4t": v4 | 64, "5t": v4 | 80}
    plans = {r: build_fused_plan(engine.plan, **{**base, "variant": v}) for r, v in variants.items()
             if any(c[2] == r for c in candidates)}
    ng = len(plans[4].groups)
    times = {}
    for cand in candidates:
        minb, kb, r = int(cand[0]), int(cand[1]), cand[2]
        nt = int(cand[3]) if len(cand) > 3 else threads
        fp = plans[r]
        jp = JitPlan(engine.plan, fp, lib, minb=minb, threads=threads,
                     group_cfg={gi: (minb, kb, nt) for gi in range(ng)})
        t = _time_groups(engine, fp, jp, params_dev, repeats)
        jp.close()
        for gi in range(ng):  # a group that fell back to the dimension-4 scalar kernel is timed there
            if (r in (5, "5t") and not int(fp.groups[gi]["variant"]) & 16) or (r == "4p" and not packable(fp, gi)):
                t[gi] = float("inf")
        times[(minb, kb, r, nt)] = t
    choice = {gi: min(times, key=lambda c: times[c][gi]) for gi in range(ng)}
    group_variant = {gi: variants[c[2]] for gi, c in choice.items() if c[2] != 4}
    group_cfg = {gi: (c[0], c[1]) if c[3] == threads else (c[0], c[1], c[3]) for gi, c in choice.items()}
    engine.fplan.jit.close()
    engine.fused_config = {**base, "group_variant": group_variant}
    engine.jit_group_cfg = group_cfg
    engine.fplan = engine._build_fplan()
    total = sum(_time_groups(engine, engine.fplan, engine.fplan.jit, params_dev, repeats))
    report = {"group_cfg": {str(g): list(c) for g, c in group_cfg.items()},
              "group_variant": {str(g): v for g, v in group_variant.items()}, "seconds": total,
              "per_candidate_seconds": {"/".join(map(str, c)): sum(x for x in t if x != float("inf"))
                                        for c, t in times.items()},
              "per_group_ms": {str(g): {"/".join(map(str, c)): round(times[c][g] * 1e3, 4) for c in times
                                        if times[c][g] != float("inf")} for g in range(ng)}}
    if save:
        key = f"{fingerprint(engine.plan)}|{torch.cuda.get_device_name(engine.device)}"
        data = _load()
        entry = dict(data.get(key) or {})
        if entry and all(entry.get(k) == base.get(k) for k in PLAN_KEYS if k in entry):
            entry["group_cfg"] = report["group_cfg"]
            entry["group_variant"] = report["group_variant"]
            entry["seconds"] = round(total, 4)
            data[key] = entry
            try:
                CACHE.write_text(json.dumps(data, indent=1) + "\n")
            except OSError:
                pass
    return report
