"""Time the REFERENCE's own CPU route of the hot path on this machine's cores, beside the
oracle's C/OpenMP executor (the CPU baseline that bench.py runs on GPU machines, where the
reference cannot run), on the same samples of the two small workloads.

The reference route: ``ConditionalBlockGPU`` (source/sampling/conditional_block_gpu.py:25-177)
unmodified, with its per-step kernel call (``_prefix``, :92-126) served by the reference's
Numba gather step ``scan_kernel._step`` (source/dcs_rankwidth/scan_kernel.py:26-51) plus its
``_scale`` and ``_maxabs`` (:54-65), complex128, then ``sampling_protocol.draw_checked``.  The
reference is imported unmodified (stubs and a NumPy-backed ``cupy`` as in make_golden.py);
Numba's cache goes to a temporary directory so that nothing is written into the reference.

    REFERENCE_ROOT=<checkout> python tests/golden/time_reference_cpu.py

Writes ``reference_cpu_timing.json`` next to this file: samples/s of both routes, the thread
count, and whether they drew the same indices.
"""
import json
import os
import sys
import tempfile
import time
from pathlib import Path

os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="numba_cache_"))

import numpy as np  # noqa: E402

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import make_golden  # noqa: E402,F401  (installs the reference: stubs, NumPy-backed cupy, sys.path)
from make_golden import GatherEngine, draw_checked, make_protocol  # noqa: E402

from dcs245_classical_sampling_b200.workloads import build_workload  # noqa: E402
from oracle import block_ref  # noqa: E402
from oracle import c as oc  # noqa: E402

# workload: samples timed (the 16-qubit configuration's 256, a subset of the 40-qubit one's 1,000)
CASES = {"ring16_d20_t24_k8": 256, "ring40_d45_t190_k16": 8}


def main():
    import numba
    out = {"numba_threads": numba.get_num_threads(), "cpu_count": os.cpu_count(), "cases": {}}
    lib = oc.load()
    for name, count in CASES.items():
        w = build_workload(name)
        args = (w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"], w["open_vertices"])
        ref = GatherEngine(*args)
        ref.alloc()
        recs = make_protocol(24520, count, w["n"], w["open_vertices"])["records"]
        xs = [np.array([int(c) for c in r["input_data_bits"]], np.uint8) for r in recs]
        us = [r["draw_uniform"] for r in recs]
        v, _ = ref.block(xs[0])  # Numba compilation outside the timing
        draw_checked(np.asarray(v), us[0])
        t0 = time.perf_counter()
        ri = [draw_checked(np.asarray(ref.block(x)[0]), u)["A_index"] for x, u in zip(xs, us)]
        t_ref = time.perf_counter() - t0
        cs = oc.CpuSampler(block_ref.OracleEngine(*args), lib)
        cs.sample(xs[0], us[0])
        t0 = time.perf_counter()
        pi = [cs.sample(x, u)["A_index"] for x, u in zip(xs, us)]
        t_port = time.perf_counter() - t0
        out["cases"][name] = {"samples": count, "reference_numba_samples_per_s": count / t_ref,
                              "port_c_openmp_samples_per_s": count / t_port, "port_over_reference": t_ref / t_port,
                              "port_threads": int(lib.oracle_threads()), "same_indices": ri == pi,
                              "gather_rmax": int(ref.rmax)}
        print(name, out["cases"][name], flush=True)
    (HERE / "reference_cpu_timing.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
