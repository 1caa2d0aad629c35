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
from make_golden import draw_checked, make_protocol  # noqa: E402
from conditional_block_gpu import ConditionalBlockGPU  # noqa: E402
from dcs_rankwidth import scan_kernel  # noqa: E402

from dcs245_classical_sampling_b200.workloads import build_workload  # noqa: E402
from oracle import block_ref  # noqa: E402
from oracle import c as oc  # noqa: E402

# workload: samples timed (the 16-qubit configuration's 256, a subset of the 40-qubit one's 1,000)
CASES = {"ring16_d20_t24_k8": 256, "ring40_d45_t190_k16": 8}


class NumbaEngine(ConditionalBlockGPU):
    """The reference engine with NumPy buffers and its Numba CPU step as the per-step kernel."""

    def alloc(self, dtype=np.complex128, device=0):
        cp = sys.modules["cupy"]
        self.cp = cp
        self.use_fp64 = True
        size = 1 << self.rmax
        self.d_buf = [np.zeros(size, np.complex128), np.zeros(size, np.complex128)]
        self.d_max = np.zeros(1, np.uint64)
        self.d_tables = [T.reshape(-1) for T in self.tables]
        self.d_combos = [np.asarray(c, np.uint64) for c in self.combos]
        self._grid = self._block = None
        self._kernel = self._numba_step
        # the syndrome map and open-edge phase of ConditionalBlockGPU.alloc (conditional_block_gpu.py:80-89)
        ids = np.arange(1 << self.terminal_rank, dtype=np.uint64)
        self.d_syndrome_map = np.zeros_like(ids)
        for j, b in enumerate(self.terminal_basis):
            self.d_syndrome_map ^= ((ids >> np.uint64(j)) & np.uint64(1)) * np.uint64(b)
        self.d_phase = np.ones(1 << len(self.open_full), np.float64)
        ids = np.arange(len(self.d_phase), dtype=np.uint64)
        for a, b in self.open_edges:
            self.d_phase *= 1 - 2 * (((ids >> np.uint64(a)) & (ids >> np.uint64(b)) & np.uint64(1)).astype(np.float64))

    def _numba_step(self, grid, block, args):
        (A, B, n_out, T, nbytes, combos, _ncombos, r_in, beta, ov, free, f0r, f0i, f1r, f1i, y, scale, d_max) = args
        n = int(n_out)
        scan_kernel._step(A, B, n, T.reshape(-1, 256), int(nbytes), combos, int(r_in), np.uint64(beta),
                          np.uint64(ov), int(free), complex(f0r, f0i), complex(f1r, f1i), int(y))
        scan_kernel._scale(B, n, float(scale))
        m = scan_kernel._maxabs(B, n)
        d_max[0] = np.array([m * m], np.float64).view(np.uint64)[0]


def main():
    import numba
    out = {"numba_threads": numba.get_num_threads(), "cpu_count": os.cpu_count(), "cases": {}}
    lib = oc.load()
    for name, count in CASES.items():
        w = build_workload(name)
        args = (w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"], w["open_vertices"])
        ref = NumbaEngine(*args)
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
