"""Generate the golden fixtures under tests/golden/ by running the REFERENCE itself.

Run in a container that has the reference checkout (read-only); its location is
given by the environment variable REFERENCE_ROOT (required).  The GPU machines do
not have it, which is why the outputs are committed.  The reference is imported unmodified:

* ``qiskit`` and ``stim`` are stubbed (they are used only by circuit
  preparation, which the fixtures replace with this project's seeded ring
  circuits from ``dcs245_classical_sampling_b200.circuits``);
* ``cupy`` is a NumPy-backed module (the same trick the reference uses in
  ``source/production/make_synthetic_worker_fixture.py:53-59``);
* the engine is ``InplaceConditionalBlockGPU`` (``sampling/conditional_block_inplace_gpu.py``)
  with ``alloc`` rebuilt on NumPy and ``_prefix`` routed to the reference's exact
  complex128 executor ``kernel_opt/inplace_plan.py:execute_inplace``; the slice
  loop, syndrome scatter and Walsh-Hadamard tail are the reference's own
  ``ConditionalBlockGPU.block`` (``sampling/conditional_block_gpu.py:128-177``).

Outputs: ``<case>.json`` (inputs, reference plan, draws, meta) and
``<case>.npz`` (graph, unitaries, reference blocks).

    REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py [--cases c1 small c2 c64plan ...]
"""
import argparse
import json
import math
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
if not os.environ.get("REFERENCE_ROOT"):
    raise SystemExit("set REFERENCE_ROOT to the reference checkout")
REF = Path(os.environ["REFERENCE_ROOT"]) / "source"
# write nothing into the reference checkout: no bytecode, and Numba's cache (its kernels are
# declared with cache=True) in a temporary directory
sys.dont_write_bytecode = True
os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="numba_cache_"))


def install_reference():
    for name in ("qiskit", "stim"):
        mod = types.ModuleType(name)
        mod.QuantumCircuit = object
        mod.transpile = lambda *a, **k: None
        sys.modules.setdefault(name, mod)
    cp = types.ModuleType("cupy")
    for attr in ("zeros", "ones", "arange", "zeros_like", "empty", "uint64", "uint32",
                 "complex128", "complex64", "float64", "asarray"):
        setattr(cp, attr, getattr(np, attr))
    cp.asnumpy = np.asarray
    cuda = types.ModuleType("cupy.cuda")
    cuda.get_current_stream = lambda: types.SimpleNamespace(synchronize=lambda: None)
    cp.cuda = cuda
    sys.modules["cupy"] = cp
    sys.modules["cupy.cuda"] = cuda
    for sub in ("", "sampling", "kernel_opt", "review", "production"):
        p = str(REF / sub) if sub else str(REF)
        if p not in sys.path:
            sys.path.insert(0, p)
    sys.path.insert(0, str(REPO))


install_reference()
from conditional_block_inplace_gpu import InplaceConditionalBlockGPU  # noqa: E402
from inplace_plan import compile_inplace, execute_inplace  # noqa: E402
from sampling_protocol import draw_checked, make_protocol, assemble_output  # noqa: E402
from protocol_common import actual_cdf_law_vector, make_run_protocol  # noqa: E402
from full_vector_audit_certificate import audit_vector_pair  # noqa: E402
from dcs_rankwidth.parity_slicing import choose_parity_slices, prefix_ranks_matrix  # noqa: E402
from dcs_rankwidth import scan_plan  # noqa: E402

from dcs245_classical_sampling_b200.circuits import build_ring_instance  # noqa: E402
from dcs245_classical_sampling_b200.workloads import build_workload  # noqa: E402


class OracleEngine(InplaceConditionalBlockGPU):
    """Reference engine with NumPy storage and the exact complex128 executor."""

    def alloc(self, dtype=np.complex128, device=0):
        self.cp = sys.modules["cupy"]
        self.inplace_fp64 = True
        self.use_fp64 = True
        stop = len(self.steps)
        self.inplace_steps, self.inplace_terminal_basis, self.inplace_maxslots = compile_inplace(
            self.order, self.fut, self.fixed, stop)
        self.inplace_rmax = max([0] + [len(s.active_out) for s in self.inplace_steps])
        self.terminal_basis = [b >> self.stop for _, b in sorted(self.inplace_terminal_basis.items())]
        self.terminal_rank = len(self.terminal_basis)
        ids = np.arange(1 << self.terminal_rank, dtype=np.uint64)
        self.d_syndrome_map = np.zeros_like(ids)
        for j, b in enumerate(self.terminal_basis):
            self.d_syndrome_map ^= ((ids >> np.uint64(j)) & np.uint64(1)) * np.uint64(b)
        self.d_phase = np.ones(1 << len(self.open_full), np.float64)
        ids = np.arange(len(self.d_phase), dtype=np.uint64)
        for a, b in self.open_edges:
            self.d_phase *= 1 - 2 * (((ids >> np.uint64(a)) & (ids >> np.uint64(b)) & np.uint64(1)).astype(np.float64))

    def _prefix(self, f, yfix):
        env, ls, offset, _ = execute_inplace(self.inplace_steps, f, yfix, self.fut, self.inplace_maxslots)
        if not np.any(env):
            return None, ls, offset >> self.stop
        return env, ls, offset >> self.stop


class GatherEngine:
    """The reference's gather engine (sampling/conditional_block_gpu.py:25-177), unmodified, with
    NumPy buffers and its per-step kernel served by the reference's Numba gather step
    (dcs_rankwidth/scan_kernel.py:26-65); complex128."""

    def __new__(cls, *args):
        from conditional_block_gpu import ConditionalBlockGPU
        from dcs_rankwidth import scan_kernel

        class _Engine(ConditionalBlockGPU):
            def alloc(self, dtype=np.complex128, device=0):
                self.cp = sys.modules["cupy"]
                self.use_fp64 = True
                size = 1 << self.rmax
                self.d_buf = [np.zeros(size, np.complex128), np.zeros(size, np.complex128)]
                self.d_max = np.zeros(1, np.uint64)
                self.d_tables = [T.reshape(-1) for T in self.tables]
                self.d_combos = [np.asarray(c, np.uint64) for c in self.combos]
                self._grid = self._block = None
                self._kernel = self._numba_step
                ids = np.arange(1 << self.terminal_rank, dtype=np.uint64)
                self.d_syndrome_map = np.zeros_like(ids)
                for j, b in enumerate(self.terminal_basis):
                    self.d_syndrome_map ^= ((ids >> np.uint64(j)) & np.uint64(1)) * np.uint64(b)
                self.d_phase = np.ones(1 << len(self.open_full), np.float64)
                ids = np.arange(len(self.d_phase), dtype=np.uint64)
                for a, b in self.open_edges:
                    self.d_phase *= 1 - 2 * (((ids >> np.uint64(a)) & (ids >> np.uint64(b))
                                              & np.uint64(1)).astype(np.float64))

            def _numba_step(self, grid, block, args):
                (A, B, n_out, T, nbytes, combos, _nc, r_in, beta, ov, free, f0r, f0i, f1r, f1i, y, scale,
                 d_max) = args
                n = int(n_out)
                scan_kernel._step(A, B, n, T.reshape(-1, 256), int(nbytes), combos, int(r_in), np.uint64(beta),
                                  np.uint64(ov), int(free), complex(f0r, f0i), complex(f1r, f1i), int(y))
                scan_kernel._scale(B, n, float(scale))
                m = scan_kernel._maxabs(B, n)
                d_max[0] = np.array([m * m], np.float64).view(np.uint64)[0]

        return _Engine(*args)


def gather_case(name):
    """The reference gather engine's plan and blocks for a golden case's prefixes, beside the in-place
    engine's blocks of the same case (both are exact contractions of the same block)."""
    case = json.loads((HERE / f"{name}.json").read_text())
    arrays = dict(np.load(HERE / f"{name}.npz"))
    eng = GatherEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                       [tuple(op) for op in case["parity_operations"]], case["open_vertices"])
    out = {"name": name, "rmax": int(eng.rmax), "work": int(eng.work), "stop": int(eng.stop),
           "terminal_basis": [int(b) for b in eng.terminal_basis],
           "rank_profile": [int(r) for r in eng.rank_profile],
           "steps": [{"v": int(st.v), "free": bool(st.free), "r_in": int(st.r_in), "r_out": int(st.r_out),
                      "beta": int(st.beta), "Lcols": [int(c) for c in st.Lcols], "kernel": [int(k) for k in st.kernel]}
                     for st in eng.steps], "blocks_rel_l2_vs_inplace": []}
    eng.alloc()
    for rec in case["protocol"]["records"]:
        x = np.array([int(c) for c in rec["input_data_bits"]], np.uint8)
        v, meta = eng.block(x)
        want = arrays[f"block_{rec['sample_id']}"]
        out["blocks_rel_l2_vs_inplace"].append(float(np.linalg.norm(np.asarray(v) - want) / np.linalg.norm(want)))
    return out


def plan_json(engine):
    steps = []
    for st in engine.inplace_steps:
        steps.append({"v": st.v, "j": st.j, "kind": st.kind, "active_in": list(st.active_in),
                      "active_out": list(st.active_out), "beta": st.beta, "K": st.K, "Ka": st.Ka,
                      "pivot": st.pivot, "pivot_a": st.pivot_a, "free": bool(st.free)})
    return {"steps": steps, "terminal_basis": [int(b) for b in engine.terminal_basis],
            "terminal_slots": sorted(int(p) for p in engine.inplace_terminal_basis),
            "maxslots": engine.inplace_maxslots, "inplace_rmax": engine.inplace_rmax,
            "stop": engine.stop, "rmax": engine.rmax, "work": engine.work,
            "open_edges": [list(map(int, e)) for e in engine.open_edges],
            "order": list(map(int, engine.order)), "fixed": sorted(map(int, engine.fixed)),
            "fut": [int(x) for x in engine.fut], "slices": list(map(int, engine.slices))}


def jsonable(d):
    out = {}
    for k, v in d.items():
        if isinstance(v, (np.integer,)):
            v = int(v)
        elif isinstance(v, (np.floating,)):
            v = float(v)
        out[k] = v
    return out


def make_case(name, workload, n_prefixes, n_uniforms, blocks=True, proto_seed=None, store_blocks=True):
    """store_blocks=False keeps the reference's draws and a per-block summary (mass, selected
    weight, weights hash) but not the blocks themselves (large blocks, many prefixes)."""
    w = build_workload(workload)
    n, openv, order, ops = w["n"], w["open_vertices"], w["order"], w["parity_operations"]
    A = w["graph"]
    N = len(A)
    inst = w
    case = {"name": name, "workload": workload, "n": n, "depth": w["depth"], "t_count": w["t_count"],
            "seed": w["seed"],
            "open_vertices": openv, "order": list(map(int, order)),
            "parity_operations": [[a, b, c] for a, b, c in ops], "N": N}
    t0 = __import__("time").time()
    eng = OracleEngine(A, inst["unitaries"], n, order, ops, openv)
    eng.alloc()
    case["plan"] = plan_json(eng)
    case["prefix_cut_ranks_order"] = [int(x) for x in prefix_ranks_matrix(A.copy(), list(order))]
    proto = make_protocol(proto_seed if proto_seed is not None else 1000 + w["seed"], n_prefixes, n, openv)
    case["protocol"] = {"seed": proto["seed"], "records": [
        {"sample_id": r["sample_id"], "input_data_bits": r["input_data_bits"],
         "draw_uniform": r["draw_uniform"], "branch_uniform": r["branch_uniform"]}
        for r in proto["records"]]}
    arrays = {"graph": A, "unitaries": inst["unitaries"], "order": np.asarray(order)}
    draws = []
    if blocks:
        rng = np.random.default_rng(7)
        for r in proto["records"]:
            x = np.asarray(list(map(int, r["input_data_bits"])), np.uint8)
            v, meta = eng.block(x)
            v = np.asarray(v)
            if store_blocks:
                arrays[f"block_{r['sample_id']}"] = v
            us = [r["draw_uniform"]] + [float(u) for u in rng.random(n_uniforms - 1)]
            for u in us:
                d = draw_checked(v, u)
                bits, qiskit = assemble_output(r["input_data_bits"], openv, d["A_index"], inst["ring"])
                d = jsonable(d)
                d["sample_id"] = r["sample_id"]
                d["data_bits_ring_order"] = bits
                d["bitstring_qiskit"] = qiskit
                draws.append(d)
            meta = {k2: v2 for k2, v2 in meta.items() if k2 != "seconds"}
            case.setdefault("block_meta", []).append(jsonable(meta))
        case["draws"] = draws
    case["seconds"] = __import__("time").time() - t0
    return case, arrays


def sampler_cases():
    """Known-answer cases of the reference sampler and audit helpers on fixed vectors."""
    out = {"selftest": [], "law": [], "audit": []}
    for weights in [np.array([0., 1., 0., 2., 3., 0., 4., 0.]),
                    np.array([1e-100, 1., .5, 0., 7., 2e-100, 1., .1])]:
        v = np.sqrt(weights) * np.exp(1j * np.arange(len(weights)))
        cdf = np.cumsum(weights) / np.sum(weights)
        for idx in np.flatnonzero(weights):
            lo = cdf[idx - 1] if idx else 0.
            if cdf[idx] == lo:
                continue
            u = (lo + cdf[idx]) / 2
            d = draw_checked(v, u)
            out["selftest"].append({"re": v.real.tolist(), "im": v.imag.tolist(), "u": u,
                                    "draw": jsonable({k: d[k] for k in d if k != "replay_scope"})})
    for a in [np.array([0, 1, 1j, 1 + 1j, 0, 2, 1 - 1j, 0], complex),
              np.array([1e-15, 1e-8j, 1, 1j, 2 + 3j, .17, .21j, .01], complex)]:
        law, meta = actual_cdf_law_vector(a)
        d = draw_checked(a, .381245)
        out["law"].append({"re": a.real.tolist(), "im": a.imag.tolist(), "law_re": law.real.tolist(),
                           "law_im": law.imag.tolist(), "meta": jsonable(meta), "A_index": d["A_index"]})
    rng = np.random.default_rng(3)
    for _ in range(3):
        ref = rng.normal(size=16) + 1j * rng.normal(size=16)
        approx = (ref + 1e-3 * (rng.normal(size=16) + 1j * rng.normal(size=16))).astype(np.complex64)
        approx = approx.astype(np.complex128)
        out["audit"].append({"ref_re": ref.real.tolist(), "ref_im": ref.imag.tolist(),
                             "ap_re": approx.real.tolist(), "ap_im": approx.imag.tolist(),
                             "result": jsonable(audit_vector_pair(ref, approx, 0))})
    proto = make_protocol(733245, 113, 6, [5, 1, 3], .45)
    out["protocol_733245"] = [{"sample_id": r["sample_id"], "conditional_branch": r["conditional_branch"],
                               "branch_uniform": r["branch_uniform"], "draw_uniform": r["draw_uniform"],
                               "input_data_bits": r["input_data_bits"]} for r in proto["records"]]
    out["assemble"] = [list(assemble_output("000000", [5, 1, 3], i, [5, 0, 4, 1, 3, 2])) for i in range(8)]
    # a 64-qubit record with 20 free bits and a non-identity ring (a seeded permutation standing
    # in for a device's ring order), several indices
    p64 = make_protocol(24520, 3, 64, list(range(44, 64)))
    ring64 = [int(q) for q in np.random.default_rng(64).permutation(64)]
    out["assemble64"] = {"ring": ring64, "free": list(range(44, 64)), "cases": [
        {"input_data_bits": r["input_data_bits"], "A_index": int(a),
         "out": list(assemble_output(r["input_data_bits"], list(range(44, 64)), int(a), ring64))}
        for r in p64["records"] for a in (0, 1, 123456, (1 << 20) - 1)]}
    # the generation protocol records themselves (config-3 seeds, 64 qubits, 20 free bits)
    out["protocol64"] = [{k: r[k] for k in ("sample_id", "conditional_branch", "branch_uniform", "draw_uniform",
                                            "input_data_bits")} for r in p64["records"]]
    # audit ids chosen before generation (production/protocol_common.py:22-31): the reference's
    # own make_run_protocol on a small two-worker case and on the 2048-sample, 64-audit case
    audit = []
    for seed, aseed, count, workers, per, n_, free_ in ((7324501, 7324502, 24, 2, 2, 6, [5, 1, 3]),
                                                       (24520, 24521, 2048, 1, 64, 64, list(range(44, 64)))):
        rp = make_run_protocol(seed, aseed, count, workers, per, n_, free_, "fp32")
        audit.append({"seed": seed, "audit_seed": aseed, "count": count, "workers": workers, "per_worker": per,
                      "n": n_, "free": free_, "ids_by_worker": rp["audit"]["ids_by_worker"],
                      "ids": rp["audit"]["ids"]})
    out["audit_ids"] = audit
    return out


def chooser_case():
    """Reference parity-slice chooser and cut ranks on a small synthetic graph (unfiltered)."""
    inst = build_ring_instance(12, 10, 14, 77)
    A = inst["graph"]
    N = len(A)
    edges = [(int(a), int(b)) for a, b in zip(*np.nonzero(np.triu(A, 1)))]
    order = list(map(int, inst["natural_order"]))
    ops, S = choose_parity_slices(N, edges, order, 3, seed=0, verbose=False)
    return {"n": 12, "depth": 10, "t_count": 14, "seed": 77, "order": order,
            "ops": [[a, b, c] for a, b, c in ops], "removed": S,
            "cut_ranks": [int(x) for x in prefix_ranks_matrix(A.copy(), order)]}


CASES = {
    # 16-qubit ring, depth 20, 24 T, 8 open bits (the small CPU-runnable workload)
    "c1": dict(workload="ring16_d20_t24_k8", n_prefixes=4, n_uniforms=4),
    # a mid-size ring with two parity slices
    "small": dict(workload="ring24_d24_t60_k10", n_prefixes=3, n_uniforms=3),
    # 40-qubit ring, depth 45, 190 T, 16 open bits (one prefix; ~2^22 tables)
    "c2": dict(workload="ring40_d45_t190_k16", n_prefixes=1, n_uniforms=4),
    # all 256 samples of the 16-qubit workload (same protocol seed as c1: records 0-3 are c1's),
    # one draw per sample with its own protocol uniform
    "c1full": dict(workload="ring16_d20_t24_k8", n_prefixes=256, n_uniforms=1),
    # 8 prefixes of the 40-qubit workload (record 0 is c2's); draws only, blocks not stored
    "c2draws": dict(workload="ring40_d45_t190_k16", n_prefixes=8, n_uniforms=2, store_blocks=False),
    # plan only: 64-qubit ring, depth 73, 314 T, 20 open bits, two parity slices
    "c64plan": dict(workload="ring64_d73_t314_k20", n_prefixes=2, n_uniforms=0, blocks=False),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", nargs="*", default=list(CASES) + ["sampler", "chooser", "gather"])
    args = ap.parse_args()
    for name in args.cases:
        if name == "sampler":
            (HERE / "sampler.json").write_text(json.dumps(sampler_cases(), indent=1))
            continue
        if name == "chooser":
            (HERE / "chooser.json").write_text(json.dumps(chooser_case(), indent=1))
            continue
        if name == "gather":
            g = {c: gather_case(c) for c in ("c1", "small", "c2")}
            (HERE / "gather.json").write_text(json.dumps(g, indent=1))
            print("gather", {c: max(v["blocks_rel_l2_vs_inplace"]) for c, v in g.items()}, flush=True)
            continue
        case, arrays = make_case(name, **CASES[name])
        (HERE / f"{name}.json").write_text(json.dumps(case, indent=1))
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        print(name, "N", case["N"], "rmax", case["plan"]["inplace_rmax"], "ops", case["parity_operations"],
              "%.1fs" % case["seconds"], flush=True)


if __name__ == "__main__":
    main()
