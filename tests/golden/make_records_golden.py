"""Golden fixture for the production record rows, checked by the REFERENCE's own verifier.

Run in a container that has the reference checkout (read-only); the environment variable
REFERENCE_ROOT (required) gives its location.  It

1. makes a synthetic production protocol for the 16-qubit ring case ``c1`` with the reference's
   ``make_run_protocol`` (source/production/protocol_common.py:18-45): 8 samples, one worker,
   2 preselected audits;
2. builds every sample row and audit row with this project's ``records`` module from exact
   blocks of the oracle (complex128 as the audit reference; the same blocks rounded to complex64
   as the sampled vectors) and the reference's own ``draw_checked`` and ``audit_vector_pair``;
3. writes them with the worker's other artifacts into a synthetic bundle (the worker's
   control-plane files are written here, by this script, only so that the verifier can run);
4. runs the reference's ``verify_run(bundle, artifacts, ledger, synthetic=True)``
   (source/production/verify.py:351-618) and records its verdict and failures.

Outputs ``records.json`` (the protocol, the rows without their timing fields, the verdict) and
``records.npz`` (the sampled and reference vectors).

    REFERENCE_ROOT=<checkout> python tests/golden/make_records_golden.py
    REFERENCE_ROOT=<checkout> python tests/golden/make_records_golden.py --verify-artifacts DIR [--engine half]

With ``--verify-artifacts``, DIR holds samples.jsonl, audits.jsonl and the vectors that
``records.write_rows`` wrote for the same protocol on a GPU; the script completes the
control-plane files around them and prints the reference verifier's verdict.
"""
import argparse
import hashlib
import json
import shutil
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import make_golden  # noqa: E402  (installs the reference: stubs, NumPy-backed cupy, sys.path)
from make_golden import audit_vector_pair, draw_checked  # noqa: E402
from protocol_common import make_run_protocol  # noqa: E402
import verify as ref_verify  # noqa: E402

from dcs245_classical_sampling_b200 import records  # noqa: E402
from oracle import block_ref  # noqa: E402

CASE = "c1"
SEED, AUDIT_SEED, COUNT, WORKERS, AUDITS = 245101, 245102, 8, 1, 2
TIMING_KEYS = {"cdf_seconds", "sample_seconds_before_json_write", "approximate_vector_write_seconds",
               "compare_seconds", "reference_vector_write_seconds", "audit_seconds_before_json_write"}


def sha256(path):
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def load_case():
    case = json.loads((HERE / f"{CASE}.json").read_text())
    arrays = dict(np.load(HERE / f"{CASE}.npz"))
    return case, arrays


def make_protocol_json(case, engine="fp32"):
    n, free = case["n"], case["open_vertices"]
    anchor = {"engine": engine, "source_plan": "inplace_k2_fp32" if engine == "fp32" else "half_k1",
              "source_prefix_index": 0,
              "input_data_bits": "0" * n, "expected_amplitudes_sha256": "0" * 64,
              "expected_device_name": "SYNTHETIC DEVICE", "expected_numpy_version": np.__version__,
              "expected_cupy_version": "SYNTHETIC NO CUPY", "scope": "SYNTHETIC ANCHOR, NO EXPERIMENT"}
    return make_run_protocol(SEED, AUDIT_SEED, COUNT, WORKERS, AUDITS, n, free, engine, anchor)


def contraction_meta(case, arrays, dtype):
    eng = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                 case["parity_operations"], case["open_vertices"])
    return eng, {"seconds": 0.0, "part": 0, "parts": 1, "slices_evaluated": 2 ** len(case["parity_operations"]),
                 "prefix_dtype": dtype, "rmax": case["plan"]["rmax"], "terminal_rank": len(eng.terminal_basis),
                 "work_per_slice": case["plan"]["work"], "open_vertices": case["open_vertices"],
                 "vector_scale": "sqrt(2^(n-k)); sum all complex parts before probabilities"}


def build_rows(case, arrays, protocol, outdir):
    """Rows from the records module, with oracle blocks and the reference's draw and audit."""
    n, free = case["n"], case["open_vertices"]
    ring = list(range(n))
    eng, gen_meta = contraction_meta(case, arrays, "complex64")
    _, ref_meta = contraction_meta(case, arrays, "complex128")
    ident = {"worker_id": 0, "manifest_sha256": "", "protocol_sha256": ""}
    audit_ids = protocol["audit"]["ids_by_worker"]["0"]
    samples, audits, vectors = [], [], {}
    rows_by_id = {}
    with (outdir / "samples.jsonl").open("x") as stream:
        for rec in protocol["generation"]["records"]:
            x = np.array([int(c) for c in rec["input_data_bits"]], np.uint8)
            exact, _ = eng.block(x)
            approx = exact.astype(np.complex64).astype(np.complex128)
            draw = draw_checked(approx, rec["draw_uniform"])
            row = records.sample_row(rec, draw, gen_meta, n=n, free=free, ring=ring, audit_ids=audit_ids,
                                     cdf_seconds=0.0, **ident)
            if rec["sample_id"] in audit_ids:
                meta, sec = records.save_vector(outdir / f"approx_{rec['sample_id']:06d}.npy", approx)
                row["approximate_vector_file"] = meta
                row["approximate_vector_write_seconds"] = sec
                vectors[f"approx_{rec['sample_id']}"] = approx
                vectors[f"reference_{rec['sample_id']}"] = exact
            row["sample_seconds_before_json_write"] = 0.0
            records.append_row(stream, row)
            samples.append(row)
            rows_by_id[rec["sample_id"]] = row
    with (outdir / "audits.jsonl").open("x") as stream:
        for sid in audit_ids:
            ref = vectors[f"reference_{sid}"]
            meta, sec = records.save_vector(outdir / f"reference_{sid:06d}.npy", ref)
            row = records.audit_row(rows_by_id[sid], vectors[f"approx_{sid}"], ref, ref_meta, n=n, free=free,
                                    reference_vector_file=meta, audit_vector_pair=audit_vector_pair, **ident)
            row.update({"compare_seconds": 0.0, "reference_vector_write_seconds": sec,
                        "audit_seconds_before_json_write": 0.0})
            records.append_row(stream, row)
            audits.append(row)
    return samples, audits, vectors


def write_bundle(bundle, case, protocol):
    """A synthetic bundle the verifier accepts with synthetic=True (no circuit data)."""
    (bundle / "inputs").mkdir(parents=True)
    (bundle / "protocol.json").write_text(json.dumps(protocol, indent=2) + "\n")
    n = case["n"]
    ops = [list(o) for o in case["parity_operations"]]
    plans = {"open_vertices": case["open_vertices"],
             "plans": [{"name": name, "operations": ops, "rmax": case["plan"]["rmax"]}
                       for name in (protocol["generation_plan"], "inplace_k3_fp64")]}
    (bundle / "inputs" / "plans.json").write_text(json.dumps(plans, indent=2) + "\n")
    np.savez(bundle / "inputs" / "injected_graph.npz", graph=np.zeros((n, n), np.uint8),
             unitaries=np.asarray([np.eye(2)] * n), order=np.arange(n), ring=np.arange(n))
    files = {str(p.relative_to(bundle)): sha256(p) for p in sorted(bundle.rglob("*")) if p.is_file()}
    manifest = {"schema_version": "dcs245-bundle-v1", "synthetic_only": True, "n": n, "files": files,
                "scope": "SYNTHETIC TEST BUNDLE"}
    (bundle / "manifest.json").write_text(json.dumps(manifest, indent=2) + "\n")


def complete_worker(bundle, wdir, protocol):
    """The worker's control-plane files around its rows (worker.py:46-60, 78-82, 164-190)."""
    mh, ph = sha256(bundle / "manifest.json"), sha256(bundle / "protocol.json")
    ids = [r["sample_id"] for r in protocol["generation"]["records"]]
    audit_ids = protocol["audit"]["ids_by_worker"]["0"]
    for name in ("samples.jsonl", "audits.jsonl"):  # bind the rows to this bundle
        rows = [json.loads(line) for line in (wdir / name).read_text().splitlines() if line.strip()]
        for r in rows:
            r["manifest_sha256"], r["protocol_sha256"] = mh, ph
        (wdir / name).write_text("".join(json.dumps(r) + "\n" for r in rows))
    source = {"worker_id": 0, "worker_count": WORKERS, "synthetic_only": True, "manifest_sha256": mh,
              "protocol_sha256": ph, "sample_ids": ids, "audit_ids": audit_ids, "engine": protocol["engine"]}
    hardware = {"device_name": "SYNTHETIC DEVICE", "compute_capability": [0, 0], "numpy": np.__version__,
                "cupy": "SYNTHETIC NO CUPY", "visible_device_count": 1, "cuda_driver_version": 0,
                "cuda_runtime_version": 0, "nvrtc_version": [0, 0]}
    anchor = protocol["anchor"]
    anchor_rec = {"worker_id": 0, "input_data_bits": anchor["input_data_bits"],
                  "expected_amplitudes_sha256": anchor["expected_amplitudes_sha256"],
                  "actual_amplitudes_sha256": anchor["expected_amplitudes_sha256"], "passed": True,
                  **{k: hardware[k] for k in ("device_name", "numpy", "cupy", "cuda_driver_version",
                                              "cuda_runtime_version", "nvrtc_version")}}
    for name, value in (("source.json", source), ("hardware.json", hardware), ("anchor.json", anchor_rec)):
        (wdir / name).write_text(json.dumps(value, indent=2) + "\n")
    now = time.time()
    summary = {"completed": True, **source, "sample_count": len(ids), "audit_count": len(audit_ids),
               "anchor_amplitudes_sha256": anchor["expected_amplitudes_sha256"], "process_start_unix": now,
               "samples_sha256": sha256(wdir / "samples.jsonl"), "audits_sha256": sha256(wdir / "audits.jsonl"),
               **{k: 0.0 for k in ("generation_setup_seconds", "generation_seconds", "generation_contraction_seconds",
                                   "generation_cdf_seconds", "generation_write_seconds", "reference_setup_seconds",
                                   "audit_seconds", "audit_contraction_seconds", "audit_compare_seconds",
                                   "audit_write_seconds", "anchor_seconds")},
               "worker_seconds_to_summary_build": 1.0}
    (wdir / "summary.json").write_text(json.dumps(summary, indent=2) + "\n")
    files = {p.name: {"bytes": p.stat().st_size, "sha256": sha256(p)} for p in sorted(wdir.iterdir()) if p.is_file()}
    (wdir / "artifacts.json").write_text(json.dumps({"worker_id": 0, "files": files}, indent=2) + "\n")
    completed = {"completed": True, "worker_id": 0, "worker_seconds_to_complete_marker": 2.0, "end_unix": now + 2,
                 "summary_sha256": sha256(wdir / "summary.json"), "artifacts_sha256": sha256(wdir / "artifacts.json")}
    (wdir / "completed.json").write_text(json.dumps(completed, indent=2) + "\n")


def run_verifier(root, protocol, case, rows_dir):
    bundle, artifacts = root / "bundle", root / "artifacts"
    write_bundle(bundle, case, protocol)
    wdir = artifacts / "worker0"
    shutil.copytree(rows_dir, wdir)
    complete_worker(bundle, wdir, protocol)
    ledger = root / "ledger.json"
    ledger.write_text(json.dumps({"terminal": "Succeeded", "log_return_code": 0, "declared_gpu_limit": WORKERS,
                                  "worker_count": WORKERS, "gpus_per_worker": 1,
                                  "central_monotonic_submit_to_terminal_observed_seconds": 1.0,
                                  "central_monotonic_submit_to_all_logs_returned_seconds": 1.0,
                                  "central_monotonic_submit_to_all_artifacts_verified_seconds": 2.0,
                                  "max_observed_running_workers": 1}))
    return ref_verify.verify_run(bundle, artifacts, ledger, synthetic=True)


def strip(row):
    return {k: v for k, v in row.items() if k not in TIMING_KEYS and k not in ("manifest_sha256", "protocol_sha256")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--verify-artifacts", type=Path, default=None)
    ap.add_argument("--engine", default="fp32", choices=["fp32", "half"],
                    help="protocol engine of the verified artifacts (half: HalfConditionalBlockGPU rows)")
    args = ap.parse_args()
    case, arrays = load_case()
    if args.verify_artifacts is not None:
        protocol = make_protocol_json(case, args.engine)
        with tempfile.TemporaryDirectory() as tmp:
            result = run_verifier(Path(tmp), protocol, case, args.verify_artifacts)
        print(json.dumps({k: result[k] for k in ("validation_passed", "record_and_full_vector_validation_passed",
                                                 "timing_validation_passed", "sample_count", "audit_count",
                                                 "failures")}, indent=1))
        return
    protocol = make_protocol_json(case)
    with tempfile.TemporaryDirectory() as tmp:
        rows_dir = Path(tmp) / "rows"
        rows_dir.mkdir()
        samples, audits, vectors = build_rows(case, arrays, protocol, rows_dir)
        result = run_verifier(Path(tmp) / "verify", protocol, case, rows_dir)
    out = {"case": CASE, "protocol": protocol, "samples": [strip(r) for r in samples],
           "audits": [strip(r) for r in audits],
           "verifier": {k: result[k] for k in ("validation_passed", "record_and_full_vector_validation_passed",
                                               "timing_validation_passed", "sample_count", "audit_count",
                                               "failures")}}
    (HERE / "records.json").write_text(json.dumps(out, indent=1))
    np.savez_compressed(HERE / "records.npz", **vectors)
    print(json.dumps(out["verifier"], indent=1))


if __name__ == "__main__":
    main()
