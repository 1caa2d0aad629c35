"""Production record rows in the reference worker's schema (samples.jsonl, audits.jsonl).

The reference worker (source/production/worker.py:95-170) writes one JSON row per sample and
one per audit, plus the sampled and reference vectors of every audited sample as .npy files.
Its independent CPU verifier (source/production/verify.py:351-618) replays those rows: the
PCG64 states, the draw record and its CDF intervals, the output bit mapping, the probability
identities, and for audits the 53-bit CDF-law vector and both overlap witnesses.  The builders
here make the same rows from this package's engine, sampler and audit, so the reference's
verifier stays usable on B200 runs.

Not built: the bundle manifest and its validation, hardware.json, the pilot anchor,
summary.json, artifacts.json and completed.json.  They are the worker's control plane around
the rows, not the sampling path.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import time
from pathlib import Path

import numpy as np

from .sampling import assemble_output

PROBABILITY_SCOPE = ("Circuit estimate uses approximate amplitudes; sampler probability includes uniform prefix "
                     "and the finite-grid CDF law.")
AUDIT_SCOPE = "Preselected full-vector audit; XEB shown only for this audited subset; FP64 reference is numerical."


def sha256_bytes(data):
    return hashlib.sha256(data).hexdigest()


def _host(v):
    """A block as a host complex128 array (torch tensors are copied from the device)."""
    if hasattr(v, "detach"):
        v = v.detach().cpu().numpy()
    return np.asarray(v, dtype=np.complex128)


def actual_cdf_law_vector(amplitudes):
    """Amplitudes whose probabilities are the sampler's 53-bit CDF law, and their commitments
    (protocol_common.py:48-70).  The sequential float64 cumsum is the sampler's own CDF, so the
    grid counts are exact integers of that CDF; phases come from the source amplitudes."""
    a = _host(amplitudes)
    if a.ndim != 1 or not len(a) or not np.isfinite(a).all():
        raise ValueError("Invalid vector")
    weights = np.asarray(a.real * a.real + a.imag * a.imag, dtype="<f8", order="C")
    cumulative = np.cumsum(weights, dtype=np.float64)
    if not cumulative[-1] > 0:
        raise ArithmeticError("Zero conditional vector; no silent replacement")
    total = float(cumulative[-1])
    cumulative /= total
    cumulative[-1] = 1.0
    ends = np.ceil(cumulative * 2.0 ** 53).astype(np.uint64)
    counts = np.diff(ends, prepend=np.uint64(0))
    if int(counts.sum(dtype=np.uint64)) != 1 << 53:
        raise AssertionError("Grid counts do not normalize")
    phases = np.ones(len(a), np.complex128)
    nz = np.abs(a) > 0
    phases[nz] = a[nz] / np.abs(a[nz])
    law = phases * np.sqrt(counts.astype(np.float64) / 2.0 ** 53)
    meta = {"grid_bits": 53, "grid_total": 1 << 53,
            "grid_counts_sha256": sha256_bytes(counts.astype("<u8", copy=False).tobytes()),
            "actual_law_vector_sha256": sha256_bytes(law.astype("<c16", copy=False).tobytes()),
            "source_amplitudes_sha256": sha256_bytes(a.astype("<c16", copy=False).tobytes()),
            "source_weights_sha256": sha256_bytes(weights.tobytes()), "source_cdf_total": total,
            "law_norm_squared": float(np.vdot(law, law).real)}
    return law, meta


def save_vector(path, value):
    """A complex128 vector as .npy, durably written, with the metadata rows bind it by
    (worker.py:24-30).  Returns (metadata, seconds)."""
    start = time.perf_counter()
    value = _host(value)
    path = Path(path)
    with path.open("xb") as f:
        np.save(f, value, allow_pickle=False)
        f.flush()
        os.fsync(f.fileno())
    digest = hashlib.sha256(path.read_bytes()).hexdigest()
    meta = {"path": path.name, "file_sha256": digest,
            "payload_sha256": sha256_bytes(value.astype("<c16", copy=False).tobytes()),
            "shape": list(value.shape), "dtype": "complex128"}
    return meta, time.perf_counter() - start


def append_row(stream, row):
    """One JSON line, flushed and fsync'd (worker.py:33-35).  Returns the seconds spent."""
    t = time.perf_counter()
    stream.write(json.dumps(row) + "\n")
    stream.flush()
    os.fsync(stream.fileno())
    return time.perf_counter() - t


def sample_row(record, draw, contraction, *, worker_id, manifest_sha256, protocol_sha256, n, free, ring,
               audit_ids, cdf_seconds):
    """The sample row of worker.py:115-123 (without the vector file and the final timing, which
    the writer adds).  `record` is a make_protocol record with its PCG64 states."""
    D = 2.0 ** (n - len(free))
    bits, qiskit = assemble_output(record["input_data_bits"], free, draw["A_index"], ring)
    grid = math.ceil(draw["cdf_upper_numpy"] * 2.0 ** 53) - math.ceil(draw["cdf_lower_numpy"] * 2.0 ** 53)
    return {**record, "worker_id": worker_id, "manifest_sha256": manifest_sha256,
            "protocol_sha256": protocol_sha256, "is_preselected_audit": record["sample_id"] in audit_ids,
            "draw": draw, "contraction": contraction, "cdf_seconds": cdf_seconds,
            "data_bits_ring_order": bits, "bitstring_qiskit": qiskit,
            "approximate_circuit_probability_estimate": draw["selected_scaled_weight"] / D,
            "actual_53bit_conditional_probability": grid / 2.0 ** 53,
            "actual_joint_sampler_probability": grid / 2.0 ** 53 / D,
            "probability_scope": PROBABILITY_SCOPE}


def audit_row(sample, approx, reference, reference_contraction, *, worker_id, manifest_sha256, protocol_sha256,
              n, free, reference_vector_file, audit_vector_pair):
    """The audit row of worker.py:149-158 for one audited sample (without the timing fields).

    `approx` is the vector the sampler drew from, `reference` the complex128 recontraction;
    `audit_vector_pair` is the overlap function (audit.audit_vector_pair on the device)."""
    sid = sample["sample_id"]
    a = _host(approx)
    if sha256_bytes(a.astype("<c16", copy=False).tobytes()) != sample["draw"]["amplitudes_sha256"]:
        raise AssertionError("Actual sampled approximate vector changed")
    law, lawmeta = actual_cdf_law_vector(a)
    if lawmeta["source_weights_sha256"] != sample["draw"]["weights_sha256"]:
        raise AssertionError("Audit weights changed")
    ref = _host(reference)
    index = sample["draw"]["A_index"]
    D = 2.0 ** (n - len(free))
    p_ref = float(abs(ref[index]) ** 2 / D)
    return {"audit_id": sid, "worker_id": worker_id, "manifest_sha256": manifest_sha256,
            "protocol_sha256": protocol_sha256, "witness": audit_vector_pair(ref, law, sid),
            "raw_vector_witness": audit_vector_pair(ref, a, sid), "actual_cdf_law": lawmeta,
            "approximate_vector_file": sample["approximate_vector_file"],
            "reference_vector_file": reference_vector_file, "reference_contraction": reference_contraction,
            "A_index": index, "reference_selected_probability": p_ref,
            "reference_selected_linear_xeb": float(2.0 ** n * p_ref - 1),
            "approximate_selected_probability_estimate": sample["approximate_circuit_probability_estimate"],
            "scope": AUDIT_SCOPE}


def write_rows(engine, reference, records, audit_ids, outdir, *, worker_id, manifest_sha256, protocol_sha256,
               n, free, ring):
    """Generate `records` with `engine` (complex64 or half storage), draw each with
    draw_checked, then recontract the audited samples with `reference` (complex128) and write
    samples.jsonl, audits.jsonl and the approx_/reference_ vectors into `outdir`, as the
    reference worker's generation and audit phases do (worker.py:103-163).

    Returns (sample rows, audit rows)."""
    from .audit import audit_vector_pair
    from .sampling import draw_checked
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    samples, selected, audits = {}, {}, []
    with (outdir / "samples.jsonl").open("x") as stream:
        for record in records:
            if not record["conditional_branch"]:
                raise ValueError("This worker requires lambda=1")
            begin = time.perf_counter()
            sid = record["sample_id"]
            x = np.asarray([int(c) for c in record["input_data_bits"]], np.uint8)
            v, contraction = engine.block(x)
            host = v.cpu().numpy()
            del v
            t = time.perf_counter()
            # NumPy's sequential CDF values: the row's grid count is computed from them
            draw = draw_checked(host, record["draw_uniform"], exact_cdf=True)
            cdf_seconds = time.perf_counter() - t
            row = sample_row(record, draw, contraction, worker_id=worker_id, manifest_sha256=manifest_sha256,
                             protocol_sha256=protocol_sha256, n=n, free=free, ring=ring, audit_ids=audit_ids,
                             cdf_seconds=cdf_seconds)
            if sid in audit_ids:
                selected[sid] = host
                meta, elapsed = save_vector(outdir / f"approx_{sid:06d}.npy", host)
                row["approximate_vector_file"] = meta
                row["approximate_vector_write_seconds"] = elapsed
            row["sample_seconds_before_json_write"] = time.perf_counter() - begin
            append_row(stream, row)
            samples[sid] = row
    with (outdir / "audits.jsonl").open("x") as stream:
        for sid in audit_ids:
            begin = time.perf_counter()
            sample = samples[sid]
            x = np.asarray([int(c) for c in sample["input_data_bits"]], np.uint8)
            v, contraction = reference.block(x)
            ref = v.cpu().numpy()
            del v
            t = time.perf_counter()
            meta, elapsed = save_vector(outdir / f"reference_{sid:06d}.npy", ref)
            row = audit_row(sample, selected[sid], ref, contraction, worker_id=worker_id,
                            manifest_sha256=manifest_sha256, protocol_sha256=protocol_sha256, n=n, free=free,
                            reference_vector_file=meta, audit_vector_pair=audit_vector_pair)
            row["compare_seconds"] = time.perf_counter() - t - elapsed
            row["reference_vector_write_seconds"] = elapsed
            row["audit_seconds_before_json_write"] = time.perf_counter() - begin
            append_row(stream, row)
            audits.append(row)
    return [samples[r["sample_id"]] for r in records], audits
