"""Production record rows (records.py) against rows the reference's own verifier accepted.

tests/golden/make_records_golden.py built these rows with records.py, ran the reference's
verify_run (source/production/verify.py:351-618) over them in a synthetic bundle, and stored
its verdict.  Here the rows are rebuilt from the same inputs and must come out identical, so
every row records.py writes today is one the reference verifier accepted.
"""
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN
from dcs245_classical_sampling_b200 import records
from oracle import sampler_ref

TIMING = {"cdf_seconds", "sample_seconds_before_json_write", "approximate_vector_write_seconds",
          "compare_seconds", "reference_vector_write_seconds", "audit_seconds_before_json_write",
          "manifest_sha256", "protocol_sha256"}


@pytest.fixture(scope="module")
def fixture():
    data = json.loads((GOLDEN / "records.json").read_text())
    vectors = dict(np.load(GOLDEN / "records.npz"))
    return data, vectors


def _strip(row):
    return {k: v for k, v in row.items() if k not in TIMING}


def _audit_pair(ref, approx, audit_id):
    """The reference's audit record (full_vector_audit_certificate.py:15-43) from the oracle's
    overlap (oracle/sampler_ref.py:audit_pair)."""
    r = sampler_ref.audit_pair(ref, approx)
    ov = r["normalized_conditional_overlap_abs"]
    return {"audit_id": audit_id, "vector_length": len(ref), "reference_scaled_mass": r["reference_scaled_mass"],
            "approximate_input_mass": r["approximate_input_mass"], "normalized_conditional_overlap_abs": ov,
            "normalized_conditional_fidelity": ov ** 2 if ov is not None else None,
            "uncapped_overlap_witness": r["uncapped_overlap_witness"], "clipped_weight": r["clipped_weight"],
            "loss": 1 - r["clipped_weight"],
            "reference_arithmetic": "complex128 numerical reference; not an interval-arithmetic proof"}


def _same(a, b, path=""):
    """Equal JSON values; floats to 1e-14 relative (the verifier's own tolerance is 3e-13)."""
    if isinstance(a, dict):
        assert set(a) == set(b), (path, set(a) ^ set(b))
        for k in a:
            _same(a[k], b[k], f"{path}.{k}")
    elif isinstance(a, list):
        assert len(a) == len(b), path
        for i, (x, y) in enumerate(zip(a, b)):
            _same(x, y, f"{path}[{i}]")
    elif isinstance(a, float) and isinstance(b, float):
        assert math.isclose(a, b, rel_tol=1e-14, abs_tol=0.0), (path, a, b)
    else:
        assert a == b, (path, a, b)


def test_reference_verifier_accepted_the_golden_rows(fixture):
    data, _ = fixture
    v = data["verifier"]
    assert v["validation_passed"] and v["record_and_full_vector_validation_passed"] and not v["failures"]
    assert v["sample_count"] == len(data["samples"]) and v["audit_count"] == len(data["audits"])


def test_sample_and_audit_rows_rebuild_identically(fixture, tmp_path):
    data, vectors = fixture
    protocol = data["protocol"]
    g = protocol["generation"]
    n, free = g["n"], g["free_vertices"]
    audit_ids = protocol["audit"]["ids_by_worker"]["0"]
    ident = {"worker_id": 0, "manifest_sha256": "", "protocol_sha256": ""}
    rows = {}
    for rec, want in zip(g["records"], data["samples"]):
        row = records.sample_row(rec, want["draw"], want["contraction"], n=n, free=free, ring=list(range(n)),
                                 audit_ids=audit_ids, cdf_seconds=0.0, **ident)
        sid = rec["sample_id"]
        if sid in audit_ids:
            meta, _ = records.save_vector(tmp_path / f"approx_{sid:06d}.npy", vectors[f"approx_{sid}"])
            row["approximate_vector_file"] = meta
        _same(_strip(row), want)
        rows[sid] = row
    for want in data["audits"]:
        sid = want["audit_id"]
        ref = vectors[f"reference_{sid}"]
        meta, _ = records.save_vector(tmp_path / f"reference_{sid:06d}.npy", ref)
        row = records.audit_row(rows[sid], vectors[f"approx_{sid}"], ref, want["reference_contraction"], n=n,
                                free=free, reference_vector_file=meta, audit_vector_pair=_audit_pair, **ident)
        _same(_strip(row), want)


def test_law_vector_matches_reference_known_answers(golden):
    """records.actual_cdf_law_vector against protocol_common.actual_cdf_law_vector's outputs."""
    s, _ = golden("sampler")
    for case in s["law"]:
        a = np.array(case["re"]) + 1j * np.array(case["im"])
        law, meta = records.actual_cdf_law_vector(a)
        assert np.array_equal(law, np.array(case["law_re"]) + 1j * np.array(case["law_im"]))
        for key, value in case["meta"].items():
            assert meta[key] == value, key


def test_row_errors(fixture, tmp_path):
    """A changed sampled vector or weights is an error, never a silent rewrite (worker.py:141-145)."""
    data, vectors = fixture
    protocol = data["protocol"]
    g = protocol["generation"]
    sid = protocol["audit"]["ids_by_worker"]["0"][0]
    sample = dict(data["samples"][sid])
    sample["approximate_vector_file"] = {"path": "x"}
    approx = vectors[f"approx_{sid}"].copy()
    approx[0] *= 1 + 1e-12
    with pytest.raises(AssertionError):
        records.audit_row(sample, approx, vectors[f"reference_{sid}"], {}, worker_id=0, manifest_sha256="",
                          protocol_sha256="", n=g["n"], free=g["free_vertices"], reference_vector_file={},
                          audit_vector_pair=_audit_pair)
    with pytest.raises(ArithmeticError):
        records.actual_cdf_law_vector(np.zeros(8, complex))
    meta, _ = records.save_vector(tmp_path / "v.npy", approx)
    with pytest.raises(FileExistsError):  # rows and vectors are written once, never replaced
        records.save_vector(tmp_path / "v.npy", approx)
    assert meta["shape"] == [len(approx)] and meta["dtype"] == "complex128"


def test_law_vector_grid_counts_by_exact_rationals():
    """The 53-bit law of records.actual_cdf_law_vector against grid counts computed with exact
    rationals from the sequential float64 CDF (the check of test_protocol_cpu.py:22-36), on
    the reference's two vectors and on random ones."""
    from fractions import Fraction
    rng = np.random.default_rng(7)
    vecs = [np.array([0, 1, 1j, 1 + 1j, 0, 2, 1 - 1j, 0], complex),
            np.array([1e-15, 1e-8j, 1, 1j, 2 + 3j, .17, .21j, .01], complex)]
    vecs += [rng.normal(size=64) + 1j * rng.normal(size=64) for _ in range(3)]
    for a in vecs:
        law, meta = records.actual_cdf_law_vector(a)
        weights = a.real * a.real + a.imag * a.imag
        cum, acc = [], 0.0
        for w in weights:
            acc = float(acc + float(w))
            cum.append(acc)
        cum = [float(c / acc) for c in cum]
        cum[-1] = 1.0
        ends = [math.ceil(Fraction.from_float(c) * (1 << 53)) for c in cum]
        counts = [b - a_ for a_, b in zip([0] + ends[:-1], ends)]
        assert sum(counts) == 1 << 53
        target = np.asarray(counts, dtype=float) / 2 ** 53
        assert np.max(np.abs(np.abs(law) ** 2 - target)) < 4e-16
        assert meta["grid_total"] == 1 << 53 and abs(meta["law_norm_squared"] - 1) < 1e-12
        d = sampler_ref.draw(a, .381245)
        assert target[d["A_index"]] > 0
