"""Production record rows written on the GPU (records.write_rows) pass the reference verifier's
per-row checks (source/production/verify.py:300-328, 430-530), restated here with the oracle."""
import hashlib
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _rows(path):
    return [json.loads(line) for line in path.read_text().splitlines() if line.strip()]


def _check_rows(outdir, protocol, n_ops, engine_kind):
    from oracle import sampler_ref
    g = protocol["generation"]
    n, free = g["n"], g["free_vertices"]
    D = 2.0 ** (n - len(free))
    audit_ids = protocol["audit"]["ids_by_worker"]["0"]
    samples = _rows(outdir / "samples.jsonl")
    audits = _rows(outdir / "audits.jsonl")
    assert [r["sample_id"] for r in samples] == [r["sample_id"] for r in g["records"]]
    assert [r["audit_id"] for r in audits] == audit_ids
    by_id = {}
    for row, rec in zip(samples, g["records"]):
        sid = row["sample_id"]
        for key in ("conditional_branch", "branch_uniform", "draw_uniform", "input_data_bits"):
            assert row[key] == rec[key], key
        assert row["is_preselected_audit"] is (sid in audit_ids)
        assert ("approximate_vector_file" in row) == (sid in audit_ids)
        d = row["draw"]
        u = rec["draw_uniform"]
        assert 0 <= d["A_index"] < 2 ** len(free) and d["uniform"] == u
        assert 0 < d["selected_scaled_weight"] <= d["scaled_mass_fsum"]
        for m in ("numpy", "fsum"):
            assert 0 <= d["cdf_lower_" + m] <= u < d["cdf_upper_" + m] <= 1
        assert math.isclose(d["cdf_upper_fsum"] - d["cdf_lower_fsum"], d["selected_scaled_weight"] / d["scaled_mass_fsum"],
                            rel_tol=1e-8, abs_tol=3e-15)
        assert d["independent_cdf_check_passed"] is True
        bits, qiskit = sampler_ref.assemble(rec["input_data_bits"], free, d["A_index"], list(range(n)))
        assert row["data_bits_ring_order"] == bits and row["bitstring_qiskit"] == qiskit
        assert row["approximate_circuit_probability_estimate"] == d["selected_scaled_weight"] / D
        grid = math.ceil(d["cdf_upper_numpy"] * 2 ** 53) - math.ceil(d["cdf_lower_numpy"] * 2 ** 53)
        assert grid > 0 and row["actual_53bit_conditional_probability"] == grid / 2 ** 53
        c = row["contraction"]
        assert c["parts"] == 1 and c["part"] == 0 and c["slices_evaluated"] == 2 ** n_ops
        assert c["open_vertices"] == free and c["prefix_dtype"] == "complex64"
        if engine_kind == "half":
            assert c["intermediate_storage"] == "float16 real/imaginary components"
        by_id[sid] = row
    for row in audits:
        sid = row["audit_id"]
        sample = by_id[sid]
        vec = {}
        for kind, meta in (("approx", row["approximate_vector_file"]), ("reference", row["reference_vector_file"])):
            path = outdir / meta["path"]
            assert hashlib.sha256(path.read_bytes()).hexdigest() == meta["file_sha256"]
            v = np.load(path, allow_pickle=False)
            assert v.dtype == np.complex128 and v.shape == (2 ** len(free),)
            assert hashlib.sha256(v.astype("<c16").tobytes()).hexdigest() == meta["payload_sha256"]
            vec[kind] = v
        a = vec["approx"]
        draw = sampler_ref.draw(a, sample["draw_uniform"])
        assert row["A_index"] == sample["draw"]["A_index"] == draw["A_index"]
        weights = np.asarray(a.real * a.real + a.imag * a.imag, dtype="<f8")
        assert hashlib.sha256(weights.tobytes()).hexdigest() == sample["draw"]["weights_sha256"]
        assert hashlib.sha256(a.astype("<c16").tobytes()).hexdigest() == sample["draw"]["amplitudes_sha256"]
        law, counts = sampler_ref.cdf_law_vector(vec["approx"])
        lm = row["actual_cdf_law"]
        assert lm["grid_counts_sha256"] == hashlib.sha256(counts.astype("<u8").tobytes()).hexdigest()
        assert lm["actual_law_vector_sha256"] == hashlib.sha256(law.astype("<c16").tobytes()).hexdigest()
        for label, approx in (("witness", law), ("raw_vector_witness", vec["approx"])):
            want = sampler_ref.audit_pair(vec["reference"], approx)
            for key, value in want.items():
                assert math.isclose(row[label][key], value, rel_tol=1e-11), (label, key)
        rc = row["reference_contraction"]
        assert rc["prefix_dtype"] == "complex128" and rc["parts"] == 1 and rc["slices_evaluated"] == 2 ** n_ops
        p_ref = float(abs(vec["reference"][row["A_index"]]) ** 2 / D)
        assert row["reference_selected_probability"] == p_ref
        assert row["approximate_selected_probability_estimate"] == sample["approximate_circuit_probability_estimate"]
        assert row["witness"]["normalized_conditional_overlap_abs"] > 0.9999


@pytest.mark.parametrize("engine_kind", ["fp32", "half"])
def test_written_rows_pass_verifier_row_checks(golden, tmp_path, engine_kind):
    from dcs245_classical_sampling_b200 import records
    from dcs245_classical_sampling_b200.engine import HalfConditionalBlockGPU, InplaceConditionalBlockGPU
    data = json.loads((GOLDEN / "records.json").read_text())
    protocol = data["protocol"]
    case, arrays = golden(data["case"])
    args = (arrays["graph"], arrays["unitaries"], case["n"], case["order"], case["parity_operations"],
            case["open_vertices"])
    eng = (HalfConditionalBlockGPU if engine_kind == "half" else InplaceConditionalBlockGPU)(*args)
    eng.alloc(np.complex64)
    ref = InplaceConditionalBlockGPU(*args)
    ref.alloc(np.complex128)
    g = protocol["generation"]
    records.write_rows(eng, ref, g["records"], protocol["audit"]["ids_by_worker"]["0"], tmp_path, worker_id=0,
                       manifest_sha256="m", protocol_sha256="p", n=g["n"], free=g["free_vertices"],
                       ring=list(range(g["n"])))
    _check_rows(tmp_path, protocol, len(case["parity_operations"]), engine_kind)
