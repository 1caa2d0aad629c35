"""Host-side sampler interface against the reference's own outputs (no GPU): the PCG64 protocol
schedule, the index -> bitstring mapping with a non-identity ring, and the audit selection."""
import numpy as np
import pytest

from dcs245_classical_sampling_b200 import sampling


def test_make_protocol_matches_reference_records(golden):
    """sampling_protocol.py:14-41: every record field the reference wrote, for a mixture weight
    below 1 (both branches) and for the 64-qubit workload's prefixes."""
    s, _ = golden("sampler")
    got = sampling.make_protocol(733245, 113, 6, [5, 1, 3], .45)["records"]
    assert len(got) == len(s["protocol_733245"])
    for g, want in zip(got, s["protocol_733245"]):
        for key in ("sample_id", "conditional_branch", "branch_uniform", "draw_uniform", "input_data_bits"):
            assert g[key] == want[key], key
    got64 = sampling.make_protocol(24520, 3, 64, list(range(44, 64)))["records"]
    for g, want in zip(got64, s["protocol64"]):
        for key in want:
            assert g[key] == want[key], key


def test_make_protocol_errors():
    with pytest.raises(ValueError):
        sampling.make_protocol(1, 4, 6, [5, 5])
    with pytest.raises(ValueError):
        sampling.make_protocol(1, 4, 6, [6])
    with pytest.raises(ValueError):
        sampling.make_protocol(1, 0, 6, [1])
    with pytest.raises(ValueError):
        sampling.make_protocol(1, 4, 6, [1], mixture_weight=1.5)


def test_assemble_output_matches_reference(golden):
    """sampling_protocol.py:91-100 with the reference's small permutation and with a 64-qubit
    non-identity ring (20 free bits)."""
    s, _ = golden("sampler")
    for i, (bits, qiskit) in enumerate(s["assemble"]):
        assert sampling.assemble_output("000000", [5, 1, 3], i, [5, 0, 4, 1, 3, 2]) == (bits, qiskit)
    a = s["assemble64"]
    assert sorted(a["ring"]) == list(range(64)) and a["ring"] != list(range(64))
    for c in a["cases"]:
        assert list(sampling.assemble_output(c["input_data_bits"], a["free"], c["A_index"], a["ring"])) == c["out"]


def test_assemble_output_errors():
    with pytest.raises(ValueError):
        sampling.assemble_output("000000", [5, 1, 3], 8)
    with pytest.raises(ValueError):
        sampling.assemble_output("000000", [5, 1, 3], 1, [0, 0, 1, 2, 3, 4])


def test_audit_ids_match_reference(golden):
    """production/protocol_common.py:22-31: the audit ids of the reference's make_run_protocol."""
    s, _ = golden("sampler")
    for c in s["audit_ids"]:
        got = sampling.make_audit_ids(c["audit_seed"], c["count"], c["workers"], c["per_worker"])
        assert {str(w): ids for w, ids in got.items()} == c["ids_by_worker"]
        assert sorted(i for ids in got.values() for i in ids) == c["ids"]


def test_audit_ids_errors():
    with pytest.raises(ValueError):
        sampling.make_audit_ids(1, 10, 4, 3)
    with pytest.raises(ValueError):
        sampling.make_audit_ids(1, 10, 0, 1)


def test_straddle_margin_bounds_the_cdf_shift():
    """The straddle margin: two blocks within relative L2 error r have normalised CDFs within 2r."""
    rng = np.random.default_rng(9)
    for r in (1e-5, 1e-3, 1e-2):
        for _ in range(20):
            a = rng.normal(size=4096) + 1j * rng.normal(size=4096)
            e = rng.normal(size=4096) + 1j * rng.normal(size=4096)
            b = a + e * (r * np.linalg.norm(a) / np.linalg.norm(e))
            pa, pb = np.abs(a) ** 2, np.abs(b) ** 2
            shift = np.max(np.abs(np.cumsum(pa) / pa.sum() - np.cumsum(pb) / pb.sum()))
            assert shift <= 2 * r
    assert sampling.CDF_SHIFT_BOUND == 2 * sampling.COMPLEX64_REL_L2


def test_scale_flags_raise_the_right_error():
    """Bit 0 of an item's scale flags is the reference's nonfinite error; bit 2 a generated
    kernel's wait between tiles that gave up."""
    from dcs245_classical_sampling_b200.engine import raise_for_flags
    raise_for_flags(np.array([0, 2], np.int64))
    with pytest.raises(ArithmeticError, match="Nonfinite"):
        raise_for_flags(np.array([0, 1], np.int64))
    with pytest.raises(RuntimeError, match="gave up"):
        raise_for_flags(np.array([5, 0], np.int64))
