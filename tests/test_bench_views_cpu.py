"""The bench line's compute view: entry-steps and FP32 operations of the 64-qubit plan's slice,
and the view's arithmetic on a made-up launch list (no GPU)."""
import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402
from dcs245_classical_sampling_b200 import plan as P  # noqa: E402
from dcs245_classical_sampling_b200.plan import orbit_kind  # noqa: E402


def test_fp32_operations_of_the_64_qubit_slice(golden):
    """Every step of the 64-qubit plan costs 4 FP32 operations per input entry except grows
    (2 per output entry, 4 per input), fixed steps by y, and replace/shrink steps with an even
    partner sign (3); the slice totals are the ones the design quotes."""
    case, arrays = golden("c64plan")
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    es = sum(1 << max(len(st.active_in), len(st.active_out)) for st in bp.steps)
    ops = sum(bench.step_fp32_ops(st, 1) for st in bp.steps)
    assert es == 229817205351
    assert 7.9e11 < ops < 8.1e11
    for st in bp.steps:
        n = 1 << len(st.active_in)
        kind = orbit_kind(st)[0]
        if kind == 4:
            assert (bench.step_fp32_ops(st, 0), bench.step_fp32_ops(st, 1)) == (0, 4 * n)
        elif kind == 5:
            assert (bench.step_fp32_ops(st, 0), bench.step_fp32_ops(st, 1)) == (n, 3 * n)
        elif kind in (3, 6, 7):
            assert bench.step_fp32_ops(st, 1) == (4 if bin(st.K & st.beta).count("1") & 1 else 3) * n


def test_compute_view_arithmetic():
    dom = {"launch_ms": [1.0, 3.0], "launch_entry_steps": [10 ** 9, 3 * 10 ** 9],
           "launch_fp32_ops": [4 * 10 ** 9, 12 * 10 ** 9]}
    v = bench.compute_view(dom, 148, 2000.0)
    assert v["peak"] == pytest.approx(148 * 128 * 2e9 / 1e12)
    assert v["achieved"] == pytest.approx(16e9 / 4e-3 / 1e12)
    assert v["frac"] == pytest.approx(v["achieved"] / v["peak"])
    assert v["entry_steps_per_s"] == pytest.approx(1e12)
    assert v["ps_per_entry_step"] == pytest.approx(1.0)
    assert [x[0] for x in v["slowest_launches"]] == [1, 0]
