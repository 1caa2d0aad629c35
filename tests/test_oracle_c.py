"""The C/OpenMP CPU-baseline restatement agrees with the NumPy oracle."""
import math

import numpy as np
import pytest

from conftest import rel_l2
from dcs245_classical_sampling_b200 import plan as P
from dcs245_classical_sampling_b200.engine import SliceParams
from oracle import block_ref
from oracle import c as oc


@pytest.mark.parametrize("name", ["c1", "small", "c2"])
def test_c_port_matches_numpy_oracle(golden, name):
    lib = oc.load()
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    oe = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                case["parity_operations"], case["open_vertices"])
    x = np.array([int(c) for c in case["protocol"]["records"][0]["input_data_bits"]], np.uint8)
    _, items = SliceParams(bp).items(x)
    steps = oc.encode(bp.steps)
    for (coef, params, xor), (_, f, yfix, _) in zip(items, [s for s in oe.slice_inputs(x) if s[0]]):
        E = np.zeros(1 << bp.maxslots, np.complex128)
        E[0] = 1
        ls = oc.run_steps(lib, steps, oc.encode_params(params), E)
        term = block_ref._addr(bp.terminal_slots).astype(np.int64)
        want, wls, _ = block_ref.execute(oe.steps, f, yfix, oe.fut, oe.maxslots)
        if not np.any(want):
            assert not np.any(E[term])
        else:
            assert rel_l2(E[term] * math.exp(ls), want * math.exp(wls)) < 1e-13


@pytest.mark.parametrize("name", ["c1", "small"])
def test_cpu_sampler_blocks_and_draws_match_reference(golden, name):
    """The CPU comparator of the small workloads (complete samples with the C executor) against
    the reference's complex128 blocks and draws."""
    from oracle import block_ref
    from oracle.c import CpuSampler
    case, arrays = golden(name)
    eng = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                 case["parity_operations"], case["open_vertices"])
    cs = CpuSampler(eng)
    recs = {r["sample_id"]: r for r in case["protocol"]["records"]}
    for sid, rec in recs.items():
        x = np.array([int(c) for c in rec["input_data_bits"]], np.uint8)
        assert rel_l2(cs.block(x), arrays[f"block_{sid}"]) < 1e-13
    for d in case["draws"]:
        x = np.array([int(c) for c in recs[d["sample_id"]]["input_data_bits"]], np.uint8)
        assert cs.sample(x, d["uniform"])["A_index"] == d["A_index"]
