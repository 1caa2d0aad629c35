"""The reference's gather engine (ConditionalBlockGPU, two-table executor) on the GPU against the
reference's blocks and gather plan."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

CASES = ["c1", "small", "c2"]


def _engine(case, arrays, dtype, **kw):
    from dcs245_classical_sampling_b200.gather import ConditionalBlockGPU
    eng = ConditionalBlockGPU(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                              case["parity_operations"], case["open_vertices"])
    eng.alloc(dtype=dtype, **kw)
    return eng


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-13), (np.complex64, 1e-5)])
@pytest.mark.parametrize("name", CASES)
def test_gather_blocks_match_reference(golden, name, dtype, tol):
    """Blocks of the gather engine equal the reference's (its gather and in-place engines agree to
    2e-15 on these cases), with the reference gather engine's meta."""
    from dcs245_classical_sampling_b200.engine import DeviceBlock
    case, arrays = golden(name)
    g = golden("gather")[0][name]
    eng = _engine(case, arrays, dtype)
    assert eng.rmax == g["rmax"] and eng.work == g["work"] and eng.terminal_basis == g["terminal_basis"]
    for rec in case["protocol"]["records"]:
        x = np.array([int(c) for c in rec["input_data_bits"]], np.uint8)
        v, meta = eng.block(x)
        assert isinstance(v, DeviceBlock) and v.dtype == torch.complex128
        assert rel_l2(v.cpu().numpy(), arrays[f"block_{rec['sample_id']}"]) < tol
        assert meta["rmax"] == g["rmax"] and meta["work_per_slice"] == g["work"]
        assert meta["terminal_rank"] == len(g["terminal_basis"])


def test_gather_one_item_at_a_time_and_parts(golden):
    """One work item per launch gives the same block as all slices at once, and the parts of a
    block sum to it (conditional_block_gpu.py:128-140)."""
    case, arrays = golden("small")
    rec = case["protocol"]["records"][0]
    x = np.array([int(c) for c in rec["input_data_bits"]], np.uint8)
    many = _engine(case, arrays, np.complex128)
    one = _engine(case, arrays, np.complex128, items=1)
    a = many.block(x)[0].cpu().numpy()
    b = one.block(x)[0].cpu().numpy()
    assert rel_l2(a, b) < 1e-14
    parts = sum(one.block(x, part=p, parts=3)[0].cpu().numpy() for p in range(3))
    assert rel_l2(parts, a) < 1e-13


def test_gather_errors(golden):
    from dcs245_classical_sampling_b200.gather import ConditionalBlockGPU
    case, arrays = golden("c1")
    with pytest.raises(ValueError):
        ConditionalBlockGPU(arrays["graph"], arrays["unitaries"], case["n"], case["order"], case["parity_operations"],
                            [0, 0])
    eng = ConditionalBlockGPU(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                              case["parity_operations"], case["open_vertices"])
    with pytest.raises(ValueError):
        eng.alloc(np.float32)
