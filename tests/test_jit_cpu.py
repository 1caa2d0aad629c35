"""Plan-specialised group kernels: the generated sources of the golden plans compile with NVRTC
for sm_100a (no GPU needed), one kernel per group with register runs."""
import ctypes

import pytest

from dcs245_classical_sampling_b200 import _lib
from dcs245_classical_sampling_b200 import jit
from dcs245_classical_sampling_b200 import plan as P
from dcs245_classical_sampling_b200.fused import build_fused_plan


@pytest.mark.parametrize("name", ["c1", "small", "c2"])
@pytest.mark.parametrize("variant", [4, 12])
def test_generated_group_kernels_compile(golden, name, variant):
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    fp = build_fused_plan(bp, max_dim=13, low=4, variant=variant)
    with_runs = [gi for gi in range(len(fp.groups)) if int(fp.groups[gi]["variant"]) & 4]
    assert with_runs
    units = jit.plan_sources(bp, fp, parts=2)
    assert sorted(g for _, gis in units for g in gis) == with_runs
    lib = _lib.load()
    for src, gis in units:
        for gi in gis:
            assert f"dcs_g{gi}(" in src
        img = jit.compile_source(lib, src)
        assert img[:4] == b"\x7fELF"  # a cubin


def test_compile_errors_raise_with_the_log():
    lib = _lib.load()
    with pytest.raises(_lib.DCSError, match="error"):
        jit.compile_source(lib, '#include "runs_jit.cuh"\nextern "C" __global__ void k() { undefined_name(); }\n')
