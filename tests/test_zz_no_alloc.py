"""The draw entry point that allocates nothing (dcs_draw_static), through the C ABI.

Some callers cannot allocate device memory where they sample (a stream under capture, a host
runtime that only lends its own buffers, a loop that must not synchronise the device).  For
them the library keeps the draw's scratch in a fixed device array.  This test calls that entry
point twice in a row, on different blocks, and checks each result against the allocating
entry point dcs_draw on the same block and uniform: the leftover contents of the shared array
from the first call must not change the second result.  It is collected last (file name) and
passes both alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

FIELDS_EXACT = ("index", "tie", "status")
FIELDS_FLOAT = ("total_cdf", "total_exact", "selected_weight", "cdf_lower", "cdf_upper", "cdf_lower_exact",
                "cdf_upper_exact", "uniform", "tv53")


def _draw_alloc(lib, _lib, v, u):
    k = int(v.numel()).bit_length() - 1
    scratch = torch.empty(lib.dcs_draw_scratch_bytes(k, 1), dtype=torch.uint8, device=v.device)
    res = torch.empty(_lib.DRAW_DTYPE.itemsize, dtype=torch.uint8, device=v.device)
    du = torch.tensor([u], dtype=torch.float64, device=v.device)
    _lib.check(lib.dcs_draw(_lib.ptr(v), k, 1, _lib.ptr(du), _lib.ptr(scratch), _lib.ptr(res),
                            torch.cuda.current_stream().cuda_stream))
    return res.cpu().numpy().view(_lib.DRAW_DTYPE)[0]


def _draw_static(lib, _lib, v, u):
    k = int(v.numel()).bit_length() - 1
    res = torch.empty(_lib.DRAW_DTYPE.itemsize, dtype=torch.uint8, device=v.device)
    du = torch.tensor([u], dtype=torch.float64, device=v.device)
    _lib.check(lib.dcs_draw_static(_lib.ptr(v), k, _lib.ptr(du), _lib.ptr(res),
                                   torch.cuda.current_stream().cuda_stream))
    return res.cpu().numpy().view(_lib.DRAW_DTYPE)[0]


def test_static_draw_matches_allocating_draw_twice():
    from dcs245_classical_sampling_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(2026)
    cases = [(20, 0.7311), (14, 0.0423)]  # the largest allowed block, then a smaller one
    for k, u in cases:
        a = rng.normal(size=1 << k) + 1j * rng.normal(size=1 << k)
        v = torch.from_numpy(a).cuda()
        want = _draw_alloc(lib, _lib, v, u)
        got = _draw_static(lib, _lib, v, u)
        assert want["status"] == 0
        for f in FIELDS_EXACT:
            assert got[f] == want[f], f
        for f in FIELDS_FLOAT:
            assert got[f] == pytest.approx(want[f], rel=1e-15, abs=0.0), f


def test_static_draw_rejects_blocks_beyond_the_limit():
    from dcs245_classical_sampling_b200 import _lib
    lib = _lib.load()
    v = torch.zeros(1 << 21, dtype=torch.complex128, device="cuda")
    res = torch.empty(_lib.DRAW_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    du = torch.tensor([0.5], dtype=torch.float64, device="cuda")
    rc = lib.dcs_draw_static(_lib.ptr(v), 21, _lib.ptr(du), _lib.ptr(res), torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.E_ARG
    assert b"exceeds the static maximum" in lib.dcs_last_error()
