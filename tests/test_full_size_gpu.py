"""Parity at the full 64-qubit size (ring64_d73_t314_k20: rmax 34, 128 GiB complex64 table, 2^20
block) through size-independent properties: the tuned fused block against an independent
complex128 recontraction with one more parity slice (c_y, as the reference's audits), and the
draw of the block against the oracle sampler on the same vector."""
import gc

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_64_qubit_block_audit_and_draw():
    from dcs245_classical_sampling_b200.audit import audit_vector_pair, relative_l2
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    from dcs245_classical_sampling_b200.sampling import draw_checked, make_protocol
    from dcs245_classical_sampling_b200.workloads import build_workload
    from oracle import sampler_ref
    free = torch.cuda.mem_get_info()[0]
    if free < 140 * 2 ** 30:
        pytest.skip("needs a 180 GB device (128 GiB tables)")
    w = build_workload("ring64_d73_t314_k20")
    eng = InplaceConditionalBlockGPU(w["graph"], w["unitaries"], w["n"], w["order"], w["parity_operations"],
                                     w["open_vertices"])
    eng.alloc(np.complex64, mode="fused")  # the tuned configuration (autotune_cache.json)
    rec = make_protocol(245, 1, w["n"], w["open_vertices"])["records"][0]
    x = np.array([int(c) for c in rec["input_data_bits"]], np.uint8)
    v, meta = eng.block(x)
    assert meta["slices_evaluated"] == 4 and v.shape == (1 << 20,)
    d = draw_checked(v, rec["draw_uniform"])
    host = v.cpu().numpy()
    ref_draw = sampler_ref.draw(host, rec["draw_uniform"])
    assert d["A_index"] == ref_draw["A_index"] or d["cdf_tie"]
    del eng, v
    gc.collect()
    torch.cuda.empty_cache()
    wa = build_workload("ring64_d73_t314_k20_audit")
    ref = InplaceConditionalBlockGPU(wa["graph"], wa["unitaries"], wa["n"], wa["order"], wa["parity_operations"],
                                     wa["open_vertices"])
    ref.alloc(np.complex128, mode="device")
    r, rmeta = ref.block(x)
    assert rmeta["slices_evaluated"] == 8
    a = audit_vector_pair(r, host, 0)
    assert a["normalized_conditional_overlap_abs"] >= 0.9999
    assert relative_l2(r, host) < 1e-5
    del ref, r
    gc.collect()
    torch.cuda.empty_cache()
