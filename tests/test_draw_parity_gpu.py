"""Draw parity on the GPU: indices drawn from blocks this build contracts (complex64 and
complex128) against the reference's draws from its own complex128 blocks, given the same
uniforms; the exact sequential CDF mode; the pipelined per-sample loop."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _engine(case, arrays, dtype, mode, jit_shape=False):
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    eng = InplaceConditionalBlockGPU(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                     case["parity_operations"], case["open_vertices"])
    eng.alloc(dtype=dtype, mode=mode)
    if jit_shape:  # the bench's executor: plan-specialised register runs
        low = 4 if eng.plan.maxslots < 16 else 3
        grouping = "greedy" if eng.plan.maxslots < 16 else "bytes"
        eng.set_fused_config(variant=12, low=low, grouping=grouping, jit=True)
        assert eng.fplan.jit is not None and eng.fplan.jit.kernels
    return eng


def _x(rec):
    return np.array([int(c) for c in rec["input_data_bits"]], np.uint8)


@pytest.mark.parametrize("mode", ["device", "fused-jit"])
@pytest.mark.parametrize("name", ["c1full", "c2draws"])
def test_complex64_draws_match_reference_indices(golden, name, mode):
    """Every draw of the widened fixtures (all 256 samples of the 16-qubit workload; 8 prefixes
    of the 40-qubit one): the index drawn from this build's complex64 block equals the
    reference's index from its complex128 block for the same uniform.  The only allowed
    difference is a straddle: the uniform lies within the complex64 error bound of an edge of the
    reference's CDF bin (the draw's cdf_straddle flags such uniforms by a statistical margin)."""
    from dcs245_classical_sampling_b200.sampling import CDF_SHIFT_BOUND, draw_checked
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, "fused" if mode == "fused-jit" else "device",
                  jit_shape=mode == "fused-jit")
    recs = {r["sample_id"]: r for r in case["protocol"]["records"]}
    blocks = {}
    straddles, flagged = 0, 0
    for d in case["draws"]:
        sid = d["sample_id"]
        if sid not in blocks:
            blocks[sid], _ = eng.block(_x(recs[sid]))
            if f"block_{sid}" in arrays:
                assert rel_l2(blocks[sid].cpu().numpy(), arrays[f"block_{sid}"]) < 1e-5
        got = draw_checked(blocks[sid], d["uniform"], hashes=False)
        flagged += got["cdf_straddle"]
        if got["A_index"] != d["A_index"]:
            assert d["uniform_to_nearest_boundary"] < CDF_SHIFT_BOUND, (sid, got["A_index"], d["A_index"])
            straddles += 1
        else:
            assert got["cdf_lower_fsum"] == pytest.approx(d["cdf_lower_fsum"], rel=1e-4, abs=2 * CDF_SHIFT_BOUND)
    print(f"{name} {mode}: {len(case['draws'])} draws, {straddles} straddles, {flagged} near a bin edge")


@pytest.mark.parametrize("name", ["c1", "small", "c2"])
def test_complex128_fused_blocks_match_reference(golden, name):
    """The plan-specialised kernels compiled in FP64 (the complex128 audit executor) against the
    reference's complex128 blocks, and their draws against the reference's draws."""
    from dcs245_classical_sampling_b200.sampling import draw_checked
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex128, "fused")
    assert eng.fplan.fp64 and eng.fplan.jit is not None and eng.fplan.jit.kernels
    for rec in case["protocol"]["records"]:
        v, meta = eng.block(_x(rec))
        assert meta["prefix_dtype"] == "complex128"
        assert rel_l2(v.cpu().numpy(), arrays[f"block_{rec['sample_id']}"]) < 1e-13
        for d in case["draws"]:
            if d["sample_id"] == rec["sample_id"]:
                assert draw_checked(v, d["uniform"], hashes=False)["A_index"] == d["A_index"]


def test_complex128_fused_rejects_library_kernels(golden):
    case, arrays = golden("c1")
    eng = _engine(case, arrays, np.complex128, "fused")
    with pytest.raises(ValueError):
        eng.set_fused_config(jit=False)


@pytest.mark.parametrize("name", ["c1full", "small", "c2"])
def test_exact_cdf_mode_is_numpy_bit_for_bit(golden, name):
    """exact_cdf=True: NumPy's sequential CDF values, bit for bit, for every golden draw (the
    default mode reports the compensated values where it certified the index)."""
    from dcs245_classical_sampling_b200.sampling import draw_checked
    case, arrays = golden(name)
    for d in case["draws"]:
        v = torch.from_numpy(arrays[f"block_{d['sample_id']}"]).cuda()
        got = draw_checked(v, d["uniform"], hashes=False, exact_cdf=True)
        assert got["A_index"] == d["A_index"]
        for key in ("cdf_lower_numpy", "cdf_upper_numpy", "scaled_mass_cdf", "selected_scaled_weight"):
            assert got[key] == d[key], key
        for key in ("cdf_lower_fsum", "cdf_upper_fsum", "scaled_mass_fsum"):
            assert got[key] == pytest.approx(d[key], rel=4e-16, abs=1e-300), key


def test_exact_cdf_mode_on_ties_and_edges():
    """Uniforms on and next to float64 CDF edges of a 2^12 block: the exact mode gives NumPy's
    index and values where the reference accepts the draw, and the reference's error where its
    independent interval check rejects it."""
    from dcs245_classical_sampling_b200.sampling import draw_checked
    from oracle import sampler_ref
    rng = np.random.default_rng(11)
    v = rng.normal(size=1 << 12) + 1j * rng.normal(size=1 << 12)
    w = v.real * v.real + v.imag * v.imag
    cdf = np.cumsum(w) / np.cumsum(w)[-1]
    for i in (0, 31, 32, 33, 2047, 4094):
        for u in (float(cdf[i]), float(np.nextafter(cdf[i], 0)), float(np.nextafter(cdf[i], 1))):
            if not 0 <= u < 1:
                continue
            try:
                want = sampler_ref.draw(v, u)
            except ArithmeticError:
                with pytest.raises(ArithmeticError):
                    draw_checked(v, u, exact_cdf=True)
                continue
            got = draw_checked(v, u, exact_cdf=True)
            assert got["A_index"] == want["A_index"]
            for key in ("cdf_lower_numpy", "cdf_upper_numpy", "scaled_mass_cdf"):
                assert got[key] == want[key], key


def test_sample_checked_equals_block_and_draw(golden):
    """The pipelined per-sample loop gives, sample by sample, the records of engine.block +
    draw_checked (hashes included), and the same host blocks."""
    from dcs245_classical_sampling_b200.sampling import draw_checked, sample_checked
    case, arrays = golden("c1full")
    eng = _engine(case, arrays, np.complex64, "fused", jit_shape=True)
    recs = case["protocol"]["records"][:12]
    xs = [_x(r) for r in recs]
    us = [r["draw_uniform"] for r in recs]
    got, host = sample_checked(eng, xs, us, hashes=True, exact_cdf=True, keep_host_blocks=True)
    assert len(got) == len(xs) == len(host)
    for x, u, g, h in zip(xs, us, got, host):
        v, _ = eng.block(x)
        want = draw_checked(v, u, hashes=True, exact_cdf=True)
        assert g == want
        assert np.array_equal(h, v.cpu().numpy())
    assert sample_checked(eng, [], []) == []
    with pytest.raises(ValueError):
        sample_checked(eng, xs[:1], [1.0])


@pytest.mark.parametrize("kb", [4, 8, 16])
@pytest.mark.parametrize("name", ["small", "c2"])
def test_staged_first_run_is_bit_identical(golden, name, kb):
    """The generated kernels with the next tile's first-run entries staged by asynchronous copies
    compute the same values as without staging, bit for bit, and match the reference."""
    from dcs245_classical_sampling_b200.jit import prefetch_layout
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, "fused", jit_shape=True)
    xs = [_x(r) for r in case["protocol"]["records"]]
    plain = [eng.block(x)[0].cpu().numpy() for x in xs]
    eng.set_fused_config(prefetch_kb=kb)
    assert any(prefetch_layout(eng.fplan, gi) for gi in range(len(eng.fplan.groups)))
    for x, want, rec in zip(xs, plain, case["protocol"]["records"]):
        got = eng.block(x)[0].cpu().numpy()
        assert np.array_equal(got, want)
        assert rel_l2(got, arrays[f"block_{rec['sample_id']}"]) < 1e-5


def test_block_is_copied_to_host_as_the_reference_worker_does(golden):
    """engine.block's vector: np.asarray (the reference fixture's cp.asnumpy stand-in) and the
    CUDA array interface (cupy.asnumpy) give the host block, and the worker's draw on the host
    copy equals the draw on the device tensor (production/worker.py:109-110)."""
    from dcs245_classical_sampling_b200.engine import DeviceBlock
    from dcs245_classical_sampling_b200.sampling import draw_checked
    case, arrays = golden("c1")
    eng = _engine(case, arrays, np.complex64, "fused", jit_shape=True)
    rec = case["protocol"]["records"][0]
    v, meta = eng.block(_x(rec))
    assert isinstance(v, DeviceBlock) and v.is_cuda and v.dtype == torch.complex128
    cai = v.__cuda_array_interface__
    assert cai["typestr"] == "<c16" and cai["shape"] == (1 << len(case["open_vertices"]),)
    host = np.asarray(v)
    np.testing.assert_array_equal(host, v.cpu().numpy())
    assert draw_checked(host, rec["draw_uniform"]) == draw_checked(v, rec["draw_uniform"])


@pytest.mark.parametrize("name", ["small", "c2"])
def test_dimension5_runs_and_group_tuning_are_bit_identical(golden, name):
    """Register runs of dimension 5 (variant bit 4) and the per-group kernel choice of
    autotune.tune_groups compute the same blocks, bit for bit, as the dimension-4 kernels; the
    packed FP32x2 form (variant bit 1) within the complex64 tolerance."""
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, "fused", jit_shape=True)
    xs = [_x(r) for r in case["protocol"]["records"]]
    want = [eng.block(x)[0].cpu().numpy() for x in xs]
    eng.set_fused_config(variant=28)
    assert any(int(v) & 16 for v in eng.fplan.groups["variant"])
    for x, w in zip(xs, want):
        assert np.array_equal(eng.block(x)[0].cpu().numpy(), w)
    from dcs245_classical_sampling_b200.jit import packable
    eng.set_fused_config(variant=14)  # packed FP32x2 form where the runs leave tile bit 0 free
    assert any(packable(eng.fplan, gi) for gi in range(len(eng.fplan.groups)))
    for x, w, rec in zip(xs, want, case["protocol"]["records"]):  # FP32x2 may round differently
        got = eng.block(x)[0].cpu().numpy()
        assert rel_l2(got, w) < 1e-5 and rel_l2(got, arrays[f"block_{rec['sample_id']}"]) < 1e-5
    eng.set_fused_config(variant=12)
    rep = eng.tune_groups(save=False, repeats=1)
    assert set(rep["group_cfg"]) == {str(g) for g in range(len(eng.fplan.groups))}
    for x, w in zip(xs, want):
        assert np.array_equal(eng.block(x)[0].cpu().numpy(), w)


@pytest.mark.parametrize("name", ["small", "c2"])
def test_smaller_ctas_are_bit_identical(golden, name):
    """Generated kernels of 128 threads per CTA (each thread taking two cosets of the larger runs),
    with and without staging and with dimension-5 runs, give the 256-thread kernels' blocks bit
    for bit."""
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, "fused", jit_shape=True)
    xs = [_x(r) for r in case["protocol"]["records"]][:3]
    want = [eng.block(x)[0].cpu().numpy() for x in xs]
    ng = len(eng.fplan.groups)
    for variant, kb in ((12, 0), (12, 8), (28, 8)):
        eng.set_fused_config(variant=variant, group_cfg={gi: (3, kb, 128) for gi in range(ng)})
        assert {k[3] for k in eng.fplan.jit.kernels.values()} == {128}
        for x, w in zip(xs, want):
            assert np.array_equal(eng.block(x)[0].cpu().numpy(), w)


@pytest.mark.parametrize("name", ["small", "c2"])
def test_touching_run_bases_are_bit_identical(golden, name):
    """Register runs whose bases may touch other roles (variant bit 6: representatives and dead
    entries by parities of several local bits, fewer runs), at dimension 4 and 5, with and
    without staging, give the default kernels' blocks bit for bit; the library refuses them."""
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, "fused", jit_shape=True)
    xs = [_x(r) for r in case["protocol"]["records"]][:3]
    want = [eng.block(x)[0].cpu().numpy() for x in xs]
    for variant, kb in ((76, 0), (76, 8), (92, 16), (92, 0)):
        eng.set_fused_config(variant=variant, prefetch_kb=kb)
        assert any(t1 or t2 for t1, t2, _ in eng.fplan.step_touch.values())
        for x, w in zip(xs, want):
            assert np.array_equal(eng.block(x)[0].cpu().numpy(), w)
    with pytest.raises(ValueError, match="touching"):
        eng.set_fused_config(variant=76, jit=False)
        eng.block(xs[0])


def test_wait_between_tiles_gives_up_and_reports(golden):
    """A generated kernel whose wait between tiles can never be satisfied (a test build: the
    barrier's phase needs 64 tiles' arrivals) ends every wait after its poll limit, and the engine
    raises instead of returning the block; the engine then runs normally again."""
    from dcs245_classical_sampling_b200.jit import JitPlan
    case, arrays = golden("c2")
    eng = _engine(case, arrays, np.complex64, "fused", jit_shape=True)
    x = _x(case["protocol"]["records"][0])
    want = eng.block(x)[0].cpu().numpy()
    good = eng.fplan.jit
    eng.fplan.jit = JitPlan(eng.plan, eng.fplan, eng.lib, minb=good.minb, threads=good.threads,
                            group_cfg=good.group_cfg, wait_check=True)
    with pytest.raises(RuntimeError, match="gave up"):
        eng.block(x)
    eng.fplan.jit.close()
    eng.fplan.jit = good
    assert np.array_equal(eng.block(x)[0].cpu().numpy(), want)
