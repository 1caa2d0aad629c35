"""GPU parity: the CUDA path (through the C ABI) against the reference's outputs and the oracle."""
import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

CASES = ["c1", "small", "c2"]


def _engine(case, arrays, dtype, mode="device", **kw):
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    eng = InplaceConditionalBlockGPU(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                     case["parity_operations"], case["open_vertices"])
    eng.alloc(dtype=dtype, mode=mode, **kw)
    return eng


def _x(rec):
    return np.array([int(c) for c in rec["input_data_bits"]], np.uint8)


@pytest.mark.parametrize("name", CASES)
def test_complex128_block_matches_reference(golden, name):
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex128)
    for rec in case["protocol"]["records"]:
        v, meta = eng.block(_x(rec))
        assert v.dtype == torch.complex128 and v.is_cuda
        want = arrays[f"block_{rec['sample_id']}"]
        assert rel_l2(v.cpu().numpy(), want) < 1e-13
        ref_meta = case["block_meta"][rec["sample_id"]]
        for key in ("slices_evaluated", "rmax", "terminal_rank", "work_per_slice", "prefix_dtype"):
            assert meta[key] == ref_meta[key], key


@pytest.mark.parametrize("mode", ["device", "plain", "fused"])
@pytest.mark.parametrize("name", CASES)
def test_complex64_block_matches_reference(golden, name, mode):
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, mode=mode)
    for rec in case["protocol"]["records"]:
        v, meta = eng.block(_x(rec))
        want = arrays[f"block_{rec['sample_id']}"]
        err = rel_l2(v.cpu().numpy(), want)
        assert err < 1e-5, err
        assert meta["prefix_dtype"] == "complex64"


@pytest.mark.parametrize("name", CASES)
def test_fused_step_pairs_match_reference(golden, name):
    """The fused kernel with two steps per shared-memory round trip (autotuner option)."""
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, mode="fused")
    eng.set_fused_config(pairs=True)
    assert int(eng.fplan.tile_steps["pair"].sum()) > 0
    for rec in case["protocol"]["records"]:
        v, _ = eng.block(_x(rec))
        assert rel_l2(v.cpu().numpy(), arrays[f"block_{rec['sample_id']}"]) < 1e-5


@pytest.mark.parametrize("name", ["c1", "small", "c2"])
@pytest.mark.parametrize("variant", [2, 3, 4, 12, 13, 6, 7, 15])
def test_fused_kernel_variants_match_reference(golden, name, variant):
    """Paired layout with packed FP32x2 arithmetic (2, 3), register runs of local dimension 3 or
    4 (4, 12, 13) and packed register runs (6, 7, 15): every autotuner variant against the
    reference blocks."""
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, mode="fused")
    eng.set_fused_config(variant=variant, pairs=False, max_dim=13, low=4)
    assert (eng.fplan.groups["variant"] == variant).any()
    for rec in case["protocol"]["records"]:
        v, _ = eng.block(_x(rec))
        assert rel_l2(v.cpu().numpy(), arrays[f"block_{rec['sample_id']}"]) < 1e-5


@pytest.mark.parametrize("name", ["c1", "small", "c2"])
@pytest.mark.parametrize("variant,pairs", [(4, False), (12, False), (4, True), (13, True), (6, False), (15, False)])
def test_plan_specialised_kernels_match_reference(golden, name, variant, pairs):
    """Group kernels generated and compiled for the plan (jit.py) against the reference blocks,
    and against the library's register-run kernel on the same configuration (pairs: two cosets
    per loop iteration in the generated kernels)."""
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, mode="fused")
    eng.set_fused_config(variant=variant, pairs=pairs, max_dim=13, low=4, jit=False)
    lib_blocks = [eng.block(_x(rec))[0].cpu().numpy() for rec in case["protocol"]["records"]]
    eng.set_fused_config(jit=True)
    assert eng.fplan.jit is not None and eng.fplan.jit.kernels
    for rec, lb in zip(case["protocol"]["records"], lib_blocks):
        v, _ = eng.block(_x(rec))
        v = v.cpu().numpy()
        want = arrays[f"block_{rec['sample_id']}"]
        err = rel_l2(v, want)
        assert err < 1e-5
        # the generated kernels divide f0 out of the weights (unit weights), so their FP32
        # rounding differs from the library kernels'; their error must stay as small
        assert err <= max(2.0 * rel_l2(lb, want), 2e-6), (err, rel_l2(lb, want))


@pytest.mark.parametrize("name", ["small", "c2"])
@pytest.mark.parametrize("low", [3, 4])
def test_plan_specialised_kernels_min_bytes_groups(golden, name, low):
    """The tuned shape: groups of fewest table bytes (grouping="bytes"), 3 or 4 low bits."""
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, mode="fused")
    eng.set_fused_config(variant=12, pairs=False, max_dim=13, low=low, grouping="bytes", jit=True)
    for rec in case["protocol"]["records"]:
        v, _ = eng.block(_x(rec))
        assert rel_l2(v.cpu().numpy(), arrays[f"block_{rec['sample_id']}"]) < 1e-5


@pytest.mark.parametrize("threads,minb", [(512, 2), (1024, 1), (128, 6)])
def test_plan_specialised_kernels_other_block_sizes(golden, threads, minb):
    """The generated kernels at other thread counts per CTA (the coset index takes as many thread
    bits) give the reference blocks."""
    case, arrays = golden("c2")
    eng = _engine(case, arrays, np.complex64, mode="fused")
    eng.set_fused_config(variant=4, pairs=False, max_dim=13, low=4, jit=True, threads=threads, minb=minb)
    assert eng.fplan.jit.threads == threads
    for rec in case["protocol"]["records"]:
        v, _ = eng.block(_x(rec))
        assert rel_l2(v.cpu().numpy(), arrays[f"block_{rec['sample_id']}"]) < 1e-5


def test_plan_specialised_kernels_fall_back_without_unit_weights(golden):
    """A free step whose f0 is zero (a custom reference bra orthogonal to the first column of
    its unitary) cannot divide f0 out: that item runs the library kernels and the block still
    equals the oracle's."""
    from oracle import block_ref
    case, arrays = golden("small")
    eng = _engine(case, arrays, np.complex64, mode="fused")
    eng.set_fused_config(variant=12, pairs=False, max_dim=13, low=4, jit=True)
    oeng = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                  case["parity_operations"], case["open_vertices"])
    n = case["n"]
    refs = [q for q in range(n, len(arrays["graph"])) if q in eng.plan.relabel and q not in eng.plan.slices
            and eng.plan.relabel[q] not in eng.plan.fixed]
    q = refs[0]
    U = np.asarray(eng.plan.U_full[q])
    w = {r: np.array([1.0, np.exp(1j * np.pi / 4)]) for r in range(n, len(arrays["graph"]))}
    w[q] = np.array([U[1, 0], -U[0, 0]])  # w . U[:, 0] = 0: f0 = 0 at q's step
    x = _x(case["protocol"]["records"][0])
    prep = eng.prepare([x], w)
    assert not all(prep["unit_ok"])
    v, _ = eng.block(x, w)
    want, _ = oeng.block(x, w)
    assert rel_l2(v.cpu().numpy(), want) < 1e-5


@pytest.mark.parametrize("name", ["small", "c2"])
def test_plan_specialised_kernels_with_staged_tiles(golden, name):
    """The generated kernels with the tile staged through shared memory on load and store
    (direct_io off) give the same blocks as the default direct table I/O."""
    from dcs245_classical_sampling_b200.jit import JitPlan
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, mode="fused")
    eng.set_fused_config(variant=12, pairs=False, max_dim=13, low=4, jit=True)
    direct = [eng.block(_x(rec))[0].cpu().numpy() for rec in case["protocol"]["records"]]
    eng.fplan.jit.close()
    eng.fplan.direct_io = False
    eng.fplan.jit = JitPlan(eng.plan, eng.fplan, eng.lib)
    for rec, d in zip(case["protocol"]["records"], direct):
        v = eng.block(_x(rec))[0].cpu().numpy()
        assert rel_l2(v, arrays[f"block_{rec['sample_id']}"]) < 1e-5
        assert rel_l2(v, d) < 1e-6


def test_one_item_at_a_time_equals_batched_slices(golden):
    case, arrays = golden("small")
    a = _engine(case, arrays, np.complex128, items=1)
    b = _engine(case, arrays, np.complex128)
    assert b.items > 1
    x = _x(case["protocol"]["records"][0])
    va, _ = a.block(x)
    vb, _ = b.block(x)
    assert torch.equal(va, vb)  # slice order is kept: bitwise identical


def test_parts_sum_to_the_block(golden):
    case, arrays = golden("small")
    eng = _engine(case, arrays, np.complex128)
    x = _x(case["protocol"]["records"][1])
    full, _ = eng.block(x)
    parts = sum(eng.block(x, part=p, parts=3)[0] for p in range(3))
    assert rel_l2(parts.cpu().numpy(), full.cpu().numpy()) < 1e-14


def test_batched_prefixes_equal_single_blocks(golden):
    case, arrays = golden("small")
    eng = _engine(case, arrays, np.complex64)
    xs = [_x(r) for r in case["protocol"]["records"]]
    many = eng.blocks(xs)
    for i, x in enumerate(xs):
        one, _ = eng.block(x)
        assert rel_l2(many[i].cpu().numpy(), one.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("name", CASES)
def test_draws_match_reference(golden, name):
    from dcs245_classical_sampling_b200.sampling import draw_checked
    case, arrays = golden(name)
    for d in case["draws"]:
        v = torch.from_numpy(arrays[f"block_{d['sample_id']}"]).cuda()
        got = draw_checked(v, d["uniform"])
        assert got["A_index"] == d["A_index"]
        assert got["weights_sha256"] == d["weights_sha256"]
        assert got["amplitudes_sha256"] == d["amplitudes_sha256"]
        assert got["selected_scaled_weight"] == d["selected_scaled_weight"]
        for key in ("cdf_lower_fsum", "cdf_upper_fsum", "scaled_mass_fsum"):
            assert got[key] == pytest.approx(d[key], rel=4e-16, abs=1e-300), key
        if not got["cdf_tie"]:
            for key in ("cdf_lower_numpy", "cdf_upper_numpy"):
                assert got[key] == pytest.approx(d[key], rel=1e-12, abs=1e-300), key
        # the 53-bit grid TV depends on the last ulp of every CDF value; both are O(n 2^-53)
        n = len(arrays[f"block_{d['sample_id']}"])
        tv_got = got["finite_53bit_draw_TV_against_computed_normalized_weights"]
        tv_ref = d["finite_53bit_draw_TV_against_computed_normalized_weights"]
        assert 0 <= tv_got <= n * 2.0 ** -52 and abs(tv_got - tv_ref) <= n * 2.0 ** -53


def test_sampler_known_answers(golden):
    from dcs245_classical_sampling_b200.sampling import draw_checked
    s, _ = golden("sampler")
    for c in s["selftest"]:
        v = np.array(c["re"]) + 1j * np.array(c["im"])
        got = draw_checked(v, c["u"])
        assert got["A_index"] == c["draw"]["A_index"]
    for c in s["law"]:
        a = np.array(c["re"]) + 1j * np.array(c["im"])
        assert draw_checked(a, .381245)["A_index"] == c["A_index"]


def test_tie_path_is_numpy_exact():
    """u placed exactly on a float64 CDF boundary: the device must fall back to the exact
    sequential CDF and still return numpy's index."""
    from dcs245_classical_sampling_b200.sampling import draw_checked
    from oracle import sampler_ref
    rng = np.random.default_rng(5)
    v = rng.normal(size=1 << 12) + 1j * rng.normal(size=1 << 12)
    w = v.real * v.real + v.imag * v.imag
    cdf = np.cumsum(w) / np.cumsum(w)[-1]
    for i in (3, 1000, 4000):
        for u in (float(cdf[i]), float(np.nextafter(cdf[i], 0)), float(np.nextafter(cdf[i], 1))):
            try:
                want = sampler_ref.draw(v, u)
            except ArithmeticError:  # the reference's own fsum cross-check rejects this u
                with pytest.raises(ArithmeticError):
                    draw_checked(v, u)
                continue
            got = draw_checked(v, u)
            assert got["A_index"] == want["A_index"]
            assert got["cdf_tie"]
            assert got["cdf_lower_numpy"] == want["cdf_lower_numpy"]
            assert got["cdf_upper_numpy"] == want["cdf_upper_numpy"]


def test_draw_errors():
    from dcs245_classical_sampling_b200.sampling import draw_checked
    with pytest.raises(ArithmeticError):
        draw_checked(np.zeros(8, complex), 0.5)
    with pytest.raises(ValueError):
        draw_checked(np.array([np.nan, 1, 1, 1], complex), 0.5)
    with pytest.raises(ValueError):
        draw_checked(np.ones(6, complex), 0.5)


@pytest.mark.parametrize("mode", ["device", "plain"])
@pytest.mark.parametrize("name", CASES)
def test_half_storage_matches_oracle(golden, name, mode):
    """The half-storage tier (inplace_half_gpu.py): binary16 tables, FP64 arithmetic, rounding
    FP64 -> FP32 -> binary16 on every store, max of the stored values.  Against the oracle's
    emulation of the same executor the block agrees to FP64 rounding (a differently ordered FP64
    sum flips a binary16 rounding with probability ~2^-40 per entry); against the exact
    reference block it is within the tier's own error."""
    from oracle import block_ref
    case, arrays = golden(name)
    eng = _engine(case, arrays, np.complex64, mode=mode, storage="float16")
    assert eng.table.dtype == torch.float16
    oeng = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                  case["parity_operations"], case["open_vertices"])
    assert eng.inplace_storage == "float16-components"
    for rec in case["protocol"]["records"][: (1 if name == "c2" else None)]:
        v, meta = eng.block(_x(rec))
        assert meta["prefix_dtype"] == "complex64"
        want, _ = oeng.block(_x(rec), storage="float16")
        got = v.cpu().numpy()
        assert rel_l2(got, want) < 1e-9, rel_l2(got, want)
        assert rel_l2(got, arrays[f"block_{rec['sample_id']}"]) < 5e-3


def test_half_engine_class_matches_reference_surface(golden):
    """HalfConditionalBlockGPU: the reference class name, alloc(dtype, device), the meta
    annotations its worker and verifier read, and the same block as alloc(storage="float16")."""
    from dcs245_classical_sampling_b200.engine import HalfConditionalBlockGPU
    case, arrays = golden("small")
    eng = HalfConditionalBlockGPU(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                  case["parity_operations"], case["open_vertices"])
    eng.alloc(np.complex64, 0)
    plain = _engine(case, arrays, np.complex64, mode="device", storage="float16")
    rec = case["protocol"]["records"][0]
    v, meta = eng.block(_x(rec))
    w, _ = plain.block(_x(rec))
    assert torch.equal(v, w)
    assert meta["intermediate_storage"] == "float16 real/imaginary components"
    assert meta["prefix_dtype"] == "complex64" and meta["parts"] == 1
    with pytest.raises(ValueError):
        eng.alloc(np.complex128)


def test_empty_batch_and_repeated_prefixes(golden):
    """No prefixes give an empty (0, 2^k) batch without launching; a batch that repeats a prefix
    gives the same block twice (work items of equal inputs do not interfere)."""
    case, arrays = golden("small")
    eng = _engine(case, arrays, np.complex64, mode="device")
    empty = eng.blocks([])
    assert empty.shape == (0, 1 << len(case["open_vertices"])) and empty.dtype == torch.complex128
    x = _x(case["protocol"]["records"][0])
    two = eng.blocks([x, x]).cpu().numpy()
    one = eng.block(x)[0].cpu().numpy()
    assert np.array_equal(two[0], two[1]) and np.array_equal(two[0], one)


def test_nonfinite_table_raises(golden):
    """An infinite maximum raises ArithmeticError (inplace_gpu.py:121).  NaN entries are
    dropped by fmax exactly as in the reference kernel, so an all-NaN table reads as zero:
    the slice is skipped and the draw of the resulting zero block raises."""
    from dcs245_classical_sampling_b200.sampling import draw_checked
    case, arrays = golden("c1")
    for dtype, storage in ((np.complex64, None), (np.complex128, None), (np.complex64, "float16")):
        eng = _engine(case, arrays, dtype, storage=storage)
        with pytest.raises(ArithmeticError):
            eng.block(_x(case["protocol"]["records"][0]), w=np.array([1e300, 1e300]) if dtype == np.complex128
                      else np.array([1e30, 1e30]))
    eng = _engine(case, arrays, np.complex64)
    v, _ = eng.block(_x(case["protocol"]["records"][0]), w=np.array([np.nan, 1.0]))
    assert not torch.any(v.abs() > 0)
    with pytest.raises(ArithmeticError):
        draw_checked(v, 0.5)


def test_reference_compatible_kernel(golden):
    """dcs_inplace_step takes the reference kernel's own arguments (byte tables, host scale,
    d_max): running the reference's host loop over it reproduces the oracle environment."""
    from dcs245_classical_sampling_b200 import _lib
    from dcs245_classical_sampling_b200 import plan as P
    from oracle import block_ref
    lib = _lib.load()
    case, arrays = golden("small")
    oe = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                case["parity_operations"], case["open_vertices"])
    x = _x(case["protocol"]["records"][0])
    coef, f, yfix, flips = next(s for s in oe.slice_inputs(x) if s[0])
    want, wls, _ = block_ref.execute(oe.steps, f, yfix, oe.fut, oe.maxslots)
    for dtype, tol in ((_lib.C128, 1e-13), (_lib.C64, 1e-6)):
        E = torch.zeros(1 << oe.maxslots, dtype=torch.complex128 if dtype else torch.complex64, device="cuda")
        dmax = torch.zeros(1, dtype=torch.int64, device="cuda")
        E[0] = 1
        offset, ls, maximum = 0, 0.0, 1.0
        for st in oe.steps:
            kind, omit = P.orbit_kind(P.OrbitStep(st["v"], st["j"], st["kind"], st["active_in"], st["active_out"],
                                                   st["beta"], st["K"], st["Ka"], st["pivot"], st["pivot_a"],
                                                   st["free"]))
            slots = [p for p in st["active_in"] if p not in omit]
            T = np.zeros((max(1, (len(slots) + 7) // 8), 256), np.uint64)
            for b in range(T.shape[0]):
                for val in range(256):
                    acc = 0
                    for t in range(8):
                        i = 8 * b + t
                        if i < len(slots) and (val >> t) & 1:
                            acc ^= 1 << slots[i]
                    T[b, val] = acc
            dT = torch.from_numpy(T.reshape(-1).view(np.int64)).cuda()
            identity = int(slots == list(range(len(slots))))
            j = st["j"]
            ov = (offset >> j) & 1
            offset &= ~(1 << j)
            y = 0
            if not st["free"]:
                y = int(yfix[st["v"]])
                if y:
                    offset ^= oe.fut[j]
            f0, f1 = map(complex, f[st["v"]])
            e = math.frexp(maximum)[1]
            ls += e * math.log(2.0)
            dmax.zero_()
            _lib.check(lib.dcs_inplace_step(dtype, _lib.ptr(E), 1 << len(slots), _lib.ptr(dT), T.shape[0], identity,
                                            kind, st["K"], st["Ka"], st["pivot"], st["beta"], ov, f0.real, f0.imag,
                                            f1.real, f1.imag, y, math.ldexp(1.0, -e), _lib.ptr(dmax), 0,
                                            torch.cuda.current_stream().cuda_stream))
            bits = int(dmax.cpu().numpy()[0])
            m2 = float(np.array([bits], np.uint64).view(np.float64)[0]) if dtype else \
                float(np.array([bits & 0xffffffff], np.uint32).view(np.float32)[0])
            if m2 == 0:
                break
            maximum = math.sqrt(m2)
        term = block_ref._addr(oe.steps[-1]["active_out"]).astype(np.int64)
        got = E.cpu().numpy()[term].astype(np.complex128)
        assert rel_l2(got * math.exp(ls), want * math.exp(wls)) < tol


def test_audit_pair_matches_reference_record(golden):
    from dcs245_classical_sampling_b200.audit import audit_vector_pair, relative_l2
    s, _ = golden("sampler")
    for c in s["audit"]:
        ref = np.array(c["ref_re"]) + 1j * np.array(c["ref_im"])
        ap = np.array(c["ap_re"]) + 1j * np.array(c["ap_im"])
        got = audit_vector_pair(ref, ap, 0)
        for key in ("normalized_conditional_overlap_abs", "uncapped_overlap_witness", "reference_scaled_mass",
                    "approximate_input_mass", "loss"):
            assert got[key] == pytest.approx(c["result"][key], rel=1e-14, abs=1e-15), key
    case, arrays = golden("c2")
    want = arrays["block_0"]
    eng = _engine(case, arrays, np.complex64, mode="fused")
    v, _ = eng.block(_x(case["protocol"]["records"][0]))
    rec = audit_vector_pair(torch.from_numpy(want).cuda(), v, 0)
    assert rec["normalized_conditional_overlap_abs"] >= 0.9999
    assert relative_l2(torch.from_numpy(want).cuda(), v) < 1e-5
