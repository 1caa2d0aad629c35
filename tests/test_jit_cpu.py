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


@pytest.mark.parametrize("name", ["small", "c2"])
def test_fp64_and_staged_kernels_compile(golden, name):
    """The complex128 (FP64) form and the staged-first-run form of the generated kernels compile;
    staging changes only shared memory (per-group sizes from group_smem), and a per-group
    configuration reaches every group's source."""
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    lib = _lib.load()
    fp64 = build_fused_plan(bp, max_dim=12, low=3, variant=12, grouping="bytes", fp64=True)
    for src, _ in jit.plan_sources(bp, fp64, minb=2, parts=1):
        assert "#define DCS_JIT_FP64 1" in src
        assert jit.compile_source(lib, src)[:4] == b"\x7fELF"
    fp = build_fused_plan(bp, max_dim=13, low=3, variant=12, grouping="bytes")
    staged = [gi for gi in range(len(fp.groups)) if jit.prefetch_layout(fp, gi, kb=16)]
    assert staged
    for gi in staged:
        assert jit.group_smem(fp, gi, kb=16) > jit.group_smem(fp, gi, kb=0) - 8 * (1 << 13)
    cfg = {gi: (2, 16) if gi in staged else (3, 0) for gi in range(len(fp.groups))}
    units = jit.plan_sources(bp, fp, parts=1, group_cfg=cfg)
    src = units[0][0]
    assert src.count("cp_async_wait_all") == len(staged)
    assert jit.compile_source(lib, src)[:4] == b"\x7fELF"
    # a third entry sets the group's CTA size: one translation unit per thread count
    cfg = {gi: (3, 8, 128) if gi in staged else (3, 0) for gi in range(len(fp.groups))}
    units = jit.plan_sources(bp, fp, parts=1, group_cfg=cfg)
    assert len(units) == (2 if len(staged) < len(fp.groups) else 1)
    for src, gis in units:
        nt = 128 if set(gis) <= set(staged) else 256
        assert src.startswith(f"#define DCS_JIT_THREADS {nt}\n") and f"__launch_bounds__({nt}, 3)" in src
        assert jit.compile_source(lib, src)[:4] == b"\x7fELF"


@pytest.mark.parametrize("name", ["small", "c2"])
def test_dimension5_runs_plan_and_compile(golden, name):
    """Variant bit 4: register runs of dimension 5 (32 local offsets per run, kept beside the
    library's 16-entry records), falling back to dimension 4 per group; the kernels compile, and
    the library refuses such plans."""
    from dcs245_classical_sampling_b200.fused import run_dim
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    fp = build_fused_plan(bp, max_dim=13, low=3, variant=28, grouping="bytes")
    dims = [run_dim(int(v)) for v in fp.groups["variant"] if int(v) & 4]
    assert 5 in dims
    for gi, g in enumerate(fp.groups):
        if int(g["variant"]) & 4:
            for s, n in jit._group_runs(fp, gi):
                assert len(fp.run_off[int(g["first"]) + s]) == 1 << run_dim(int(g["variant"]))
    one = build_fused_plan(bp, max_dim=13, low=3, variant=12, grouping="bytes", group_variant={1: 28})
    assert all(run_dim(int(v)) <= 4 for gi, v in enumerate(one.groups["variant"]) if gi != 1)
    lib = _lib.load()
    for src, _ in jit.plan_sources(bp, fp, minb=2, parts=1):
        assert jit.compile_source(lib, src)[:4] == b"\x7fELF"
    with pytest.raises(ValueError):
        fp.launch_library(lib, 0, 0, 0, 1, 0, 0, None)


def test_packed_form_compiles(golden):
    """The packed FP32x2 form (variant bit 1) of the groups whose runs leave tile bit 0 free."""
    case, arrays = golden("c2")
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    fp = build_fused_plan(bp, max_dim=13, low=3, variant=14, grouping="bytes")
    packed = [gi for gi in range(len(fp.groups)) if jit.packable(fp, gi)]
    assert packed
    lib = _lib.load()
    for src, _ in jit.plan_sources(bp, fp, parts=1):
        assert "jit::pbody" in src
        assert jit.compile_source(lib, src)[:4] == b"\x7fELF"


@pytest.mark.parametrize("name", ["small", "c2"])
def test_touching_run_bases_compile_and_pair_only_even_offsets(golden, name):
    """Variant bit 6 kernels compile; a run whose basis touches tile bit 0 from another vector
    (some entries with the pair bit clear at odd offsets) moves single entries, never a 16-byte
    word at an odd entry."""
    from dcs245_classical_sampling_b200.fused import run_dim
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    lib = _lib.load()
    odd = 0
    for variant in (76, 92):
        fp = build_fused_plan(bp, max_dim=13, low=3, variant=variant, grouping="bytes", prefetch_kb=16)
        for gi, g in enumerate(fp.groups):
            if not int(g["variant"]) & 4:
                continue
            R = run_dim(int(g["variant"]))
            for s, _ in jit._group_runs(fp, gi):
                offs = fp.run_off[int(g["first"]) + s]
                k0 = jit.pair_bit(offs, R)
                raw = next((k for k in range(R) if int(offs[1 << k]) == 1), None)
                odd += raw is not None and k0 is None
                if k0 is not None:
                    assert all(int(offs[j]) % 2 == 0 for j in range(1 << R) if not (j >> k0) & 1)
        for src, _ in jit.plan_sources(bp, fp, minb=2, parts=1):
            assert jit.compile_source(lib, src)[:4] == b"\x7fELF"
    assert odd  # the case the guard exists for


@pytest.mark.parametrize("name", ["small", "c2"])
@pytest.mark.parametrize("kb", [0, 16])
def test_split_barrier_between_tiles_structure(golden, name, kb):
    """Every generated kernel with a tile buffer arrives once per thread per tile on the split
    barrier (after the last run's buffer loads; threads without a coset in that run and skipped
    tiles at once) and waits once, before the first run's buffer writes; no kernel has a barrier
    at the tile's start, and one-run kernels have none in the tile loop."""
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    fp = build_fused_plan(bp, max_dim=13, low=3, variant=28, grouping="bytes", prefetch_kb=kb)
    seen = 0
    for gi in range(len(fp.groups)):
        src = jit.group_source(bp, fp, gi, 2, 256, kb)
        if src is None:
            continue
        loop = src[src.index("for (uint64_t tile"):src.index("jit::block_max")]
        nruns = len(jit._group_runs(fp, gi))
        assert "sign_bits<COUNT>(g" not in loop or "warp_sign_bits" in loop
        if jit.uses_tile_buffer(fp, gi):
            seen += 1
            assert loop.count("jit::mbar_arrive(&tile_bar)") == 3
            assert loop.count("jit::mbar_wait(&tile_bar") == 1
            assert loop.count("__syncthreads();") == nruns - 1  # between runs only
            assert loop.index("jit::mbar_wait") < loop.index("__syncthreads();")
        else:
            assert "__syncthreads" not in loop and "mbar_" not in loop
    assert seen
