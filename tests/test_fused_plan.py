"""CPU emulation of the fused coset-tile executor (same load/step/store rules as
csrc/fused.cu), checked against the oracle's one-buffer executor on the golden plans."""
import math

import numpy as np
import pytest

from conftest import rel_l2
from dcs245_classical_sampling_b200 import plan as P
from dcs245_classical_sampling_b200.engine import SliceParams
from dcs245_classical_sampling_b200.fused import build_fused_plan, group_steps
from oracle import block_ref


def _deposit(x, mask):
    out = np.zeros_like(x)
    src = 0
    for p in range(64):
        if (mask >> p) & 1:
            out |= ((x >> np.uint64(src)) & np.uint64(1)) << np.uint64(p)
            src += 1
    return out


def _neg(a, beta, ov):
    y = a & np.uint64(beta)
    par = np.zeros_like(y)
    while np.any(y):
        par ^= y & np.uint64(1)
        y >>= np.uint64(1)
    return (par.astype(np.int64) ^ ov).astype(bool)


def emulate(bp, fp, params):
    steps = bp.steps
    E = np.zeros(1 << bp.maxslots, np.complex128)
    E[0] = 1
    ls = 0.0
    m2 = 1.0
    for gi, g in enumerate(fp.groups):
        first, count, dim, low = int(g["first"]), int(g["count"]), int(g["tile_dim"]), int(g["low_bits"])
        e = math.frexp(math.sqrt(m2))[1] if m2 > 0 else 0
        ls += e * math.log(2.0)
        sc = math.ldexp(1.0, -e)
        cmask = 0
        for r in range(int(g["ncoset_runs"])):
            w = int(g["coset_runs"][r])
            cmask |= ((1 << ((w >> 16) & 255)) - 1) << ((w >> 8) & 255)
        bases = _deposit(np.arange(1 << int(g["coset_m"]), dtype=np.uint64), cmask)
        t = np.arange(1 << dim, dtype=np.uint64)
        taddr = t & np.uint64((1 << low) - 1)
        for i in range(dim - low):
            taddr ^= ((t >> np.uint64(low + i)) & np.uint64(1)) * np.uint64(int(g["basis"][i]))
        A = bases[:, None] ^ taddr[None, :]
        inm = P.slot_mask(steps[first].active_in)
        sh = np.where((A & np.uint64(~inm & (2**64 - 1))) == 0, E[A.astype(np.int64)] * sc, 0)
        for s in range(first, first + count):
            st = steps[s]
            kind, omit = P.orbit_kind(st)
            enum = P.slot_mask([p for p in st.active_in if p not in omit])
            ts = fp.tile_steps[s]
            pr = params[s]
            f0, f1 = complex(pr["f0r"], pr["f0i"]), complex(pr["f1r"], pr["f1i"])
            ov, y = int(pr["ov"]), int(pr["y"])
            rep = (A & np.uint64(~enum & (2**64 - 1))) == 0
            ti, tj = np.nonzero(rep)
            a = A[ti, tj]
            x = sh[ti, tj].copy()
            sg = lambda addr: np.where(_neg(addr, st.beta, ov), -1.0, 1.0)
            if kind == P.KIND_GROW:
                sh[ti, tj] = f0 * x
                sh[ti, tj ^ int(ts["tpiv"])] = f1 * x * sg(a)
            elif kind == P.KIND_MIX:
                td = tj ^ int(ts["tKa"]); b = sh[ti, td].copy(); d = a ^ np.uint64(st.Ka)
                sh[ti, tj] = f0 * x + f1 * sg(d) * b
                sh[ti, td] = f0 * b + f1 * sg(a) * x
            elif kind == P.KIND_DIAG:
                sh[ti, tj] = (f0 + f1 * sg(a)) * x
            elif kind == P.KIND_REPLACE:
                td = tj ^ int(ts["tK"]); b = sh[ti, td].copy(); d = a ^ np.uint64(st.K)
                sh[ti, tj] = f0 * (x + b)
                sh[ti, td] = f1 * (sg(a) * x + sg(d) * b)
            elif kind == P.KIND_FIXED:
                sh[ti, tj] = (f1 * sg(a) if y else f0) * x
            elif kind == P.KIND_FIXED_SHRINK:
                td = tj ^ int(ts["tK"]); b = sh[ti, td].copy(); d = a ^ np.uint64(st.K)
                sh[ti, tj] = f1 * (sg(a) * x + sg(d) * b) if y else f0 * (x + b)
            elif kind == P.KIND_SHRINK4:
                t1 = tj ^ int(ts["tK"]); td = tj ^ int(ts["tKa"]); td1 = td ^ int(ts["tK"])
                b, gg, h = sh[ti, t1].copy(), sh[ti, td].copy(), sh[ti, td1].copy()
                c1 = a ^ np.uint64(st.K); d = a ^ np.uint64(st.Ka); d1 = d ^ np.uint64(st.K)
                sh[ti, tj] = f0 * (x + b) + f1 * (sg(d) * gg + sg(d1) * h)
                sh[ti, td] = f0 * (gg + h) + f1 * (sg(a) * x + sg(c1) * b)
            else:
                td = tj ^ int(ts["tK"]); b = sh[ti, td].copy(); d = a ^ np.uint64(st.K)
                sh[ti, tj] = (f0 + f1 * sg(a)) * x + (f0 + f1 * sg(d)) * b
        outm = P.slot_mask(steps[first + count - 1].active_out)
        keep = (A & np.uint64(~outm & (2**64 - 1))) == 0
        E[A[keep].astype(np.int64)] = sh[keep]
        m2 = float(np.max(np.abs(sh[keep]) ** 2)) if keep.any() else 0.0
    term = _deposit(np.arange(1 << len(bp.terminal_slots), dtype=np.uint64), P.slot_mask(bp.terminal_slots))
    return E[term.astype(np.int64)], ls


@pytest.mark.parametrize("name,dims", [("c1", [(13, 4), (6, 2), (4, 0)]), ("small", [(13, 4), (8, 3), (6, 2)]),
                                       ("c2", [(13, 4)])])
def test_fused_emulation_matches_oracle(golden, name, dims):
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    sp = SliceParams(bp)
    oe = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                case["parity_operations"], case["open_vertices"])
    x = np.array([int(c) for c in case["protocol"]["records"][0]["input_data_bits"]], np.uint8)
    _, items = sp.items(x)
    slices = oe.slice_inputs(x)
    for (coef, params, xor), (ocoef, f, yfix, flips) in zip(items, [s for s in slices if s[0]]):
        assert coef == pytest.approx(ocoef)
        want, wls, off = block_ref.execute(oe.steps, f, yfix, oe.fut, oe.maxslots)
        freeflip = sum(int(flips[q]) << j for j, q in enumerate(oe.open_red))
        assert xor == (off >> oe.stop) ^ freeflip
        for max_dim, low in dims:
            fp = build_fused_plan(bp, max_dim=max_dim, low=low)
            assert sum(c for _, c in fp.spans) == len(bp.steps)
            got, gls = emulate(bp, fp, params)
            if not np.any(want):
                assert not np.any(got)  # the slice's table vanished: the reference skips it
            else:
                assert rel_l2(got * math.exp(gls), want * math.exp(wls)) < 1e-12


def test_grouping_reduces_passes(golden):
    case, arrays = golden("c64plan")
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    fp = build_fused_plan(bp)
    per_step = P.step_bytes(bp)
    fused = fp.algorithmic_bytes(bp)
    assert len(fp.spans) < len(bp.steps) / 3
    assert fused < per_step / 3
