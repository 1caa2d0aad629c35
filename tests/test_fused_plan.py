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
            kind, _ = P.orbit_kind(st)
            ts = fp.tile_steps[s]
            pr = params[s]
            f0, f1 = complex(pr["f0r"], pr["f0i"]), complex(pr["f1r"], pr["f1i"])
            ov, y = int(pr["ov"]), int(pr["y"])
            tK, tKa, tpiv, tb = int(ts["tK"]), int(ts["tKa"]), int(ts["tpiv"]), int(ts["tbeta"])
            nins = int(ts["nins"])
            o = np.arange((1 << dim) >> nins, dtype=np.int64)
            for rho in [int(v) for v in ts["ins"][:nins]]:
                o = ((o >> rho) << (rho + 1)) | (o & ((1 << rho) - 1))
            t = np.broadcast_to(o, (len(bases), len(o))).copy()
            a = A[np.arange(len(bases))[:, None], t]
            bit = lambda q: ((a >> np.uint64(q)) & np.uint64(1)).astype(bool)
            # every enumerated representative is the reference's c (zero role slots) and active,
            # except in tiles skipped through an inactive coset slot
            live = (bases & np.uint64(int(ts["cskip"]))) == 0
            t, a = t[live], a[live]
            bit = lambda q: ((a >> np.uint64(q)) & np.uint64(1)).astype(bool)
            if kind in (0, 1, 3, 5, 6, 7):
                assert not bit(int(ts["rb1"])).any()
            if kind == 6:
                assert not bit(int(ts["rb2"])).any()
            inm = P.slot_mask(st.active_in)
            assert ((a & np.uint64(~inm & (2**64 - 1))) == 0).all()
            ti = np.repeat(np.flatnonzero(live), t.shape[1])
            tj = t.reshape(-1)
            cs = np.array([bin(int(bb) & st.beta).count("1") & 1 for bb in bases], np.int64)[ti] ^ ov
            pc = np.array([bin(int(v) & tb).count("1") & 1 for v in tj], np.int64)
            sc = pc ^ cs
            assert np.array_equal(sc, _neg(a.reshape(-1), st.beta, ov).astype(np.int64))
            sgn = lambda bits: np.where(bits, -1.0, 1.0)
            x = sh[ti, tj].copy()
            sK, sKa = int(ts["sK"]), int(ts["sKa"])
            if kind == P.KIND_GROW:
                sh[ti, tj] = f0 * x
                sh[ti, tj ^ tpiv] = f1 * x * sgn(sc)
            elif kind == P.KIND_MIX:
                td = tj ^ tKa; b = sh[ti, td].copy()
                sh[ti, tj] = f0 * x + f1 * sgn(sc ^ sKa) * b
                sh[ti, td] = f0 * b + f1 * sgn(sc) * x
            elif kind == P.KIND_DIAG:
                sh[ti, tj] = (f0 + f1 * sgn(sc)) * x
            elif kind == P.KIND_REPLACE:
                td = tj ^ tK; b = sh[ti, td].copy()
                sh[ti, tj] = f0 * (x + b)
                sh[ti, td] = f1 * (sgn(sc) * x + sgn(sc ^ sK) * b)
            elif kind == P.KIND_FIXED:
                sh[ti, tj] = (f1 * sgn(sc) if y else f0) * x
            elif kind == P.KIND_FIXED_SHRINK:
                td = tj ^ tK; b = sh[ti, td].copy()
                sh[ti, tj] = f1 * (sgn(sc) * x + sgn(sc ^ sK) * b) if y else f0 * (x + b)
            elif kind == P.KIND_SHRINK4:
                t1 = tj ^ tK; td = tj ^ tKa; td1 = td ^ tK
                b, gg, h = sh[ti, t1].copy(), sh[ti, td].copy(), sh[ti, td1].copy()
                sd = sc ^ sKa
                sh[ti, tj] = f0 * (x + b) + f1 * (sgn(sd) * gg + sgn(sd ^ sK) * h)
                sh[ti, td] = f0 * (gg + h) + f1 * (sgn(sc) * x + sgn(sc ^ sK) * b)
            else:
                td = tj ^ tK; b = sh[ti, td].copy()
                sh[ti, tj] = (f0 + f1 * sgn(sc)) * x + (f0 + f1 * sgn(sc ^ sK)) * b
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
