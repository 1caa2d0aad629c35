"""CPU emulation of the fused coset-tile executor (same load/step/store rules as
csrc/fused.cu), checked against the oracle's one-buffer executor on the golden plans."""
import math

import numpy as np
import pytest

from conftest import rel_l2
from dcs245_classical_sampling_b200 import jit
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


def emulate(bp, fp, params, packed=False):
    """packed=True follows the paired-layout kernel: packed steps where tile bit 0 is free."""
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
        s = first
        while s < first + count:
            if int(g["variant"]) & 4:
                sh = _emulate_run(bp, fp, params, s, bases, sh, dim, packed=bool(int(g["variant"]) & 2))
                s += int(fp.tile_steps[s]["run_len"])
                continue
            st = steps[s]
            kind, _ = P.orbit_kind(st)
            ts = fp.tile_steps[s]
            if packed:
                if _packable(ts, kind, dim):
                    sh = _emulate_packed(st, kind, ts, params[s], bases, A, sh, dim)
                    s += 1
                    continue
            elif int(ts["pair"]) and s + 1 < first + count:
                sh = _emulate_pair(bp, fp, params, s, bases, A, sh, dim, low)
                s += 2
                continue
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
            s += 1
        outm = P.slot_mask(steps[first + count - 1].active_out)
        keep = (A & np.uint64(~outm & (2**64 - 1))) == 0
        E[A[keep].astype(np.int64)] = sh[keep]
        m2 = float(np.max(np.abs(sh[keep]) ** 2)) if keep.any() else 0.0
    term = _deposit(np.arange(1 << len(bp.terminal_slots), dtype=np.uint64), P.slot_mask(bp.terminal_slots))
    return E[term.astype(np.int64)], ls


def _par_arr(v, mask):
    y = v & np.uint64(mask)
    par = np.zeros_like(y)
    while np.any(y):
        par ^= y & np.uint64(1)
        y >>= np.uint64(1)
    return par.astype(np.int64)


def _apply2(kind, xc, xd, sc, sd, f0, f1, y):
    sg = lambda b: np.where(b, -1.0, 1.0)
    if kind == P.KIND_GROW:
        return f0 * xc, f1 * xc * sg(sc)
    if kind == P.KIND_MIX:
        return f0 * xc + f1 * sg(sd) * xd, f0 * xd + f1 * sg(sc) * xc
    if kind == P.KIND_REPLACE:
        return f0 * (xc + xd), f1 * (sg(sc) * xc + sg(sd) * xd)
    if kind == P.KIND_FIXED_SHRINK:
        return (f1 * (sg(sc) * xc + sg(sd) * xd) if y else f0 * (xc + xd)), xd
    return (f0 + f1 * sg(sc)) * xc + (f0 + f1 * sg(sd)) * xd, xd  # shrink2


def _apply1(kind, x, s, f0, f1, y):
    sg = np.where(s, -1.0, 1.0)
    if kind == P.KIND_DIAG:
        return (f0 + f1 * sg) * x
    return f1 * sg * x if y else f0 * x


def _emulate_pair(bp, fp, params, s, bases, A, sh, dim, low):
    """Mirror of csrc/fused.cu run_pair: two steps per round trip over super-orbits."""
    a, b = bp.steps[s], bp.steps[s + 1]
    ka, kb = P.orbit_kind(a)[0], P.orbit_kind(b)[0]
    ta = fp.tile_steps[s]
    pa, pb = params[s], params[s + 1]
    fa0, fa1 = complex(pa["f0r"], pa["f0i"]), complex(pa["f1r"], pa["f1i"])
    fb0, fb1 = complex(pb["f0r"], pb["f0i"]), complex(pb["f1r"], pb["f1i"])
    two = lambda k: k not in (P.KIND_DIAG, P.KIND_FIXED)
    A2, B2 = two(ka), two(kb)
    nins = int(ta["pnins"])
    o = np.arange((1 << dim) >> nins, dtype=np.int64)
    for rho in [int(v) for v in ta["pins"][:nins]]:
        o = ((o >> rho) << (rho + 1)) | (o & ((1 << rho) - 1))
    tau1, tau2 = int(ta["tau1"]), int(ta["tau2"])
    R = np.arange(len(bases))[:, None]
    t0 = np.broadcast_to(o, (len(bases), len(o)))
    t1, t2 = t0 ^ tau1, t0 ^ tau2
    t3 = t1 ^ tau2
    a0 = A[R, t0]
    # invariants: e0 is entry c of both steps
    for st, kk in ((a, ka), (b, kb)):
        role = {P.KIND_GROW: st.pivot, P.KIND_MIX: st.pivot_a}.get(kk, st.pivot if kk in (3, 5, 7) else None)
        if role is not None:
            assert not ((a0 >> np.uint64(role)) & np.uint64(1)).any()
    cs_a = np.array([bin(int(bb) & a.beta).count("1") & 1 for bb in bases], np.int64)[:, None] ^ int(pa["ov"])
    cs_b = np.array([bin(int(bb) & b.beta).count("1") & 1 for bb in bases], np.int64)[:, None] ^ int(pb["ov"])
    tba, tbb = int(fp.tile_steps[s]["tbeta"]), int(fp.tile_steps[s + 1]["tbeta"])
    sa = _par_arr(t0.astype(np.uint64), tba) ^ cs_a
    sb = _par_arr(t0.astype(np.uint64), tbb) ^ cs_b
    s1e = [int(v) for v in ta["s1e"]]
    s2e = [int(v) for v in ta["s2e"]]
    # partner signs against the physical parity
    for tt, j in ((t1, 1), (t2, 2), (t3, 3)):
        aa = A[R, tt]
        np.testing.assert_array_equal(sa ^ s1e[j], _neg(aa.reshape(-1), a.beta, int(pa["ov"])).reshape(aa.shape))
        np.testing.assert_array_equal(sb ^ s2e[j], _neg(aa.reshape(-1), b.beta, int(pb["ov"])).reshape(aa.shape))
    live_a = ((bases & np.uint64(int(ta["cskip"]))) == 0)[:, None]
    live_b = ((bases & np.uint64(int(fp.tile_steps[s + 1]["cskip"]))) == 0)[:, None]
    e0 = sh[R, t0].copy()
    e1 = sh[R, t1].copy() if A2 else None
    e2 = sh[R, t2].copy() if B2 else None
    e3 = sh[R, t3].copy() if (A2 and B2) else None
    def sel(live, new, old):
        return np.where(live, new, old)
    if A2:
        n0, n1 = _apply2(ka, e0, e1, sa, sa ^ s1e[1], fa0, fa1, int(pa["y"]))
        e0, e1 = sel(live_a, n0, e0), sel(live_a, n1, e1)
        if B2:
            if int(ta["swapB"]):
                n3, n2 = _apply2(ka, e3, e2, sa ^ s1e[3], sa ^ s1e[2], fa0, fa1, int(pa["y"]))
            else:
                n2, n3 = _apply2(ka, e2, e3, sa ^ s1e[2], sa ^ s1e[3], fa0, fa1, int(pa["y"]))
            e2, e3 = sel(live_a, n2, e2), sel(live_a, n3, e3)
    else:
        e0 = sel(live_a, _apply1(ka, e0, sa, fa0, fa1, int(pa["y"])), e0)
        if B2:
            e2 = sel(live_a, _apply1(ka, e2, sa ^ s1e[2], fa0, fa1, int(pa["y"])), e2)
    if B2:
        n0, n2 = _apply2(kb, e0, e2, sb, sb ^ s2e[2], fb0, fb1, int(pb["y"]))
        e0, e2 = sel(live_b, n0, e0), sel(live_b, n2, e2)
        if A2:
            if int(ta["swapA"]):
                n3, n1 = _apply2(kb, e3, e1, sb ^ s2e[3], sb ^ s2e[1], fb0, fb1, int(pb["y"]))
            else:
                n1, n3 = _apply2(kb, e1, e3, sb ^ s2e[1], sb ^ s2e[3], fb0, fb1, int(pb["y"]))
            e1, e3 = sel(live_b, n1, e1), sel(live_b, n3, e3)
    else:
        e0 = sel(live_b, _apply1(kb, e0, sb, fb0, fb1, int(pb["y"])), e0)
        if A2:
            e1 = sel(live_b, _apply1(kb, e1, sb ^ s2e[1], fb0, fb1, int(pb["y"])), e1)
    sh = sh.copy()
    sh[R, t0] = e0
    if A2:
        sh[R, t1] = e1
    if B2:
        sh[R, t2] = e2
    if A2 and B2:
        sh[R, t3] = e3
    return sh


def _emulate_run(bp, fp, params, s0, bases, sh, dim, packed=False):
    """Mirror of csrc/fused.cu register runs: cosets t0 + V held in registers."""
    tr = fp.tile_runs[s0]
    n, R, nins = int(tr["count"]), int(tr["r"]), int(tr["nins"])
    assert n >= 1 and int(fp.tile_steps[s0]["run_len"]) == n
    ins = [int(v) for v in tr["ins"][:nins]]
    nb = (1 << dim) >> nins
    threads = min(nb, 256)
    o = np.arange(threads, dtype=np.int64)
    for rho in ins:
        o = ((o >> rho) << (rho + 1)) | (o & ((1 << rho) - 1))
    mhi = int(tr["mhi"])
    niter = nb >> 8 if nb > 256 else 1
    tus, tu = [], 0
    for _ in range(niter):
        tus.append(tu)
        tu = ((tu | (~mhi & 0xFFFFFFFF)) + 1) & mhi
    t0 = (o[:, None] | np.array(tus, dtype=np.int64)[None, :]).reshape(-1)
    offs = fp.run_off.get(s0) if fp.run_off else None  # every run's 2^R offsets (records hold R <= 4)
    off = np.array([int(v) for v in (offs if offs is not None else tr["off"][:1 << R])], dtype=np.int64)
    idx = t0[:, None] ^ off[None, :]                      # base, local entry
    # the cosets are disjoint and cover the tile minus the run's inactive coordinates
    assert len(np.unique(idx)) == idx.size
    if packed and nins < dim and (nins == 0 or ins[0] != 0):
        # paired layout: coset pairs (t0, t0 | 1) from spread(tid << 1) and the walk over mhi
        # without its lowest bit; local entry j of lane L sits at ((t0 ^ off_j) & ~1) + (L ^ off_j & 1)
        nb2 = nb >> 1
        o2 = np.arange(min(nb2, 256), dtype=np.int64) << 1
        for rho in ins:
            o2 = ((o2 >> rho) << (rho + 1)) | (o2 & ((1 << rho) - 1))
        m2 = mhi & (mhi - 1)
        tus2, tu = [], 0
        for _ in range(nb2 >> 8 if nb2 > 256 else 1):
            tus2.append(tu)
            tu = ((tu | (~m2 & 0xFFFFFFFF)) + 1) & m2
        tp2 = (o2[:, None] | np.array(tus2, dtype=np.int64)[None, :]).reshape(-1)
        assert not (tp2 & 1).any()
        assert np.array_equal(np.sort(np.concatenate([tp2, tp2 | 1])), np.sort(t0))
        for L in (0, 1):
            pos = ((tp2[:, None] ^ off[None, :]) & ~1) + (L ^ (off[None, :] & 1))
            assert np.array_equal(pos, (tp2[:, None] | L) ^ off[None, :])
    live = ((bases & np.uint64(int(fp.tile_steps[s0]["cskip"]))) == 0)[:, None, None]
    v = sh[:, idx].copy()                                 # tile, base, local
    for s in range(s0, s0 + n):
        st = bp.steps[s]
        kind, _ = P.orbit_kind(st)
        ts = fp.tile_steps[s]
        assert int(ts["cskip"]) == int(fp.tile_steps[s0]["cskip"])
        pr = params[s]
        f0, f1 = complex(pr["f0r"], pr["f0i"]), complex(pr["f1r"], pr["f1i"])
        y = int(pr["y"])
        gK, gKa = (-1.0 if int(ts["sK"]) else 1.0), (-1.0 if int(ts["sKa"]) else 1.0)
        tb = int(ts["tbeta"])
        ptab = int(fp.step_ptab[s]) if s in fp.step_ptab else int(ts["ptab"])
        cs = np.array([bin(int(bb) & st.beta).count("1") & 1 for bb in bases], np.int64)[:, None] ^ int(pr["ov"])
        s0b = np.array([bin(int(q) & tb).count("1") & 1 for q in t0], np.int64)[None, :] ^ cs  # tile, base
        sg = lambda j: np.where(s0b ^ ((ptab >> j) & 1), -1.0, 1.0)
        k1, k2, mix = int(ts["rk1"]), int(ts["rk2"]), int(ts["rmix"])
        dead = int(ts["rdead"])
        # bases touching other roles (variant bit 6): the representative and the dead entries
        # follow parities of several local bits (runs_jit.cuh orb1/orb4, deadp)
        t1, t2, dp = fp.step_touch.get(s, (0, 0, 0))
        dmasks = [(dp >> (6 * q)) & 63 for q in range(5) if (dp >> (6 * q)) & 63]
        par = lambda x: bin(x).count("1") & 1
        # the representative's sign from the generated kernels' local functional (jit._beff), which
        # keeps the step's own bits only where a representative can have them set
        Bl = jit._beff(kind, ts, R, ptab, touched=bool(t1 or t2))
        sg = lambda j, Bl=Bl: np.where(s0b ^ par(j & Bl), -1.0, 1.0)
        e = 1 << k1
        new = v.copy()
        for j in range(1 << R):
            if j & dead or any(par(j & m) for m in dmasks):
                continue  # a removed or not yet grown slot: the kernel skips these entries
            x = v[:, :, j]
            if kind in (P.KIND_DIAG, P.KIND_FIXED):
                if kind == P.KIND_DIAG:
                    new[:, :, j] = (f0 + sg(j) * f1) * x
                else:
                    new[:, :, j] = sg(j) * f1 * x if y else f0 * x
                continue
            if kind == P.KIND_SHRINK4:
                if j & (e | (1 << k2)):
                    continue
                mK = e | ((1 << k2) if mix & 1 else 0)
                mKa = (1 << k2) | (e if mix & 2 else 0)
                c = [q for q in (j, j ^ mK, j ^ mKa, j ^ mK ^ mKa)
                     if not par(q & (e | t1)) and not par(q & ((1 << k2) | t2))]
                assert len(c) == 1
                c = c[0]
                x, b, g_, h = v[:, :, c], v[:, :, c ^ mK], v[:, :, c ^ mKa], v[:, :, c ^ mK ^ mKa]
                new[:, :, c] = f0 * (x + b) + sg(c) * gKa * f1 * (g_ + gK * h)
                new[:, :, c ^ mKa] = f0 * (g_ + h) + sg(c) * f1 * (x + gK * b)
                continue
            if j & e:
                continue
            c = j | e if par(j & t1) else j
            d = c ^ e
            x, b = v[:, :, c], v[:, :, d]
            if kind == P.KIND_GROW:
                new[:, :, c], new[:, :, d] = f0 * x, sg(c) * f1 * x
            elif kind == P.KIND_MIX:
                new[:, :, c] = f0 * x + sg(c) * gKa * f1 * b
                new[:, :, d] = f0 * b + sg(c) * f1 * x
            elif kind == P.KIND_REPLACE:
                new[:, :, c], new[:, :, d] = f0 * (x + b), sg(c) * f1 * (x + gK * b)
            elif kind == P.KIND_FIXED_SHRINK:
                new[:, :, c] = sg(c) * f1 * (x + gK * b) if y else f0 * (x + b)
            else:
                new[:, :, c] = f0 * (x + b) + sg(c) * f1 * (x + gK * b)
        v = np.where(live, new, v)
    out = sh.copy()
    out[:, idx] = v
    return out


def _packable(ts, kind, dim):
    nins = int(ts["nins"])
    return nins < dim and (nins == 0 or int(ts["ins"][0]) != 0) and not (kind == P.KIND_GROW and int(ts["tpiv"]) & 1)


def _emulate_packed(st, kind, ts, pr, bases, A, sh, dim):
    """Mirror of csrc/fused.cu run_packed: representative pairs (t, t + 1) in two lanes."""
    nins = int(ts["nins"])
    ins = [int(v) for v in ts["ins"][:nins]]
    nrep = (1 << dim) >> (nins + 1)
    threads = min(nrep, 256)
    o = np.arange(threads, dtype=np.int64) << 1
    for rho in ins:
        o = ((o >> rho) << (rho + 1)) | (o & ((1 << rho) - 1))
    tp = o
    mhi = int(ts["mhi"]) & (int(ts["mhi"]) - 1)
    niter = nrep >> 8 if nrep > 256 else 1
    tus, tu = [], 0
    for _ in range(niter):
        tus.append(tu)
        tu = ((tu | (~mhi & 0xFFFFFFFF)) + 1) & mhi
    tus = np.array(tus, dtype=np.int64)
    t = (tp[:, None] | tus[None, :]).reshape(-1)
    # the pairs cover every representative (zero at the inserted bits) exactly once
    insmask = sum(1 << b for b in ins)
    reps = np.flatnonzero((np.arange(1 << dim) & insmask) == 0)
    assert np.array_equal(np.sort(np.concatenate([t, t + 1])), reps)
    assert not (t & 1).any()
    tb = int(ts["tbeta"])
    f0, f1 = complex(pr["f0r"], pr["f0i"]), complex(pr["f1r"], pr["f1i"])
    y = int(pr["y"])
    gK, gKa = (-1.0 if int(ts["sK"]) else 1.0), (-1.0 if int(ts["sKa"]) else 1.0)
    R = np.arange(len(bases))[:, None]
    live = ((bases & np.uint64(int(ts["cskip"]))) == 0)[:, None]
    cs = np.array([bin(int(bb) & st.beta).count("1") & 1 for bb in bases], np.int64)[:, None] ^ int(pr["ov"])
    # lane signs as the kernel forms them: parity over tp, then over tu, lane 1 flipped by tbeta bit 0
    par = lambda v: np.array([bin(int(q) & tb).count("1") & 1 for q in v], np.int64)
    s0 = (np.repeat(par(tp), niter)[None, :] ^ np.tile(par(tus), threads)[None, :]) ^ cs
    S = np.stack([np.where(s0, -1.0, 1.0), np.where(s0 ^ (tb & 1), -1.0, 1.0)])  # lane, tile, rep

    def load(off, sw):
        base = t ^ off
        lo, hi = sh[R, base], sh[R, base + 1]
        return np.stack([hi, lo]) if sw else np.stack([lo, hi])

    def store(out, off, sw, val):
        base = t ^ off
        v = val[::-1] if sw else val
        out[R, base] = np.where(live, v[0], out[R, base])
        out[R, base + 1] = np.where(live, v[1], out[R, base + 1])

    tK, tKa, tpiv = int(ts["tK"]), int(ts["tKa"]), int(ts["tpiv"])
    x = load(0, False)
    out = sh.copy()
    touched = [t >> 1]
    if kind == P.KIND_GROW:
        store(out, 0, False, f0 * x)
        store(out, tpiv & ~1, False, S * (f1 * x))
        touched.append((t ^ (tpiv & ~1)) >> 1)
    elif kind == P.KIND_MIX:
        sw = tKa & 1
        bs = S * load(tKa & ~1, sw)
        store(out, 0, False, f0 * x + gKa * f1 * bs)
        store(out, tKa & ~1, sw, S * (f0 * bs + f1 * x))
        touched.append((t ^ (tKa & ~1)) >> 1)
    elif kind == P.KIND_DIAG:
        store(out, 0, False, (f0 + S * f1) * x)
    elif kind == P.KIND_REPLACE:
        sw = tK & 1
        b = load(tK & ~1, sw)
        store(out, 0, False, f0 * (x + b))
        store(out, tK & ~1, sw, S * (f1 * (x + gK * b)))
        touched.append((t ^ (tK & ~1)) >> 1)
    elif kind == P.KIND_FIXED:
        store(out, 0, False, S * (f1 * x) if y else f0 * x)
    elif kind == P.KIND_FIXED_SHRINK:
        b = load(tK & ~1, tK & 1)
        store(out, 0, False, S * (f1 * (x + gK * b)) if y else f0 * (x + b))
        touched.append((t ^ (tK & ~1)) >> 1)
    elif kind == P.KIND_SHRINK4:
        sw1, sw2 = tK & 1, tKa & 1
        b, g = load(tK & ~1, sw1), load(tKa & ~1, sw2)
        h = load((tK ^ tKa) & ~1, sw1 ^ sw2)
        Sd = S * gKa
        store(out, 0, False, f0 * (x + b) + Sd * (f1 * (g + gK * h)))
        store(out, tKa & ~1, sw2, f0 * (g + h) + S * (f1 * (x + gK * b)))
        touched += [(t ^ (tK & ~1)) >> 1, (t ^ (tKa & ~1)) >> 1, (t ^ ((tK ^ tKa) & ~1)) >> 1]
    else:
        b = load(tK & ~1, tK & 1)
        store(out, 0, False, f0 * (x + b) + S * (f1 * (x + gK * b)))
        touched.append((t ^ (tK & ~1)) >> 1)
    # the 16-byte pairs a step touches are disjoint between representative pairs
    allp = np.concatenate(touched)
    assert len(np.unique(allp)) == len(allp)
    return out


ALL_MODES = ("plain", "pairs", "packed", "runs3", "runs4", "pruns3")


@pytest.mark.parametrize("name,dims,modes", [("c1", [(13, 4), (6, 2), (4, 0)], ALL_MODES),
                                             ("small", [(13, 4), (8, 3), (6, 2)], ALL_MODES),
                                             ("c2", [(13, 4)], ("runs4",))])  # 2^22 tables: the tuned mode
def test_fused_emulation_matches_oracle(golden, name, dims, modes):
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
        for (max_dim, low), mode in [(d, m) for d in dims for m in modes]:
            variant = {"runs3": 4, "runs4": 12, "pruns3": 6}.get(mode, 0)
            fp = build_fused_plan(bp, max_dim=max_dim, low=low, pairs=mode == "pairs", variant=variant)
            assert sum(c for _, c in fp.spans) == len(bp.steps)
            assert (int(fp.tile_steps["pair"].sum()) > 0) == (mode == "pairs")
            got, gls = emulate(bp, fp, params, packed=mode == "packed")
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


@pytest.mark.parametrize("name", ["c1", "small"])
def test_min_bytes_grouping_emulation_matches_oracle(golden, name):
    """Groups chosen by the dynamic program (fewest table bytes) obey the greedy rules and give
    the oracle's environment through the register-run emulation."""
    from dcs245_classical_sampling_b200.fused import _feasible_ends, group_steps_min_bytes
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    spans = group_steps_min_bytes(bp.steps, 13, 3)
    for first, count in spans:
        assert first + count in _feasible_ends(bp.steps, first, 13, 3, 24, 1)
    sp = SliceParams(bp)
    oe = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                case["parity_operations"], case["open_vertices"])
    x = np.array([int(c) for c in case["protocol"]["records"][0]["input_data_bits"]], np.uint8)
    _, items = sp.items(x)
    slices = [s for s in oe.slice_inputs(x) if s[0]]
    for (coef, params, xor), (ocoef, f, yfix, flips) in zip(items, slices):
        want, wls, _ = block_ref.execute(oe.steps, f, yfix, oe.fut, oe.maxslots)
        fp = build_fused_plan(bp, max_dim=13, low=3, variant=12, grouping="bytes")
        assert fp.spans == spans
        got, gls = emulate(bp, fp, params)
        if np.any(want):
            assert rel_l2(got * math.exp(gls), want * math.exp(wls)) < 1e-12


@pytest.mark.parametrize("name", ["c1", "small", "c2"])
def test_touching_run_bases_emulation_matches_oracle(golden, name):
    """Variant bit 6: register runs whose basis vectors may have other vectors' role coordinates
    (invertible at the roles) take fewer runs, and, with the representative and the dead entries
    found by parities of several local bits, give the oracle's environment."""
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    sp = SliceParams(bp)
    oe = block_ref.OracleEngine(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                case["parity_operations"], case["open_vertices"])
    x = np.array([int(c) for c in case["protocol"]["records"][0]["input_data_bits"]], np.uint8)
    _, items = sp.items(x)
    slices = [s for s in oe.slice_inputs(x) if s[0]]
    plain = build_fused_plan(bp, max_dim=13, low=3, variant=12, grouping="bytes")
    fp = build_fused_plan(bp, max_dim=13, low=3, variant=76, grouping="bytes")
    fp5 = build_fused_plan(bp, max_dim=13, low=3, variant=92, grouping="bytes")  # dimension 5
    assert fp.spans == plain.spans == fp5.spans
    def runs(f, gi):
        g = f.groups[gi]
        first, count = int(g["first"]), int(g["count"])
        return int((f.tile_steps["run_len"][first:first + count] > 0).sum()) if int(g["variant"]) & 4 else None
    both = [gi for gi in range(len(fp.groups)) if runs(fp, gi) and runs(plain, gi)]
    assert all(runs(fp, gi) <= runs(plain, gi) for gi in both)
    if name != "c1":
        assert any(t1 or t2 for t1, t2, _ in fp.step_touch.values())
        assert any(runs(fp, gi) < runs(plain, gi) for gi in both)
    for (coef, params, xor), (ocoef, f, yfix, flips) in list(zip(items, slices))[:2]:
        want, wls, _ = block_ref.execute(oe.steps, f, yfix, oe.fut, oe.maxslots)
        for f in (fp, fp5):
            got, gls = emulate(bp, f, params)
            if np.any(want):
                assert rel_l2(got * math.exp(gls), want * math.exp(wls)) < 1e-12
    with pytest.raises(ValueError):
        fp.launch_library(None, 0, 0, 0, 1, 0, 0, None)


def test_min_bytes_grouping_moves_fewer_bytes(golden):
    case, arrays = golden("c64plan")
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    greedy = build_fused_plan(bp, max_dim=13, low=4)
    dp = build_fused_plan(bp, max_dim=13, low=4, grouping="bytes", group_cost=0)
    assert dp.algorithmic_bytes(bp) <= greedy.algorithmic_bytes(bp)
    assert dp.algorithmic_bytes(bp) < 0.8 * greedy.algorithmic_bytes(bp)  # 150.5 vs 199.5 GiB
    with pytest.raises(ValueError):
        build_fused_plan(bp, grouping="other")
