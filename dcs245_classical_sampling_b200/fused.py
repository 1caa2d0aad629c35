"""Fused plan: several vertex steps per pass over the table, staged in shared memory.

Every vertex step updates disjoint orbits {c, c^K, c^Ka, c^Ka^K} or {c, c|pivot}.  For a run
of consecutive steps, let W be the GF(2) span of all their orbit vectors (K, Ka, grow pivot)
plus the unit vectors of the lowest table slots (so that each tile row is a contiguous,
aligned run of 2^low entries in HBM).  The cosets base ^ W partition the table and are closed
under every orbit map of those steps, so each coset ("tile", 2^dim entries) can be loaded into
shared memory once, pushed through all the steps, and written back once: HBM traffic drops
from one read+write per step to one per group.

Tile coordinates: W gets a reduced echelon basis — the low unit vectors e_0..e_{l-1}, then
vectors w_i with distinct top bits p_i and no other basis vector touching p_i or a low bit.
A vector v of W has coordinate bit(v, i) on e_i and bit(v, p_i) on w_i.  Coset bases are
the table addresses that are zero on every pivot and low bit and lie in the group's slot
universe U.  Entries are loaded only if active before the group and stored only if active
after it; everything else inside a tile is written by a grow before any read (the grow
pivot is in W), so the algorithmic bytes are 2^|in(first)| + 2^|out(last)| entries.

The grouping is greedy: extend while dim W <= max_dim, |U| <= (largest rank in the group)
+ max_extra and the group has at most max_steps steps (bounding the growth of un-renormalised
values inside a pass).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .engine import device_steps
from .plan import KIND_GROW, deposit_runs, orbit_kind, slot_mask

MAX_GROUP_STEPS = 24
MAX_BASIS = 16


def _orbit_vectors(st):
    kind, _ = orbit_kind(st)
    if kind == KIND_GROW:
        return [1 << st.pivot]
    vecs = []
    if st.K and kind in (3, 5, 6, 7):
        vecs.append(st.K)
    if st.Ka and kind in (1, 6):
        vecs.append(st.Ka)
    return vecs


def _low_bits(U, limit):
    l = 0
    while l < limit and (U >> l) & 1:
        l += 1
    return l


def _reduced_basis(vectors, low):
    """Reduced echelon basis (pivot = top bit) of span(vectors) with the low bits cleared."""
    lowmask = (1 << low) - 1
    piv = {}
    for v in vectors:
        v &= ~lowmask
        while v:
            t = v.bit_length() - 1
            if t in piv:
                v ^= piv[t]
            else:
                piv[t] = v
                break
    # full reduction: clear every pivot bit from the other vectors
    keys = sorted(piv)
    for t in keys:
        for o in keys:
            if o != t and (piv[o] >> t) & 1:
                piv[o] ^= piv[t]
    return [piv[t] for t in keys], keys


def _dim(vectors, low):
    return low + len(_reduced_basis(vectors, low)[0])


@dataclass
class FusedPlan:
    groups: np.ndarray
    tile_steps: np.ndarray
    dsteps: np.ndarray
    tile_runs: np.ndarray = None
    jit: object = None  # jit.JitPlan: plan-specialised group kernels (loaded), or None
    # register-run plans: with pairs=True the generated kernels take two cosets per iteration
    coset_pairs: bool = False
    # generated kernels: first and last run of a tile read and write the table directly
    direct_io: bool = True
    # complex128 table, FP64 arithmetic (generated kernels only: the audit recontraction)
    fp64: bool = False
    # generated kernels: KiB of shared memory per CTA for staging the next tile's first-run
    # entries with asynchronous copies (0: the first run loads from the table; jit.prefetch_layout)
    prefetch_kb: int = 0
    # per run (first step): the 2^R local offsets; per step: parity table of those offsets
    run_off: dict = field(default_factory=dict)
    step_ptab: dict = field(default_factory=dict)
    # variant bit 6 (generated kernels only): per step of a run whose basis touches other roles,
    # (T1, T2, packed dead parity masks) (_plan_runs)
    step_touch: dict = field(default_factory=dict)
    spans: list = field(default_factory=list)      # (first, count) per group
    universe: list = field(default_factory=list)   # |U| per group
    tiles: list = field(default_factory=list)      # tile count per group
    dims: list = field(default_factory=list)

    def launch(self, lib, table, params, g0, ng, maxbits, scale, stream):
        """Run groups [g0, g0 + ng) (device pointers as ints); returns the library status."""
        if self.jit is not None:
            return self.jit.launch(table, params, g0, ng, maxbits, scale, stream)
        return self.launch_library(lib, table, params, g0, ng, maxbits, scale, stream)

    def launch_library(self, lib, table, params, g0, ng, maxbits, scale, stream):
        """The library kernels (register runs where the groups have them)."""
        if self.fp64:
            raise ValueError("the library's fused kernels store complex64 tables")
        if any(int(v) & 16 for v in self.groups["variant"]):
            raise ValueError("register runs of dimension 5 run in the plan-specialised kernels only")
        if any(int(v) & 64 for v in self.groups["variant"]):
            raise ValueError("register runs with touching bases run in the plan-specialised kernels only")
        if self.tile_runs is not None:
            return lib.dcs_fused_runs(table, self.dsteps.ctypes.data, len(self.dsteps), self.groups.ctypes.data,
                                      len(self.groups), self.tile_steps.ctypes.data, self.tile_runs.ctypes.data,
                                      params, g0, ng, maxbits, scale, stream)
        return lib.dcs_fused_groups(table, self.dsteps.ctypes.data, len(self.dsteps), self.groups.ctypes.data,
                                    len(self.groups), self.tile_steps.ctypes.data, params, g0, ng, maxbits, scale,
                                    stream)

    def algorithmic_bytes(self, plan, elem=None):
        elem = elem or (16 if self.fp64 else 8)
        tot = 0
        for first, count in self.spans:
            tot += ((1 << len(plan.steps[first].active_in)) + (1 << len(plan.steps[first + count - 1].active_out))) * elem
        return tot


def group_steps(steps, max_dim=13, low=4, max_steps=MAX_GROUP_STEPS, max_extra=1):
    """Greedy grouping -> list of (first, count)."""
    spans = []
    j = 0
    S = len(steps)
    while j < S:
        vecs, U, rank = [], 0, 0
        count = 0
        while j + count < S and count < max_steps:
            st = steps[j + count]
            U2 = U | slot_mask(st.active_in) | slot_mask(st.active_out) | (
                (1 << st.pivot) if orbit_kind(st)[0] == KIND_GROW else 0)
            r2 = max(rank, len(st.active_in), len(st.active_out))
            v2 = vecs + _orbit_vectors(st)
            l2 = _low_bits(U2, low)
            if count and (_dim(v2, l2) > max_dim or bin(U2).count("1") > r2 + max_extra):
                break
            vecs, U, rank = v2, U2, r2
            count += 1
        spans.append((j, count))
        j += count
    return spans


def _feasible_ends(steps, i, max_dim, low, max_steps, max_extra):
    """Ends j of the groups [i, j) that group_steps' rules allow (span of the orbit vectors and
    low bits <= max_dim, at most max_steps steps, slot universe <= rank + max_extra)."""
    vecs, U, rank = [], 0, 0
    ends = []
    count = 0
    S = len(steps)
    while i + count < S and count < max_steps:
        st = steps[i + count]
        U2 = U | slot_mask(st.active_in) | slot_mask(st.active_out) | (
            (1 << st.pivot) if orbit_kind(st)[0] == KIND_GROW else 0)
        r2 = max(rank, len(st.active_in), len(st.active_out))
        v2 = vecs + _orbit_vectors(st)
        l2 = _low_bits(U2, low)
        if count and (_dim(v2, l2) > max_dim or bin(U2).count("1") > r2 + max_extra):
            break
        vecs, U, rank = v2, U2, r2
        count += 1
        ends.append(i + count)
    return ends


def group_steps_min_bytes(steps, max_dim=13, low=4, max_steps=MAX_GROUP_STEPS, max_extra=1, per_group=1 << 30):
    """Grouping with the fewest table bytes: the groups obey group_steps' rules, and a dynamic
    program over the group boundaries minimises sum (2^|in_first| + 2^|out_last|) x 8 B plus
    `per_group` bytes for each group (launch and per-tile costs).  Boundaries land where the
    table is small instead of where the greedy span fills up."""
    S = len(steps)
    inf = float("inf")
    best = [inf] * (S + 1)
    prev = [0] * (S + 1)
    best[0] = 0.0
    for i in range(S):
        if best[i] == inf:
            continue
        lo_in = 1 << len(steps[i].active_in)
        for j in _feasible_ends(steps, i, max_dim, low, max_steps, max_extra):
            c = best[i] + ((lo_in + (1 << len(steps[j - 1].active_out))) * 8 + per_group)
            if c < best[j]:
                best[j], prev[j] = c, i
    spans = []
    j = S
    while j:
        i = prev[j]
        spans.append((i, j - i))
        j = i
    return spans[::-1]


PAIR_KINDS = (0, 1, 2, 3, 4, 5, 7)  # every kind but the four-entry shrink


def _tau(kind, ts):
    """Tile-coordinate orbit vector of a step (0 for one-entry kinds)."""
    if kind == KIND_GROW:
        return int(ts["tpiv"])
    if kind == 1:
        return int(ts["tKa"])
    if kind in (3, 5, 7):
        return int(ts["tK"])
    return 0


def _role_slot(st, kind):
    if kind == KIND_GROW:
        return st.pivot
    if kind == 1:
        return st.pivot_a
    if kind in (3, 5, 7):
        return st.pivot
    return None


def _pair_steps(steps, first, count, tsteps, dim, tilepos_of, tbit, U):
    """Mark pairs of consecutive steps that can share one shared-memory round trip."""
    par = lambda v: bin(v).count("1") & 1
    s = first
    while s + 1 < first + count:
        a, b = steps[s], steps[s + 1]
        ka, kb = orbit_kind(a)[0], orbit_kind(b)[0]
        ta, tb = tsteps[s], tsteps[s + 1]
        tau1, tau2 = _tau(ka, ta), _tau(kb, tb)
        ra, rb = _role_slot(a, ka), _role_slot(b, kb)
        ok = ka in PAIR_KINDS and kb in PAIR_KINDS and not (tau1 and tau2 and (tau1 == tau2))
        ok = ok and not (ra is not None and rb is not None and ra == rb)
        if not ok:
            s += 1
            continue
        # zero bits: both role slots, and slots inactive at both steps (inactive at the first
        # step and not grown by it stay inactive at the second)
        ins = set()
        if ra is not None:
            ins.add(tbit(ra))
        if rb is not None:
            ins.add(tbit(rb))
        ina, inb = slot_mask(a.active_in), slot_mask(b.active_in)
        for q in range(64):
            if (U >> q) & 1 and not (ina >> q) & 1 and not (inb >> q) & 1 and q != ra and q != rb and tilepos_of(q):
                ins.add(tbit(q))
        ins = sorted(ins)
        if len(ins) > 16 or len(ins) > dim:
            s += 1
            continue
        t1, t2 = int(ta["tbeta"]), int(tb["tbeta"])
        offs = [0, tau1, tau2, tau1 ^ tau2]
        ta["pair"] = 1
        ta["pnins"] = len(ins)
        for i, bit in enumerate(ins):
            ta["pins"][i] = bit
        free = [bb for bb in range(dim) if bb not in ins]
        ta["pmhi"] = sum(1 << bb for bb in free[8:])
        ta["tau1"], ta["tau2"] = tau1, tau2
        # roles: entry t has zero at both role coordinates; in (t^tau2, t^tau1^tau2) step 1's entry c
        # is the one whose role coordinate is zero, i.e. the second one when tau2 has that bit
        ta["swapB"] = (tau2 >> tbit(ra)) & 1 if ra is not None else 0
        ta["swapA"] = (tau1 >> tbit(rb)) & 1 if rb is not None else 0
        for j, o in enumerate(offs):
            ta["s1e"][j] = par(o & t1)
            ta["s2e"][j] = par(o & t2)
        s += 2


def _rank(vecs):
    piv = {}
    for v in vecs:
        while v:
            t = v.bit_length() - 1
            if t in piv:
                v ^= piv[t]
            else:
                piv[t] = v
                break
    return len(piv)


def _run_vectors(st, kind, ts, tbit):
    """(vector, role coordinate) pairs of a step in tile coordinates, and the shrink4 mixing bits.

    A four-entry shrink gets the reduced pair (b1, b2) of span{K, Ka} with b1 one at K's role and
    zero at Ka's, b2 the other way round; K = b1 (+ b2 if rmix bit 0), Ka = b2 (+ b1 if bit 1)."""
    if kind == KIND_GROW:
        return [(int(ts["tpiv"]), tbit(st.pivot))], 0
    if kind == 1:
        return [(int(ts["tKa"]), tbit(st.pivot_a))], 0
    if kind in (3, 5, 7):
        return [(int(ts["tK"]), tbit(st.pivot))], 0
    if kind == 6:
        tK, tKa = int(ts["tK"]), int(ts["tKa"])
        p, pa = tbit(st.pivot), tbit(st.pivot_a)
        a, b = (tK >> pa) & 1, (tKa >> p) & 1
        if a and b:
            return None, 0
        return [(tK ^ tKa if a else tK, p), (tKa ^ tK if b else tKa, pa)], a | (b << 1)
    return [], 0


def run_dim(variant):
    """Local dimension R of a group's register runs from its variant bits: bit 4 (generated
    kernels only) R = 5, else bit 3 R = 4, else 3."""
    return 5 if variant & 16 else (4 if variant & 8 else 3)


def _role_rows(basis):
    """Row k: the local bits m whose basis vector has basis k's role coordinate."""
    return [sum(1 << m for m, (bm, _) in enumerate(basis) if (bm >> pk) & 1) for _, pk in basis]


def _plan_runs(steps, first, count, tsteps, truns, dim, R, tbit, slot_of, keep_bit0=False, run_off=None,
               step_ptab=None, touch=None):
    """Split a group's steps into register runs of local dimension R; False if a step does not fit.

    The 2^R local offsets of each run go to run_off[first step] and each step's parity table of
    those offsets to step_ptab[step]; the library's fixed-size records (dcs_tile_run,
    dcs_tile_step) hold them too where R <= 4.

    touch (a dict, generated kernels only): a basis vector may have another's role coordinate as
    long as the matrix of the basis at the role coordinates stays invertible (every coset of the
    run's span then still has exactly one entry zero at the roles).  A step's representative and
    dead entries then depend on several local bits; touch[step] = (T1, T2, DP): the other local
    bits touching the step's role(s) and the packed parity masks of the dead entries
    (runs_jit.cuh, deadp)."""
    vr = []
    for s in range(first, first + count):
        kind, _ = orbit_kind(steps[s])
        v, mix = _run_vectors(steps[s], kind, tsteps[s], tbit)
        if v is None:
            return False
        vr.append((v, mix))
    runs = []
    s = first
    while s < first + count:
        basis, n, locs = [], 0, []
        while s + n < first + count and n < 255:
            if int(tsteps[s + n]["cskip"]) != int(tsteps[s]["cskip"]):
                break
            nb = list(basis)
            loc = []
            ok = True
            for v, p in vr[s + n - first][0]:
                idx = next((i for i, (bv, _) in enumerate(nb) if bv == v), None)
                if idx is None:
                    nb.append((v, p))
                    loc.append(len(nb) - 1)
                elif nb[idx][1] != p:
                    ok = False
                else:
                    loc.append(idx)
            ok = ok and len(nb) <= R and _rank([v for v, _ in nb]) == len(nb) and len({p for _, p in nb}) == len(nb)
            if touch is None:
                # no basis vector touches another's role coordinate (the representatives of every
                # step are then the local indices with a zero at the step's own local bit)
                ok = ok and all(not (vb >> pa) & 1 for ia, (_, pa) in enumerate(nb)
                                for ib, (vb, _) in enumerate(nb) if ia != ib)
            else:
                ok = ok and _rank(_role_rows(nb)) == len(nb)
            if not ok:
                break
            basis = nb
            locs.append(loc)
            n += 1
        if n == 0:
            return False
        runs.append((s, n, basis, locs))
        s += n
    for s0, n, basis, locs in runs:
        roles = {p for _, p in basis}
        support = 0
        for v, _ in basis:
            support |= v
        active = slot_mask(steps[s0].active_in)
        inactive = [q for q in range(dim) if not (active >> slot_of(q)) & 1 and q not in roles
                    and not (support >> q) & 1]
        # pad to R dimensions with unit vectors of active coordinates outside the run's support:
        # tile bit 0 first (local entries j and j + e_0 are then one aligned 16-byte word, moved
        # by one shared-memory instruction) unless keep_bit0 (packed plans: bit 0 pairs cosets),
        # then the highest (the low coordinates stay with the threads of a warp)
        for q in ([] if keep_bit0 else [0]) + list(reversed(range(1, dim))):
            if len(basis) >= R:
                break
            if q not in roles and q not in inactive and not (support >> q) & 1:
                basis.append((1 << q, q))
                roles.add(q)
        if len(basis) < R:
            return False
        ins = sorted(roles | set(inactive))
        if len(ins) > 16:
            return False
        tr = truns[s0]
        tr["nins"], tr["count"], tr["r"] = len(ins), n, R
        for i, b in enumerate(ins):
            tr["ins"][i] = b
        free = [b for b in range(dim) if b not in ins]
        tr["mhi"] = sum(1 << b for b in free[8:])
        offs = []
        for j in range(1 << R):
            o = 0
            for k in range(R):
                if (j >> k) & 1:
                    o ^= basis[k][0]
            offs.append(o)
            if R <= 4:
                tr["off"][j] = o
        if run_off is not None:
            run_off[s0] = offs
        for i in range(n):
            ts = tsteps[s0 + i]
            act = slot_mask(steps[s0 + i].active_in)
            ts["rdead"] = sum(1 << k for k, (_, p) in enumerate(basis)
                              if k not in locs[i] and not (act >> slot_of(p)) & 1)
            if touch is not None:
                rows = _role_rows(basis)
                dead = [rows[k] for k, (_, p) in enumerate(basis) if k not in locs[i] and not (act >> slot_of(p)) & 1]
                loc2 = locs[i] + [None, None]
                t1 = rows[loc2[0]] & ~(1 << loc2[0]) if loc2[0] is not None else 0
                t2 = rows[loc2[1]] & ~(1 << loc2[1]) if loc2[1] is not None else 0
                dp = 0
                for q, mask in enumerate(dead):
                    dp |= mask << (6 * q)
                touch[s0 + i] = (t1, t2, dp)
                if dp or t1 or t2:
                    ts["rdead"] = 0  # the kernel takes the parity masks instead
            loc = locs[i] + [0, 0]
            ts["rk1"], ts["rk2"] = loc[0], loc[1]
            ts["rmix"] = vr[s0 + i - first][1]
            tb = int(ts["tbeta"])
            ptab = sum((bin(o & tb).count("1") & 1) << j for j, o in enumerate(offs))
            if R <= 4:
                ts["ptab"] = ptab
            if step_ptab is not None:
                step_ptab[s0 + i] = ptab
            ts["run_len"] = n if i == 0 else 0
    return True


def build_fused_plan(plan, max_dim=13, low=4, max_steps=MAX_GROUP_STEPS, max_extra=1, spans=None, variant=0,
                     pairs=False, grouping="greedy", group_cost=1 << 30, fp64=False, prefetch_kb=0,
                     group_variant=None):
    """grouping: "greedy" (group_steps) or "bytes" (group_steps_min_bytes, `group_cost` bytes
    charged per group).  fp64: the plan runs on a complex128 table (plan-specialised register
    runs only, see jit.py).  prefetch_kb: staging of the next tile's first-run entries in the
    generated kernels (jit.prefetch_layout).  group_variant: {group: variant} for single groups
    (variant bit 4, register runs of dimension 5, falls back to dimension 4 where a run does not
    fit)."""
    steps = plan.steps
    if spans is None:
        if grouping == "bytes":
            spans = group_steps_min_bytes(steps, max_dim, low, max_steps, max_extra, group_cost)
        elif grouping == "greedy":
            spans = group_steps(steps, max_dim, low, max_steps, max_extra)
        else:
            raise ValueError(f"grouping {grouping!r}")
    groups = np.zeros(len(spans), dtype=_lib.GROUP_DTYPE)
    tsteps = np.zeros(len(steps), dtype=_lib.TILE_STEP_DTYPE)
    runs_any = variant & 4 or any(int(v) & 4 for v in (group_variant or {}).values())
    truns = np.zeros(len(steps), dtype=_lib.TILE_RUN_DTYPE) if runs_any else None
    fp = FusedPlan(groups=groups, tile_steps=tsteps, dsteps=device_steps(steps), spans=list(spans), tile_runs=truns,
                   coset_pairs=bool(pairs and variant & 4), fp64=bool(fp64), prefetch_kb=int(prefetch_kb))
    for gi, (first, count) in enumerate(spans):
        U = 0
        vecs = []
        for st in steps[first:first + count]:
            U |= slot_mask(st.active_in) | slot_mask(st.active_out)
            if orbit_kind(st)[0] == KIND_GROW:
                U |= 1 << st.pivot
            vecs += _orbit_vectors(st)
        l = _low_bits(U, low)
        basis, pivots = _reduced_basis(vecs, l)
        # pad small tiles with unit vectors of the slot universe (longer contiguous rows first)
        nU = bin(U).count("1")
        while l + len(basis) < min(max_dim, nU):
            if l < 6 and (U >> l) & 1 and l not in pivots:
                l += 1
                basis, pivots = _reduced_basis(vecs, l)
                continue
            span_piv = set(pivots) | set(range(l))
            extra = next((q for q in range(64) if (U >> q) & 1 and q not in span_piv), None)
            if extra is None:
                break
            vecs = vecs + [1 << extra]
            basis, pivots = _reduced_basis(vecs, l)
        if len(basis) > MAX_BASIS:
            raise ValueError(f"group {gi}: {len(basis)} tile basis vectors exceed {MAX_BASIS}")
        # order the non-low coordinates by how often a step of the group inserts a zero there
        # (role slots and inactive slots): the least-inserted ones take the low coordinates, so
        # the 32 lanes of a warp mostly touch consecutive entries (fewer bank conflicts)
        group_steps_ = steps[first:first + count]
        def inserted(pv):
            c = 0
            for st in group_steps_:
                kind, omit = orbit_kind(st)
                role = {KIND_GROW: [st.pivot], 1: [st.pivot_a], 3: [st.pivot], 5: [st.pivot], 7: [st.pivot],
                        6: [st.pivot, st.pivot_a]}.get(kind, [])
                if pv in role or not (slot_mask(st.active_in) >> pv) & 1:
                    c += 1
            return c
        order_ = sorted(range(len(basis)), key=lambda i: (inserted(pivots[i]), i))
        basis = [basis[i] for i in order_]
        pivots = [pivots[i] for i in order_]
        dim = l + len(basis)
        for b in basis:
            if b & ~U:
                raise AssertionError("tile basis leaves the slot universe")
        lowmask = (1 << l) - 1
        cmask = U & ~lowmask
        for p in pivots:
            cmask &= ~(1 << p)
        runs = deposit_runs(cmask)
        if len(runs) > _lib.MAX_RUNS:
            raise ValueError(f"group {gi}: {len(runs)} coset runs exceed {_lib.MAX_RUNS}")

        def coords(v):
            t = v & lowmask
            acc = v & lowmask
            for i, (b, p) in enumerate(zip(basis, pivots)):
                if (v >> p) & 1:
                    t |= 1 << (l + i)
                    acc ^= b
            if acc != v:
                raise AssertionError("orbit vector outside the tile space")
            return t

        g = groups[gi]
        g["first"], g["count"], g["tile_dim"], g["low_bits"] = first, count, dim, l
        g["coset_m"], g["ncoset_runs"], g["step_tile_off"] = bin(cmask).count("1"), len(runs), first
        g["out_mask"] = slot_mask(steps[first + count - 1].active_out)
        gvar = int((group_variant or {}).get(gi, variant))
        g["variant"] = gvar
        for i, b in enumerate(basis):
            g["basis"][i] = b
        for r, (src, dst, ln) in enumerate(runs):
            g["coset_runs"][r] = src | (dst << 8) | (ln << 16)
        for s in range(first, first + count):
            st = steps[s]
            kind, _ = orbit_kind(st)
            ts = tsteps[s]
            tK = coords(st.K) if kind in (3, 5, 6, 7) else 0
            tKa = coords(st.Ka) if kind in (1, 6) else 0
            tpiv = coords(1 << st.pivot) if kind == KIND_GROW else 0
            ts["tK"], ts["tKa"], ts["tpiv"] = tK, tKa, tpiv
            # sign functional in tile coordinates: parity(a(t) & beta) = parity(base & beta) ^ parity(t & tbeta)
            tbeta = st.beta & lowmask
            for i, b in enumerate(basis):
                if bin(b & st.beta).count("1") & 1:
                    tbeta |= 1 << (l + i)
            ts["tbeta"] = tbeta
            par = lambda v: bin(v).count("1") & 1
            ts["sK"], ts["sKa"] = par(tK & tbeta), par(tKa & tbeta)
            # orbit representatives: the role slots (pivots of K, Ka, grow) are pivot positions of
            # the reduced tile basis, so "slot q is zero" is "tile bit tbit(q) is zero"; inserting
            # zero bits there enumerates exactly the entries c of the reference kernel
            def tbit(q):
                if q < l:
                    return q
                return l + pivots.index(q)
            role = []
            if kind == KIND_GROW:
                role = [st.pivot]
            elif kind == 1:
                role = [st.pivot_a]
            elif kind in (3, 5, 7):
                role = [st.pivot]
            elif kind == 6:
                role = [st.pivot, st.pivot_a]
            tilepos = set(range(l)) | set(pivots)
            inactive = [q for q in range(64) if (U >> q) & 1 and not (slot_mask(st.active_in) >> q) & 1
                        and q not in role]
            ins = sorted([tbit(q) for q in role] + [tbit(q) for q in inactive if q in tilepos])
            cskip = 0
            for q in inactive:
                if q not in tilepos:
                    cskip |= 1 << q
            if len(ins) > 16 or len(set(ins)) != len(ins):
                raise ValueError(f"step {s}: {len(ins)} inserted tile bits")
            ts["nins"] = len(ins)
            for i, b in enumerate(ins):
                ts["ins"][i] = b
            ts["cskip"] = cskip
            free = [b for b in range(dim) if b not in ins]
            ts["mhi"] = sum(1 << b for b in free[8:])  # 256 threads: index bits >= 8
            ts["rb1"] = max(st.pivot_a if kind == 1 else st.pivot, 0)  # role slot(s), for checking
            ts["rb2"] = max(st.pivot_a, 0) if kind == 6 else 0
        if gvar & 4:
            slot_of = lambda q: q if q < l else pivots[q - l]
            # packed plans (bit 1) keep tile bit 0 out of the runs: it is the lane bit
            # variant bit 6: run bases may touch other roles (fewer runs; generated kernels only)
            tch = fp.step_touch if gvar & 64 else None
            ok = _plan_runs(steps, first, count, tsteps, truns, dim, run_dim(gvar), tbit, slot_of,
                            keep_bit0=bool(gvar & 2), run_off=fp.run_off, step_ptab=fp.step_ptab, touch=tch)
            if not ok and gvar & 16:  # dimension 5 does not fit: dimension 4
                gvar = (gvar & ~16) | 8
                g["variant"] = gvar
                ok = _plan_runs(steps, first, count, tsteps, truns, dim, 4, tbit, slot_of,
                                keep_bit0=bool(gvar & 2), run_off=fp.run_off, step_ptab=fp.step_ptab, touch=tch)
            if not ok:
                g["variant"] = gvar & ~92  # this group keeps the one-step-per-round-trip kernel
        elif pairs:
            _pair_steps(steps, first, count, tsteps, dim, tilepos_of=lambda q: (q < l or q in pivots),
                        tbit=tbit, U=U)
        fp.universe.append(bin(U).count("1"))
        fp.tiles.append(1 << bin(cmask).count("1"))
        fp.dims.append(dim)
    return fp
