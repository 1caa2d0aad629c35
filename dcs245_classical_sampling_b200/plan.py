"""Host-side planning for the conditional-block contraction (exact GF(2) arithmetic).

Everything here is integer bookkeeping that runs once per circuit and plan, in
Python, exactly as the reference does it; only the per-step arithmetic moves to
the GPU.  Bit sets are Python integers: bit j of a "future" vector is the
vertex at position j of the contraction order, bit p of a slot mask is
physical coordinate slot p of the in-place table.

Restated reference functions (each must produce bit-identical plans, because
phase masks and plan order are part of the drop-in contract):

* ``future_masks``       <- ``source/dcs_rankwidth/scan_plan.py:45-55``
* ``structurally_fixed`` <- ``source/dcs_rankwidth/scan_plan.py:123-130``
* ``local_vectors``      <- ``source/dcs_rankwidth/scan_plan.py:108-120`` (``W_T`` :28)
* ``compile_inplace``    <- ``source/kernel_opt/inplace_plan.py:26-78``
* ``orbit_kind``         <- ``source/kernel_opt/inplace_gpu.py:74-82``
* ``local_complement``   <- ``source/dcs_rankwidth/parity_slicing.py:23-32``
* ``prefix_cut_ranks`` / ``choose_parity_slices``
                         <- ``source/dcs_rankwidth/parity_slicing.py:35-105``
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

W_T = np.array([1.0, np.exp(1j * math.pi / 4)])

# Orbit kinds executed by the device step kernel (same numbering as the
# reference executor's ``kind`` argument).
KIND_GROW, KIND_MIX, KIND_DIAG, KIND_REPLACE = 0, 1, 2, 3
KIND_FIXED, KIND_FIXED_SHRINK, KIND_SHRINK4, KIND_SHRINK2 = 4, 5, 6, 7
KIND_NAMES = ("grow", "mix", "diag_mix", "replace", "fixed", "fixed_shrink", "shrink4", "shrink2")

_RX_MINUS = np.eye(2) * math.cos(math.pi / 4) - 1j * math.sin(math.pi / 4) * np.array([[0, 1], [1, 0]])
_RZ_PLUS = np.eye(2) * math.cos(math.pi / 4) + 1j * math.sin(math.pi / 4) * np.diag([1.0, -1.0])


def _top(v: int) -> int:
    return v.bit_length() - 1


def future_masks(N, edges, order):
    """fut[j]: positions of the later neighbours of the vertex at position j."""
    pos = {int(q): j for j, q in enumerate(order)}
    fut = [0] * N
    for a, b in edges:
        pa, pb = pos[int(a)], pos[int(b)]
        lo, hi = (pa, pb) if pa < pb else (pb, pa)
        fut[lo] |= 1 << hi
    return fut


def structurally_fixed(U, N, n, tol=1e-12):
    """Vertices whose contracted value is forced for every prefix (a zero entry)."""
    fixed = set()
    for q in range(N):
        u = np.asarray(U[q], dtype=np.complex128)
        rows = (u[0], u[1]) if q < n else (W_T @ u,)
        if all(min(abs(r[0]), abs(r[1])) < tol for r in rows):
            fixed.add(q)
    return fixed


def local_vectors(U, N, n, x_bits, w=None):
    """f_q = bra_q U_q: data vertices take row x_q, references take w (default W_T)."""
    out = {}
    for q in range(N):
        u = np.asarray(U[q], dtype=np.complex128)
        if q < n:
            out[q] = u[int(x_bits[q])].copy()
        else:
            if isinstance(w, dict):
                bra = np.asarray(w[q], dtype=np.complex128)
            elif w is None:
                bra = W_T
            else:
                bra = np.asarray(w, dtype=np.complex128)
            out[q] = bra @ u
    return out


def local_complement(A, U, v):
    """Local complementation at v on adjacency A (in place) and the local Cliffords U."""
    nb = np.nonzero(A[v])[0]
    if len(nb) > 1:
        A[np.ix_(nb, nb)] ^= 1
        A[nb, nb] = 0
    if U is not None:
        U[v] = U[v] @ _RX_MINUS
        for u in nb:
            U[u] = U[u] @ _RZ_PLUS


def apply_parity_operation(A, U, kind, w, u):
    """Y: one local complementation at w.  X: pivot on edge (w, u).  Z: nothing."""
    if kind == "Y":
        local_complement(A, U, w)
    elif kind == "X":
        local_complement(A, U, u)
        local_complement(A, U, w)
        local_complement(A, U, u)
    elif kind != "Z":
        raise ValueError(kind)


@dataclass
class OrbitStep:
    """One vertex step of the preserved-coordinate plan."""
    v: int
    j: int
    kind: str
    active_in: tuple
    active_out: tuple
    beta: int
    K: int = 0
    Ka: int = 0
    pivot: int = -1
    pivot_a: int = -1
    free: bool = True


def _pivot_reduce(columns):
    """Echelon form of {slot: vector} keyed by top bit; returns (pivots, dependency masks)."""
    pivots = {}
    deps = []
    for slot in sorted(columns):
        vec = int(columns[slot])
        coef = 1 << slot
        while vec:
            t = _top(vec)
            hit = pivots.get(t)
            if hit is None:
                pivots[t] = (vec, coef)
                break
            vec ^= hit[0]
            coef ^= hit[1]
        if not vec:
            deps.append(coef)
    return pivots, deps


def _express(vec, pivots):
    """Reduce vec by the pivots while its top bit has one; returns (residual, slot mask)."""
    vec = int(vec)
    coef = 0
    while vec:
        hit = pivots.get(_top(vec))
        if hit is None:
            break
        vec ^= hit[0]
        coef ^= hit[1]
    return vec, coef


def compile_inplace(order, future, fixed, stop=None):
    """Preserved-coordinate, one-buffer plan: (steps, terminal {slot: vector}, maxslots)."""
    basis = {}
    steps = []
    maxslots = 0
    for j, v in enumerate(list(order)[:stop]):
        v = int(v)
        beta = 0
        for p, b in basis.items():
            if (b >> j) & 1:
                beta |= 1 << p
        active = tuple(sorted(basis))
        cleared = {p: b & ~(1 << j) for p, b in basis.items()}
        pivots, deps = _pivot_reduce(cleared)
        if len(deps) > 1:
            raise AssertionError("Deleting one vertex cannot drop more than one rank")
        K = deps[0] if deps else 0
        pk = _top(K)
        st = OrbitStep(v, j, "", active, (), beta, K=K, pivot=pk, free=v not in fixed)
        if not st.free:
            st.kind = "fixed_shrink" if K else "fixed"
            if K:
                del cleared[pk]
        else:
            residual, Ka = _express(future[j], pivots)
            if residual:
                if K:
                    st.kind = "replace"
                    cleared[pk] ^= future[j]
                else:
                    st.kind = "grow"
                    p = 0
                    while p in cleared:
                        p += 1
                    st.pivot = p
                    cleared[p] = future[j]
            elif K:
                st.kind = "shrink"
                if (Ka >> pk) & 1:
                    Ka ^= K
                st.Ka = Ka
                st.pivot_a = _top(Ka)
                del cleared[pk]
            else:
                st.kind = "mix"
                st.Ka = Ka
                st.pivot_a = _top(Ka)
        basis = cleared
        st.active_out = tuple(sorted(basis))
        steps.append(st)
        if basis:
            maxslots = max(maxslots, max(basis) + 1)
    return steps, basis, maxslots


def orbit_kind(st):
    """(kernel kind code, slots left out of the orbit enumeration)."""
    k = st.kind
    if k == "grow":
        return KIND_GROW, ()
    if k == "mix":
        return (KIND_MIX, (st.pivot_a,)) if st.Ka else (KIND_DIAG, ())
    if k == "replace":
        return KIND_REPLACE, (st.pivot,)
    if k == "fixed":
        return KIND_FIXED, ()
    if k == "fixed_shrink":
        return KIND_FIXED_SHRINK, (st.pivot,)
    if k == "shrink":
        return (KIND_SHRINK4, (st.pivot, st.pivot_a)) if st.Ka else (KIND_SHRINK2, (st.pivot,))
    raise ValueError(k)


def slot_mask(slots):
    m = 0
    for p in slots:
        m |= 1 << int(p)
    return m


def deposit_runs(mask: int):
    """Split a slot mask into contiguous runs (src_shift, dst_shift, length)."""
    runs = []
    src = 0
    p = 0
    while mask >> p:
        if (mask >> p) & 1:
            start = p
            while (mask >> p) & 1:
                p += 1
            runs.append((src, start, p - start))
            src += p - start
        else:
            p += 1
    return runs


# ---------------------------------------------------------------------------
# cut ranks and the greedy parity-slice chooser (planner; CPU)
# ---------------------------------------------------------------------------

def prefix_cut_ranks(A, order):
    """Cut rank of every proper prefix of `order` on the induced subgraph (length M-1), as
    prefix_ranks_matrix (parity_slicing.py:35-54) computes it; native GF(2) elimination in the
    library (dcs_prefix_cut_ranks)."""
    from . import _lib
    order = np.ascontiguousarray(np.asarray(list(order), dtype=np.int32))
    M = len(order)
    if M < 2:
        return np.zeros(0, dtype=np.int64)
    A = np.ascontiguousarray(np.asarray(A, dtype=np.uint8))
    out = np.zeros(M - 1, dtype=np.int32)
    _lib.check(_lib.load().dcs_prefix_cut_ranks(A.ctypes.data, A.shape[0], order.ctypes.data, M, out.ctypes.data))
    return out.astype(np.int64)


def _profile_cost(A, order):
    r = prefix_cut_ranks(A, order)
    m = int(r.max()) if r.size else 0
    return m, float(np.sum(2.0 ** (r - m)))


def choose_parity_slices(N, edges, order, k, window_pad=15, max_cand=60, n_pivots=4, seed=0):
    """Greedy Z/Y/X slice choice lowering (r_max, plateau); returns ([(kind, w, u)], removed)."""
    rng = np.random.default_rng(seed)
    A = np.zeros((N, N), dtype=np.uint8)
    for a, b in edges:
        A[a, b] = A[b, a] = 1
    ops, removed = [], []
    alive = list(order)
    for _ in range(k):
        r = prefix_cut_ranks(A, alive)
        m = int(r.max())
        hot = [i for i, x in enumerate(r) if x == m]
        cand = alive[max(0, min(hot) - window_pad):min(len(alive), max(hot) + window_pad + 2)]
        if len(cand) > max_cand:
            cand = list(rng.choice(cand, max_cand, replace=False))
        best = None
        alive_set = set(alive)
        for w in cand:
            rest = [x for x in alive if x != w]
            trials = [("Z", w, None), ("Y", w, None)]
            nb = [u for u in np.nonzero(A[w])[0] if u in alive_set]
            for u in (rng.choice(nb, min(n_pivots, len(nb)), replace=False) if nb else []):
                trials.append(("X", w, int(u)))
            for kind, ww, u in trials:
                B = A.copy()
                apply_parity_operation(B, None, kind, ww, u)
                c = _profile_cost(B, rest)
                if best is None or c < best[0]:
                    best = (c, kind, ww, u)
        _, kind, w, u = best
        apply_parity_operation(A, None, kind, w, u)
        ops.append((kind, int(w), None if u is None else int(u)))
        removed.append(int(w))
        alive = [x for x in alive if x != w]
    return ops, removed


# ---------------------------------------------------------------------------
# the engine-level plan (graph + parity operations + open vertices)
# ---------------------------------------------------------------------------

@dataclass
class BlockPlan:
    """Everything about one (graph, order, parity operations, open vertices) that is independent of x."""
    N_full: int
    n: int
    open_full: list
    slices: list
    U_full: dict
    relabel: dict
    keep: list
    nbrs_in_keep: dict
    slice_edges: list
    N: int
    edges: list
    order: list
    fixed: set
    open_red: list
    stop: int
    fut: list
    steps: list = field(default_factory=list)
    terminal_slots: tuple = ()
    terminal_basis: list = field(default_factory=list)
    maxslots: int = 0
    inplace_rmax: int = 0
    rmax: int = 1
    work: int = 0
    open_edges: list = field(default_factory=list)

    @property
    def terminal_rank(self):
        return len(self.terminal_basis)

    @property
    def k(self):
        return len(self.open_full)


def build_block_plan(graph, unitaries, n, order, parity_operations, open_vertices):
    """Engine constructor logic (``sampling/conditional_block_gpu.py:25-69`` and the plan half of
    ``sampling/conditional_block_inplace_gpu.py:18-34``), with the reference's errors."""
    A = np.asarray(graph, dtype=np.uint8).copy()
    N_full = len(A)
    U = {i: np.asarray(u, dtype=np.complex128).copy() for i, u in enumerate(unitaries)}
    open_full = [int(q) for q in open_vertices]
    if len(set(open_full)) != len(open_full) or not all(0 <= q < n for q in open_full):
        raise ValueError("Free vertices must be distinct data vertices")
    ops = [(str(op[0]), int(op[1]), None if op[2] is None else int(op[2])) for op in parity_operations]
    slices = [w for _, w, _ in ops]
    if set(slices) & set(range(n)):
        raise ValueError("This adapter only permits slicing reference vertices")
    for kind, w, u in ops:
        if kind not in ("X", "Y", "Z"):
            raise ValueError(kind)
        apply_parity_operation(A, U, kind, w, u)
    edges = [(int(a), int(b)) for a, b in zip(*np.nonzero(np.triu(A, 1)))]
    # vertex slicing (source/dcs_rankwidth/slicing.py:75-109)
    S = set(slices)
    keep = [v for v in range(N_full) if v not in S]
    relabel = {v: i for i, v in enumerate(keep)}
    nbrs_in_keep = {s: [] for s in slices}
    slice_edges, red_edges = [], []
    for a, b in edges:
        if a in S and b in S:
            slice_edges.append((a, b))
        elif a in S:
            nbrs_in_keep[a].append(relabel[b])
        elif b in S:
            nbrs_in_keep[b].append(relabel[a])
        else:
            red_edges.append((relabel[a], relabel[b]))
    fx_full = structurally_fixed(U, N_full, n)
    fixed = {relabel[v] for v in fx_full if v in relabel}
    red_order = [relabel[int(v)] for v in order if int(v) in relabel]
    open_red = [relabel[q] for q in open_full]
    O = set(open_red)
    red_order = [v for v in red_order if v not in O] + open_red
    fixed -= O
    N = len(keep)
    stop = N - len(O)
    fut = future_masks(N, red_edges, red_order)
    plan = BlockPlan(N_full=N_full, n=n, open_full=open_full, slices=slices, U_full=U,
                     relabel=relabel, keep=keep, nbrs_in_keep=nbrs_in_keep, slice_edges=slice_edges,
                     N=N, edges=red_edges, order=red_order, fixed=fixed, open_red=open_red,
                     stop=stop, fut=fut)
    steps, terminal, maxslots = compile_inplace(red_order, fut, fixed, stop)
    plan.steps = steps
    plan.maxslots = maxslots
    plan.inplace_rmax = max([0] + [len(s.active_out) for s in steps])
    if maxslots != plan.inplace_rmax:
        raise AssertionError("Unexpected physical slot expansion")
    plan.terminal_slots = tuple(sorted(terminal))
    plan.terminal_basis = [terminal[p] >> stop for p in plan.terminal_slots]
    # gather-plan ranks (scan_plan.make_plan): r_in = |active_in|, r_out = |active_out|,
    # kernel size = r_in + free - r_out; used only for the reported meta.
    plan.rmax = max([1] + [max(len(s.active_in), len(s.active_out)) for s in steps])
    plan.work = sum(1 << (len(s.active_in) + (1 if s.free else 0)) for s in steps)
    plan.open_edges = [(open_red.index(a), open_red.index(b)) for a, b in red_edges if a in O and b in O]
    return plan


def step_bytes(plan, elem_bytes=8):
    """Algorithmic HBM bytes of one slice: sum over steps of (2^|in| + 2^|out|) entries."""
    return sum(((1 << len(s.active_in)) + (1 << len(s.active_out))) * elem_bytes for s in plan.steps)


# ---------------------------------------------------------------------------------------------
# Gather form of the plan (source/dcs_rankwidth/scan_plan.py:58-105): the environment after step
# j is E'[c'] = sum over p in L c' + span(kernel) of E[p & mask_in] f_v(p >> r_in) sign, with two
# tables.  It is the plan of the reference's ConditionalBlockGPU (its two-buffer executor).

@dataclass
class GatherStep:
    v: int
    free: bool
    r_in: int
    r_out: int
    beta: int
    Lcols: list
    kernel: list


def _reduce_against(vec, basis, pivots):
    """(residual, coefficient bits) of vec reduced against basis vectors with the given pivots,
    in insertion order (scan_plan.py:35-42)."""
    coef = 0
    for k, (b, p) in enumerate(zip(basis, pivots)):
        if (vec >> p) & 1:
            vec ^= b
            coef |= 1 << k
    return vec, coef


def make_gather_plan(N, edges, order, fixed=frozenset()):
    """Gather plan of every position (scan_plan.py:58-105) -> (steps, rank profile)."""
    fut = future_masks(N, edges, order)
    basis = []
    steps, profile = [], []
    for j in range(N):
        v = order[j]
        free = v not in fixed
        beta = 0
        for i, b in enumerate(basis):
            beta |= ((b >> j) & 1) << i
        ws = [b & ~(1 << j) for b in basis] + ([fut[j]] if free else [])
        nb, piv, mcols = [], [], []
        for wv in ws:  # the new basis and each column's coordinates in it
            res, coef = _reduce_against(wv, nb, piv)
            if res:
                piv.append((res & -res).bit_length() - 1)
                nb.append(res)
                coef |= 1 << (len(nb) - 1)
            mcols.append(coef)
        r_out = len(nb)
        first_col = {}  # leading coordinate k -> first column that has it
        for i, m in enumerate(mcols):
            if m and (m.bit_length() - 1) not in first_col:
                first_col[m.bit_length() - 1] = i
        L = [0] * r_out  # right inverse: M L[k] = e_k
        for k in range(r_out):
            i = first_col[k]
            m = mcols[i]
            col = 1 << i
            for l in range(k):
                if (m >> l) & 1:
                    col ^= L[l]
            L[k] = col
        pivot_cols = set(first_col.values())
        kernel = []
        for i, m in enumerate(mcols):
            if i in pivot_cols:
                continue
            kv = 1 << i
            for k in range(r_out):
                if (m >> k) & 1:
                    kv ^= L[k]
            kernel.append(kv)
        steps.append(GatherStep(v=v, free=free, r_in=len(basis), r_out=r_out, beta=beta, Lcols=L, kernel=kernel))
        profile.append(r_out)
        basis = nb
    return steps, profile


def gather_byte_tables(cols, nbits):
    """Byte-wise XOR tables of c -> XOR_{i: c_i = 1} cols[i] (scan_plan.py:133-145): (nb, 256) uint64."""
    nb = max(1, (nbits + 7) // 8)
    T = np.zeros((nb, 256), dtype=np.uint64)
    for b in range(nb):
        for val in range(256):
            acc = 0
            for t in range(8):
                i = 8 * b + t
                if i < nbits and (val >> t) & 1:
                    acc ^= cols[i]
            T[b, val] = acc
    return T


def kernel_combos(kernel):
    """Every XOR combination of the kernel vectors (scan_plan.py:148-152)."""
    combos = [0]
    for kv in kernel:
        combos = combos + [c ^ kv for c in combos]
    return combos


@dataclass
class GatherPlan:
    steps: list
    rank_profile: list
    tables: list
    combos: list
    rmax: int
    work: int
    terminal_basis: list


def build_gather_plan(bp):
    """The gather plan of a block plan's reduced graph (conditional_block_gpu.py:47-64): steps up
    to `stop`, byte tables, kernel combinations, rmax, work and the terminal syndrome basis."""
    all_steps, profile = make_gather_plan(bp.N, bp.edges, bp.order, bp.fixed)
    steps = all_steps[:bp.stop]
    tables = [gather_byte_tables(st.Lcols, st.r_out) for st in steps]
    combos = [np.asarray(kernel_combos(st.kernel), np.uint64) for st in steps]
    rmax = max([1] + [max(s.r_in, s.r_out) for s in steps])
    work = sum((1 << s.r_out) * (1 << len(s.kernel)) for s in steps)
    basis = []
    for j, st in enumerate(steps):
        ws = [b & ~(1 << j) for b in basis] + ([bp.fut[j]] if st.free else [])
        nb, piv = [], []
        for old in ws:
            res, _ = _reduce_against(old, nb, piv)
            if res:
                piv.append((res & -res).bit_length() - 1)
                nb.append(res)
        basis = nb
    return GatherPlan(steps=steps, rank_profile=profile, tables=tables, combos=combos, rmax=rmax, work=work,
                      terminal_basis=[b >> bp.stop for b in basis])
