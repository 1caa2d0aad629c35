"""ORACLE (test infrastructure): NumPy complex128 restatement of the conditional-block engine.

Not part of the product.  Each function follows the reference file:line it
cites.  It is deliberately written as plain loops over explicit arrays so it
reads independently of the product's planner and kernels.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

W_T = np.array([1.0, np.exp(1j * math.pi / 4)])                      # scan_plan.py:28
_RXM = np.array([[1, -1j], [-1j, 1]]) / math.sqrt(2)                  # exp(-i pi/4 X), parity_slicing.py:20
_RZP = np.diag([np.exp(1j * math.pi / 4), np.exp(-1j * math.pi / 4)])  # exp(+i pi/4 Z), parity_slicing.py:21


def lc(A, U, v):
    """parity_slicing.py:23-32 — local complementation at v."""
    nb = list(np.flatnonzero(A[v]))
    for a in nb:
        for b in nb:
            if a != b:
                A[a, b] ^= 1
    if U is not None:
        U[v] = U[v] @ _RXM
        for u in nb:
            U[u] = U[u] @ _RZP


def future_masks(N, edges, order):
    """scan_plan.py:45-55."""
    pos = {int(v): i for i, v in enumerate(order)}
    fut = [0] * N
    for a, b in edges:
        i, j = sorted((pos[int(a)], pos[int(b)]))
        fut[i] |= 1 << j
    return fut


def is_fixed(u, data, tol=1e-12):
    """scan_plan.py:123-130 — a zero entry in every contraction row."""
    rows = [u[0], u[1]] if data else [W_T @ u]
    return all(min(abs(r[0]), abs(r[1])) < tol for r in rows)


def compile_plan(order, fut, fixed, stop):
    """inplace_plan.py:26-78 — preserved-coordinate plan; returns (steps, terminal dict, maxslots).

    Each step is a dict with kind, active_in/out, beta, K, Ka, pivot, pivot_a, free, v, j.
    """
    basis = {}
    steps = []
    maxslots = 0
    for j in range(stop):
        v = int(order[j])
        beta = sum(1 << p for p, b in basis.items() if (b >> j) & 1)
        act_in = tuple(sorted(basis))
        rest = {p: b & ~(1 << j) for p, b in basis.items()}
        # elimination by top bit, slots in increasing order
        table = {}
        deps = []
        for p in sorted(rest):
            x, c = rest[p], 1 << p
            while x:
                t = x.bit_length() - 1
                if t not in table:
                    table[t] = (x, c)
                    break
                x ^= table[t][0]
                c ^= table[t][1]
            if x == 0:
                deps.append(c)
        assert len(deps) <= 1
        K = deps[0] if deps else 0
        pk = K.bit_length() - 1
        st = dict(v=v, j=j, kind="", active_in=act_in, beta=beta, K=K, Ka=0, pivot=pk, pivot_a=-1,
                  free=v not in fixed)
        if not st["free"]:
            st["kind"] = "fixed_shrink" if K else "fixed"
            if K:
                rest.pop(pk)
        else:
            x, c = fut[j], 0
            while x:
                t = x.bit_length() - 1
                if t not in table:
                    break
                x ^= table[t][0]
                c ^= table[t][1]
            if x:
                if K:
                    st["kind"] = "replace"
                    rest[pk] ^= fut[j]
                else:
                    p = 0
                    while p in rest:
                        p += 1
                    st["kind"] = "grow"
                    st["pivot"] = p
                    rest[p] = fut[j]
            else:
                if K:
                    if (c >> pk) & 1:
                        c ^= K
                    st["kind"] = "shrink"
                    rest.pop(pk)
                else:
                    st["kind"] = "mix"
                st["Ka"] = c
                st["pivot_a"] = c.bit_length() - 1
        basis = rest
        st["active_out"] = tuple(sorted(basis))
        steps.append(st)
        if basis:
            maxslots = max(maxslots, max(basis) + 1)
    return steps, basis, maxslots


def _addr(slots, omit=()):
    """inplace_plan.py:80-83 — deposit 0..2^m-1 into the listed slots."""
    use = [p for p in slots if p not in omit]
    x = np.arange(1 << len(use), dtype=np.uint64)
    out = np.zeros_like(x)
    for i, p in enumerate(use):
        out |= ((x >> np.uint64(i)) & np.uint64(1)) << np.uint64(p)
    return out


def _sgn(c, beta, ov):
    """inplace_plan.py:85-88 — (-1)^(parity(c & beta) xor ov)."""
    y = c & np.uint64(beta)
    par = np.zeros_like(y)
    while np.any(y):
        par ^= y & np.uint64(1)
        y = y >> np.uint64(1)
    return 1 - 2 * (par.astype(np.int64) ^ int(ov))


def execute(steps, f, yfix, fut, maxslots, dtype=np.complex128):
    """inplace_plan.py:90-135 — one-buffer executor with power-of-two renormalisation.

    Returns (terminal environment, log scale, final offset)."""
    E = np.zeros(1 << maxslots, dtype=dtype)
    E[0] = 1
    offset = 0
    ls = 0.0
    for st in steps:
        j = st["j"]
        ov = (offset >> j) & 1
        offset &= ~(1 << j)
        f0, f1 = complex(f[st["v"]][0]), complex(f[st["v"]][1])
        y = int(yfix[st["v"]]) if not st["free"] else 0
        if y:
            offset ^= fut[j]
        kind, beta, K, Ka = st["kind"], st["beta"], st["K"], st["Ka"]
        ain = st["active_in"]
        if kind == "grow":
            c = _addr(ain)
            a = E[c].copy()
            E[c] = f0 * a
            E[c | np.uint64(1 << st["pivot"])] = f1 * a * _sgn(c, beta, ov)
        elif kind == "mix" and Ka:
            c = _addr(ain, (st["pivot_a"],))
            d = c ^ np.uint64(Ka)
            a, b = E[c].copy(), E[d].copy()
            E[c] = f0 * a + f1 * _sgn(d, beta, ov) * b
            E[d] = f0 * b + f1 * _sgn(c, beta, ov) * a
        elif kind == "mix":
            c = _addr(ain)
            E[c] = E[c] * (f0 + f1 * _sgn(c, beta, ov))
        elif kind == "replace":
            c = _addr(ain, (st["pivot"],))
            d = c ^ np.uint64(K)
            a, b = E[c].copy(), E[d].copy()
            E[c] = f0 * (a + b)
            E[d] = f1 * (_sgn(c, beta, ov) * a + _sgn(d, beta, ov) * b)
        elif kind == "fixed":
            c = _addr(ain)
            E[c] = E[c] * (f1 * _sgn(c, beta, ov) if y else f0)
        elif kind == "fixed_shrink":
            c = _addr(ain, (st["pivot"],))
            d = c ^ np.uint64(K)
            a, b = E[c].copy(), E[d].copy()
            if y:
                E[c] = f1 * (_sgn(c, beta, ov) * a + _sgn(d, beta, ov) * b)
            else:
                E[c] = f0 * (a + b)
        elif kind == "shrink" and Ka:
            c = _addr(ain, (st["pivot"], st["pivot_a"]))
            c1 = c ^ np.uint64(K)
            d = c ^ np.uint64(Ka)
            d1 = d ^ np.uint64(K)
            a, b, e, g = E[c].copy(), E[c1].copy(), E[d].copy(), E[d1].copy()
            E[c] = f0 * (a + b) + f1 * (_sgn(d, beta, ov) * e + _sgn(d1, beta, ov) * g)
            E[d] = f0 * (e + g) + f1 * (_sgn(c, beta, ov) * a + _sgn(c1, beta, ov) * b)
        elif kind == "shrink":
            c = _addr(ain, (st["pivot"],))
            d = c ^ np.uint64(K)
            a, b = E[c].copy(), E[d].copy()
            E[c] = (f0 + f1 * _sgn(c, beta, ov)) * a + (f0 + f1 * _sgn(d, beta, ov)) * b
        else:
            raise ValueError(kind)
        out = _addr(st["active_out"])
        m = float(np.max(np.abs(E[out]))) if len(out) else 0.0
        if m:
            e = math.frexp(m)[1]
            E[out] *= math.ldexp(1.0, -e)
            ls += e * math.log(2.0)
    active = steps[-1]["active_out"] if steps else ()
    return E[_addr(active)], ls, offset


def _to_half(x):
    """Round FP64 values to binary16 as float_to_half_((float)x) does: FP64 -> FP32 -> binary16,
    each to nearest even (inplace_half_gpu.py:18-24)."""
    return x.astype(np.float32).astype(np.float16)


def execute_half(steps, f, yfix, fut, maxslots):
    """inplace_half_gpu.py:59-78 with the orbit kernel of inplace_gpu.py:20-63 — the half-storage
    tier: every entry is stored as two binary16 components, read back exactly into FP64, combined
    in FP64, multiplied by 2^-e of the PREVIOUS step's max (1 before the first step), and rounded
    on the store.  The max is taken over the stored (rounded) values, |v|^2 summed in FP32.

    Returns (terminal environment as complex64, log scale, final offset), or (None, log scale,
    offset) when a step leaves an all-zero table (inplace_half_gpu.py:74)."""
    re = np.zeros(1 << maxslots, np.float16)
    im = np.zeros(1 << maxslots, np.float16)
    re[0] = 1.0
    offset = 0
    ls = 0.0
    maximum = 1.0

    def rd(c):
        return re[c].astype(np.float64) + 1j * im[c].astype(np.float64)

    for st in steps:
        j = st["j"]
        ov = (offset >> j) & 1
        offset &= ~(1 << j)
        f0, f1 = complex(f[st["v"]][0]), complex(f[st["v"]][1])
        y = int(yfix[st["v"]]) if not st["free"] else 0
        if y:
            offset ^= fut[j]
        e = math.frexp(maximum)[1]
        scale = math.ldexp(1.0, -e)
        ls += e * math.log(2.0)
        kind, beta, K, Ka = st["kind"], st["beta"], st["K"], st["Ka"]
        ain = st["active_in"]
        writes = []
        if kind == "grow":
            c = _addr(ain)
            a = rd(c)
            writes = [(c, f0 * a), (c | np.uint64(1 << st["pivot"]), f1 * (a * _sgn(c, beta, ov)))]
        elif kind == "mix" and Ka:
            c = _addr(ain, (st["pivot_a"],))
            d = c ^ np.uint64(Ka)
            a, b = rd(c), rd(d)
            writes = [(c, f0 * a + f1 * (b * _sgn(d, beta, ov))), (d, f0 * b + f1 * (a * _sgn(c, beta, ov)))]
        elif kind == "mix":
            c = _addr(ain)
            writes = [(c, (f0 + f1 * _sgn(c, beta, ov)) * rd(c))]
        elif kind == "replace":
            c = _addr(ain, (st["pivot"],))
            d = c ^ np.uint64(K)
            a, b = rd(c), rd(d)
            writes = [(c, f0 * (a + b)), (d, f1 * (a * _sgn(c, beta, ov) + b * _sgn(d, beta, ov)))]
        elif kind == "fixed":
            c = _addr(ain)
            writes = [(c, (f1 * _sgn(c, beta, ov) if y else f0) * rd(c))]
        elif kind == "fixed_shrink":
            c = _addr(ain, (st["pivot"],))
            d = c ^ np.uint64(K)
            a, b = rd(c), rd(d)
            writes = [(c, f1 * (a * _sgn(c, beta, ov) + b * _sgn(d, beta, ov)) if y else f0 * (a + b))]
        elif kind == "shrink" and Ka:
            c = _addr(ain, (st["pivot"], st["pivot_a"]))
            c1 = c ^ np.uint64(K)
            d = c ^ np.uint64(Ka)
            d1 = d ^ np.uint64(K)
            a, b, g, h = rd(c), rd(c1), rd(d), rd(d1)
            writes = [(c, f0 * (a + b) + f1 * (g * _sgn(d, beta, ov) + h * _sgn(d1, beta, ov))),
                      (d, f0 * (g + h) + f1 * (a * _sgn(c, beta, ov) + b * _sgn(c1, beta, ov)))]
        elif kind == "shrink":
            c = _addr(ain, (st["pivot"],))
            d = c ^ np.uint64(K)
            a, b = rd(c), rd(d)
            writes = [(c, (f0 + f1 * _sgn(c, beta, ov)) * a + (f0 + f1 * _sgn(d, beta, ov)) * b)]
        else:
            raise ValueError(kind)
        m2 = np.float32(0)
        for c, v in writes:  # every orbit is read before any write: the orbits are disjoint
            hr, hi = _to_half(v.real * scale), _to_half(v.imag * scale)
            re[c], im[c] = hr, hi
            r, i = hr.astype(np.float32), hi.astype(np.float32)
            if len(r):
                m2 = max(m2, np.max(r * r + i * i))
        if not np.isfinite(m2):
            raise ArithmeticError("Nonfinite half-storage environment")
        if m2 == 0:
            return None, ls, offset
        maximum = math.sqrt(float(m2))
    active = steps[-1]["active_out"] if steps else ()
    t = _addr(active)
    env = re[t].astype(np.float32) + 1j * im[t].astype(np.float32)
    return env.astype(np.complex64), ls, offset


class OracleEngine:
    """Restatement of ``InplaceConditionalBlockGPU`` (conditional_block_gpu.py:25-177 and
    conditional_block_inplace_gpu.py:18-38) on the CPU in complex128."""

    def __init__(self, graph, unitaries, n, order, parity_operations, open_vertices):
        A = np.asarray(graph, np.uint8).copy()
        self.N_full = N = len(A)
        self.n = n
        U = {i: np.asarray(u, complex).copy() for i, u in enumerate(unitaries)}
        self.open_full = [int(q) for q in open_vertices]
        if len(set(self.open_full)) != len(self.open_full) or not all(0 <= q < n for q in self.open_full):
            raise ValueError("Free vertices must be distinct data vertices")
        ops = [(op[0], int(op[1]), None if op[2] is None else int(op[2])) for op in parity_operations]
        self.slices = [w for _, w, _ in ops]
        if set(self.slices) & set(range(n)):
            raise ValueError("This adapter only permits slicing reference vertices")
        for kind, w, u in ops:
            if kind == "Y":
                lc(A, U, w)
            elif kind == "X":
                lc(A, U, u); lc(A, U, w); lc(A, U, u)
            elif kind != "Z":
                raise ValueError(kind)
        self.U_full = U
        edges = [(a, b) for a in range(N) for b in range(a + 1, N) if A[a, b]]
        S = set(self.slices)
        self.keep = [v for v in range(N) if v not in S]
        self.relabel = {v: i for i, v in enumerate(self.keep)}
        self.nbrs = {s: [] for s in self.slices}
        self.slice_edges = []
        red = []
        for a, b in edges:
            if a in S and b in S:
                self.slice_edges.append((a, b))
            elif a in S:
                self.nbrs[a].append(self.relabel[b])
            elif b in S:
                self.nbrs[b].append(self.relabel[a])
            else:
                red.append((self.relabel[a], self.relabel[b]))
        self.N = len(self.keep)
        fixed = {self.relabel[v] for v in range(N) if v in self.relabel and is_fixed(U[v], v < n)}
        self.open_red = [self.relabel[q] for q in self.open_full]
        O = set(self.open_red)
        order = [self.relabel[int(v)] for v in order if int(v) in self.relabel]
        self.order = [v for v in order if v not in O] + self.open_red
        self.fixed = fixed - O
        self.stop = self.N - len(O)
        self.fut = future_masks(self.N, red, self.order)
        self.steps, term, self.maxslots = compile_plan(self.order, self.fut, self.fixed, self.stop)
        self.terminal_basis = [term[p] >> self.stop for p in sorted(term)]
        self.open_edges = [(self.open_red.index(a), self.open_red.index(b)) for a, b in red
                           if a in O and b in O]
        k = len(self.open_full)
        tr = len(self.terminal_basis)
        ids = np.arange(1 << tr, dtype=np.uint64)
        self.syndrome_map = np.zeros(1 << tr, dtype=np.uint64)
        for j, b in enumerate(self.terminal_basis):
            self.syndrome_map ^= ((ids >> np.uint64(j)) & np.uint64(1)) * np.uint64(b)
        ids = np.arange(1 << k, dtype=np.uint64)
        self.phase = np.ones(1 << k)
        for a, b in self.open_edges:
            self.phase *= 1 - 2 * ((ids >> np.uint64(a)) & (ids >> np.uint64(b)) & np.uint64(1)).astype(float)

    def local_vectors(self, x_bits, w=None):
        """scan_plan.py:108-120."""
        f = {}
        for q in range(self.N_full):
            u = self.U_full[q]
            if q < self.n:
                f[q] = np.eye(2)[int(x_bits[q])] @ u
            else:
                bra = np.asarray(w[q]) if isinstance(w, dict) else (W_T if w is None else np.asarray(w))
                f[q] = bra @ u
        return f

    def slice_inputs(self, x_bits, w=None, part=0, parts=1):
        """conditional_block_gpu.py:136-152 — per-slice (coef, f, yfix, flips)."""
        f_full = self.local_vectors(x_bits, w)
        out = []
        for idx, bits in enumerate(itertools.product((0, 1), repeat=len(self.slices))):
            if idx % parts != part:
                continue
            val = dict(zip(self.slices, bits))
            coef = complex(np.prod([f_full[s][val[s]] for s in self.slices]))
            coef *= (-1) ** sum(val[a] * val[b] for a, b in self.slice_edges)
            flips = np.zeros(self.N, np.uint8)
            for s in self.slices:
                if val[s]:
                    for v in self.nbrs[s]:
                        flips[v] ^= 1
            f = {self.relabel[v]: np.asarray(f_full[v]) * np.array([1, 1 - 2 * int(flips[self.relabel[v]])])
                 for v in self.keep}
            yfix = {q: (0 if abs(f[q][0]) > 1e-12 else 1) for q in self.fixed}
            out.append((coef, f, yfix, flips))
        return out

    def block(self, x_bits, w=None, part=0, parts=1, storage=None):
        """conditional_block_gpu.py:128-177 — returns the sqrt(D)-scaled complex128 block.

        storage="float16" contracts every slice with the half-storage executor (execute_half)."""
        k = len(self.open_full)
        total = np.zeros(1 << k, np.complex128)
        count = 0
        for coef, f, yfix, flips in self.slice_inputs(x_bits, w, part, parts):
            count += 1
            if not coef:
                continue
            if storage == "float16":
                env, ls, offset = execute_half(self.steps, f, yfix, self.fut, self.maxslots)
                if env is None:
                    continue
            else:
                env, ls, offset = execute(self.steps, f, yfix, self.fut, self.maxslots)
            if not np.any(env):
                continue
            freeflip = sum(int(flips[q]) << j for j, q in enumerate(self.open_red))
            idx = self.syndrome_map ^ np.uint64((offset >> self.stop) ^ freeflip)
            c = coef * math.exp(ls - (self.N_full - self.n + k) * 0.5 * math.log(2.0))
            total[idx.astype(np.int64)] += env.astype(np.complex128) * c  # FP64, as the reference
        tail(total, k, self.phase, [self.U_full[q] for q in self.open_full])
        return total, {"slices_evaluated": count, "terminal_rank": len(self.terminal_basis)}


def tail(total, k, phase, Uopen):
    """conditional_block_gpu.py:159-171 — k Walsh-Hadamard passes, open-edge phase, U_open."""
    for q in range(k):
        v = total.reshape(-1, 2, 1 << q)
        lo, hi = v[:, 0].copy(), v[:, 1].copy()
        v[:, 0], v[:, 1] = lo + hi, lo - hi
    total *= phase
    for q in range(k):
        u = Uopen[q]
        v = total.reshape(-1, 2, 1 << q)
        lo, hi = v[:, 0].copy(), v[:, 1].copy()
        v[:, 0] = u[0, 0] * lo + u[0, 1] * hi
        v[:, 1] = u[1, 0] * lo + u[1, 1] * hi
    return total


def brute_force_block(graph, unitaries, n, open_vertices, x_bits, w=None):
    """Independent check for tiny graphs: sum over all 2^N vertex values, then read the block.

    Returns sqrt(D) * <x_closed, y_open | U | 0> over the open bits y (up to a global phase)."""
    A = np.asarray(graph, np.uint8)
    N = len(A)
    U = [np.asarray(u, complex) for u in unitaries]
    k = len(open_vertices)
    ys = np.arange(1 << N, dtype=np.int64)
    bits = ((ys[:, None] >> np.arange(N)) & 1).astype(np.int64)
    par = np.einsum("si,ij,sj->s", bits, np.triu(A, 1).astype(np.int64), bits) & 1
    graph_amp = (1 - 2 * par) / 2 ** (N / 2)
    out = np.zeros(1 << k, complex)
    for idx in range(1 << k):
        x = np.array(x_bits, dtype=np.int64).copy()
        for j, q in enumerate(open_vertices):
            x[q] = (idx >> j) & 1
        prod = np.ones(1 << N, complex)
        for q in range(N):
            if q < n:
                fq = np.eye(2)[x[q]] @ U[q]
            else:
                fq = (W_T if w is None else np.asarray(w)) @ U[q]
            prod *= fq[bits[:, q]]
        out[idx] = np.sum(prod * graph_amp)
    return out * math.sqrt(2.0 ** (n - k))
