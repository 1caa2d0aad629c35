"""Seeded ring circuits, T-gadget injection and stabilizer-to-graph-state form.

This is the CPU preparation that sits in front of the contraction path. The
reference prepares its one real circuit with qiskit + stim
(``source/dcs_rankwidth/circuit_io.py:94-100``, ``t_injection.py:21-39`` and
``t_injection.py:62-79``); neither library exists on the target machines, so
the three published steps are restated here in exact GF(2) arithmetic:

1. ``ring_circuit`` draws a seeded Clifford+T ring circuit with the layer rule
   of the synthetic workloads (one gate from {H, S, Sdg, I} per qubit and
   layer, exactly ``t_count`` of those slots replaced by T at seeded positions,
   then CZ or CX on even pairs (2i, 2i+1) in even layers and odd pairs
   (2i+1, 2i+2 mod n) in odd layers).
2. ``inject`` replaces every T on qubit q by a fresh reference qubit prepared
   in |0> and a CNOT q -> reference; the reference is later contracted with
   the functional w = (1, e^{i pi/4}) (``t_injection.py:1-14``).  References
   are numbered n, n+1, ... in order of appearance and the natural order puts
   each reference right after its data qubit (``t_injection.py:21-39``).
3. ``graph_form`` writes the resulting stabilizer state as
   (U_1 x ... x U_N) |G>, with |G> = CZ_E |+>^N, using the
   Aaronson-Gottesman tableau (quant-ph/0406196) and the standard reduction
   of Van den Nest, Dehaene and De Moor (quant-ph/0308151): Hadamards make the
   X block invertible, Gauss-Jordan elimination makes it the identity, the Z
   block is then the adjacency matrix, S-dagger removes Y diagonals and Z
   removes signs.  Every U_k is H^p S^y Z^s with exact entries.

The output dictionary matches the reference's ``inputs/injected_graph.npz``
keys: ``graph`` (N,N) u8, ``unitaries`` (N,2,2) c128, ``order``, ``ring``,
``natural_order``.
"""
from __future__ import annotations

import math

import numpy as np

_H = np.array([[1, 1], [1, -1]], dtype=np.complex128) / math.sqrt(2.0)
_S = np.diag([1, 1j]).astype(np.complex128)
_Z = np.diag([1, -1]).astype(np.complex128)
_I2 = np.eye(2, dtype=np.complex128)

ONE_QUBIT = ("h", "s", "sdg", "i")


def ring_circuit(n: int, depth: int, t_count: int, seed: int):
    """Seeded ring circuit as a list of ops ``(name, qubits)``.

    Single-qubit names: 'h', 's', 'sdg', 't' (identity slots are dropped).
    Two-qubit names: 'cz' (symmetric) and 'cx' (control, target).
    """
    if n < 2 or depth < 1:
        raise ValueError("need n >= 2 and depth >= 1")
    slots = n * depth
    if not 0 <= t_count <= slots:
        raise ValueError("t_count must lie in [0, n*depth]")
    rng = np.random.Generator(np.random.PCG64(seed))
    gates = rng.integers(0, len(ONE_QUBIT), size=(depth, n))
    tpos = np.zeros(slots, dtype=bool)
    tpos[rng.choice(slots, size=t_count, replace=False)] = True
    tpos = tpos.reshape(depth, n)
    two = rng.integers(0, 2, size=(depth, n))
    flip = rng.integers(0, 2, size=(depth, n))
    ops = []
    for layer in range(depth):
        for q in range(n):
            if tpos[layer, q]:
                ops.append(("t", (q,)))
            else:
                g = ONE_QUBIT[gates[layer, q]]
                if g != "i":
                    ops.append((g, (q,)))
        start = layer & 1
        for a in range(start, n - 1 + start, 2):
            b = (a + 1) % n
            if a == b or (start == 0 and a + 1 >= n):
                continue
            if two[layer, a]:
                ops.append(("cz", (a, b)))
            else:
                c, t = (a, b) if flip[layer, a] else (b, a)
                ops.append(("cx", (c, t)))
    return ops


def inject(ops, n: int):
    """T-gadget injection: returns (clifford ops on N qubits, N, natural order, angle per reference)."""
    refs_of = {q: [] for q in range(n)}
    out = []
    k = n
    for name, qs in ops:
        if name == "t":
            q = qs[0]
            out.append(("cx", (q, k)))
            refs_of[q].append(k)
            k += 1
        else:
            out.append((name, qs))
    order = []
    for q in range(n):
        order.append(q)
        order.extend(refs_of[q])
    return out, k, order


class Tableau:
    """Stabilizer rows of an N-qubit state, Aaronson-Gottesman convention."""

    def __init__(self, N: int):
        self.N = N
        self.x = np.zeros((N, N), dtype=np.uint8)
        self.z = np.eye(N, dtype=np.uint8)
        self.r = np.zeros(N, dtype=np.uint8)

    # ---- gates (conjugation of every row) ----
    def h(self, q):
        x, z = self.x, self.z
        self.r ^= x[:, q] & z[:, q]
        tmp = x[:, q].copy(); x[:, q] = z[:, q]; z[:, q] = tmp

    def s(self, q):
        x, z = self.x, self.z
        self.r ^= x[:, q] & z[:, q]
        z[:, q] ^= x[:, q]

    def sdg(self, q):
        x, z = self.x, self.z
        self.r ^= x[:, q] & (1 - z[:, q])
        z[:, q] ^= x[:, q]

    def zgate(self, q):
        self.r ^= self.x[:, q]

    def cx(self, c, t):
        x, z = self.x, self.z
        self.r ^= x[:, c] & z[:, t] & (x[:, t] ^ z[:, c] ^ 1)
        x[:, t] ^= x[:, c]
        z[:, c] ^= z[:, t]

    def cz(self, a, b):
        x, z = self.x, self.z
        self.r ^= x[:, a] & x[:, b] & (z[:, a] ^ z[:, b])
        z[:, a] ^= x[:, b]
        z[:, b] ^= x[:, a]

    def apply(self, ops):
        for name, qs in ops:
            if name == "cz":
                self.cz(*qs)
            elif name == "cx":
                self.cx(*qs)
            elif name == "h":
                self.h(qs[0])
            elif name == "s":
                self.s(qs[0])
            elif name == "sdg":
                self.sdg(qs[0])
            elif name == "z":
                self.zgate(qs[0])
            else:
                raise ValueError(f"not a Clifford op: {name}")
        return self

    # ---- row algebra ----
    def rowsum(self, h, i):
        """Row h <- row i * row h with the exact sign (Aaronson-Gottesman g function)."""
        x1, z1 = self.x[i].astype(np.int64), self.z[i].astype(np.int64)
        x2, z2 = self.x[h].astype(np.int64), self.z[h].astype(np.int64)
        g = np.where((x1 == 1) & (z1 == 1), z2 - x2,
            np.where((x1 == 1) & (z1 == 0), z2 * (2 * x2 - 1),
            np.where((x1 == 0) & (z1 == 1), x2 * (1 - 2 * z2), 0)))
        total = 2 * int(self.r[h]) + 2 * int(self.r[i]) + int(g.sum())
        m = total % 4
        if m not in (0, 2):
            raise AssertionError("rowsum of anticommuting rows")
        self.r[h] = m // 2
        self.x[h] ^= self.x[i]
        self.z[h] ^= self.z[i]

    def swap_rows(self, a, b):
        if a != b:
            for arr in (self.x, self.z):
                arr[[a, b]] = arr[[b, a]]
            self.r[[a, b]] = self.r[[b, a]]


def graph_form(tab: Tableau):
    """(adjacency (N,N) u8, U (N,2,2) c128) with |S> = (U_1 x ... x U_N)|G> up to a global phase."""
    T = Tableau.__new__(Tableau)
    T.N, T.x, T.z, T.r = tab.N, tab.x.copy(), tab.z.copy(), tab.r.copy()
    N = T.N
    # 1. row-reduce the X block; rows below `rank` are Z-only
    rank = 0
    for col in range(N):
        rows = np.nonzero(T.x[rank:, col])[0]
        if rows.size == 0:
            continue
        p = rank + int(rows[0])
        T.swap_rows(rank, p)
        for row in np.nonzero(T.x[:, col])[0]:
            if row != rank:
                T.rowsum(int(row), rank)
        rank += 1
        if rank == N:
            break
    # 2. pivots of the Z-only rows get a Hadamard
    had = np.zeros(N, dtype=np.uint8)
    r2 = rank
    for col in range(N):
        if r2 == N:
            break
        rows = np.nonzero(T.z[r2:, col])[0]
        if rows.size == 0:
            continue
        p = r2 + int(rows[0])
        T.swap_rows(r2, p)
        for row in np.nonzero(T.z[rank:, col])[0]:
            row = int(row) + rank
            if row != r2:
                T.rowsum(row, r2)
        had[col] = 1
        r2 += 1
    for q in np.nonzero(had)[0]:
        T.h(int(q))
    # 3. Gauss-Jordan to X = identity
    for col in range(N):
        rows = np.nonzero(T.x[col:, col])[0]
        if rows.size == 0:
            raise AssertionError("X block not invertible after Hadamards")
        T.swap_rows(col, col + int(rows[0]))
        for row in np.nonzero(T.x[:, col])[0]:
            if row != col:
                T.rowsum(int(row), col)
    if not np.array_equal(T.x, np.eye(N, dtype=np.uint8)):
        raise AssertionError("X block is not the identity")
    # 4. Y diagonals -> S-dagger, signs -> Z
    ydiag = np.diag(T.z).copy()
    for q in np.nonzero(ydiag)[0]:
        T.sdg(int(q))
    sign = T.r.copy()
    for q in np.nonzero(sign)[0]:
        T.zgate(int(q))
    A = T.z.copy()
    if np.any(np.diag(A)) or not np.array_equal(A, A.T) or np.any(T.r):
        raise AssertionError("graph-state reduction failed")
    U = np.empty((N, 2, 2), dtype=np.complex128)
    for q in range(N):
        m = _I2
        if had[q]:
            m = m @ _H
        if ydiag[q]:
            m = m @ _S
        if sign[q]:
            m = m @ _Z
        U[q] = m
    return A.astype(np.uint8), U


def build_ring_instance(n: int, depth: int, t_count: int, seed: int):
    """Seeded ring circuit -> injected graph dictionary (same keys as the reference npz)."""
    ops = ring_circuit(n, depth, t_count, seed)
    cliff, N, natural = inject(ops, n)
    tab = Tableau(N).apply(cliff)
    A, U = graph_form(tab)
    return {
        "graph": A, "unitaries": U, "order": np.asarray(natural, dtype=np.int64),
        "natural_order": np.asarray(natural, dtype=np.int64),
        "ring": np.arange(n, dtype=np.int64), "n": n, "N": N, "ops": ops,
    }
