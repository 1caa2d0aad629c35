"""Seeded ring circuits and the stabilizer -> graph-state form, checked by dense simulation."""
import math

import numpy as np
import pytest

from dcs245_classical_sampling_b200.circuits import Tableau, graph_form, inject, ring_circuit

_H = np.array([[1, 1], [1, -1]]) / math.sqrt(2)
GATES = {"h": _H, "s": np.diag([1, 1j]), "sdg": np.diag([1, -1j]), "t": np.diag([1, np.exp(1j * math.pi / 4)]),
         "z": np.diag([1, -1])}


def apply1(psi, N, q, M):
    psi = np.moveaxis(psi.reshape([2] * N), N - 1 - q, 0)
    psi = np.tensordot(M, psi, axes=(1, 0))
    return np.moveaxis(psi, 0, N - 1 - q).reshape(-1)


def dense(ops, N):
    psi = np.zeros(2 ** N, complex)
    psi[0] = 1
    idx = np.arange(2 ** N)
    for name, qs in ops:
        if name == "cz":
            a, b = qs
            psi = psi * (1 - 2 * (((idx >> a) & 1) & ((idx >> b) & 1)))
        elif name == "cx":
            c, t = qs
            psi = psi[idx ^ (((idx >> c) & 1) << t)]
        else:
            psi = apply1(psi, N, qs[0], GATES[name])
    return psi


def graph_dense(A, U):
    N = len(A)
    idx = np.arange(2 ** N)
    ph = np.zeros(2 ** N, int)
    for a in range(N):
        for b in range(a + 1, N):
            if A[a, b]:
                ph ^= ((idx >> a) & 1) & ((idx >> b) & 1)
    psi = (1 - 2 * ph) / 2 ** (N / 2) + 0j
    for q in range(N):
        psi = apply1(psi, N, q, U[q])
    return psi


@pytest.mark.parametrize("seed", range(8))
def test_graph_form_equals_dense_state(seed):
    n, d, t = 4 + seed % 3, 3 + seed % 4, 2 + seed % 5
    ops = ring_circuit(n, d, t, seed)
    cl, N, _ = inject(ops, n)
    assert N <= 14
    A, U = graph_form(Tableau(N).apply(cl))
    a, b = dense(cl, N), graph_dense(A, U)
    ov = abs(np.vdot(a, b))
    assert ov == pytest.approx(1.0, abs=1e-12)


def test_t_count_and_layer_rule():
    ops = ring_circuit(16, 20, 24, 1016)
    assert sum(1 for g, _ in ops if g == "t") == 24
    two = [(g, q) for g, q in ops if g in ("cz", "cx")]
    assert len(two) == 20 * 8  # 8 pairs per layer on a 16-ring
    for g, q in two:
        a, b = sorted(q)
        assert b - a == 1 or (a, b) == (0, 15)
