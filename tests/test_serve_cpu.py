"""Host-side serving logic: chunking of (sample, slice) items and request generation."""
import types

from dcs245_classical_sampling_b200.serve import CircuitRunner, poisson_requests


def _fake(L, cap):
    r = types.SimpleNamespace(dc=types.SimpleNamespace(nslices=L), engine=types.SimpleNamespace(items=cap))
    return lambda n: CircuitRunner._chunks(r, n)


def test_chunks_cover_every_item_once_in_slice_order():
    for L in (1, 2, 4):
        for cap in (1, 2, 3, 4, 8, 16):
            for n in (1, 2, 5, 9):
                chunks, begins = _fake(L, cap)(n)
                seen = []
                for c0, cn, b0, nb, boff in chunks:
                    bl = begins[boff:boff + nb + 1]
                    assert bl[0] == 0 and bl[-1] == cn and all(x < y for x, y in zip(bl, bl[1:]))
                    for j in range(nb):
                        for it in range(bl[j], bl[j + 1]):
                            item = c0 + it
                            assert item // L == b0 + j  # the item belongs to that block
                            seen.append(item)
                assert seen == list(range(n * L))


def test_poisson_requests_are_seeded():
    a = poisson_requests(50.0, 2.0, {"x": 5, "y": 3, "z": 2}, seed=4)
    b = poisson_requests(50.0, 2.0, {"x": 5, "y": 3, "z": 2}, seed=4)
    assert [(r.arrival, r.circuit, r.nsamples) for r in a] == [(r.arrival, r.circuit, r.nsamples) for r in b]
    assert all(1 <= r.nsamples <= 64 for r in a) and len(a) > 50
