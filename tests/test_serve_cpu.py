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


def _req(rid, n):
    from dcs245_classical_sampling_b200.serve import Request
    return Request(rid, "c", n, 0.0)


def test_round_robin_splits_large_requests():
    """A batch takes one sample of each active request in turn, so a 64-sample request does not
    hold the runner: a 1-sample request behind it is in the first batch."""
    from dcs245_classical_sampling_b200.serve import Server
    big, small, mid = _req(1, 64), _req(2, 1), _req(3, 3)
    active = [[big, 0], [small, 0], [mid, 0]]
    take, nxt = Server._pick(active, 4)
    assert take == [(1, 0), (2, 0), (3, 0), (1, 1)]
    assert [a[1] for a in active] == [0, 0, 0]  # _pick does not change the active set
    assert nxt[id(active[0])] == 2 and nxt[id(active[1])] == 1 and nxt[id(active[2])] == 1
    take, _ = Server._pick([[big, 60], [mid, 2]], 8)
    assert take == [(1, 60), (3, 2), (1, 61), (1, 62), (1, 63)]
    take, _ = Server._pick([[big, 0]], 1)
    assert take == [(1, 0)]


def test_table_pool_front_back_merge_and_reservation():
    from dcs245_classical_sampling_b200.serve import TablePool
    KB = 1024
    pool = TablePool(1000 * KB, "cpu", large=400 * KB)
    big = pool.alloc(500 * KB)
    assert big == (0, 500 * KB)  # large regions from the front
    s1 = pool.alloc(100 * KB)
    s2 = pool.alloc(100 * KB)
    assert s1[1] == pool.nbytes and s2[1] == s1[0]  # small regions from the back
    assert pool.alloc(500 * KB) is None  # only 300 KB left
    pool.release(big)
    assert pool.alloc(100 * KB) == (s2[0] - 100 * KB, s2[0])
    # a waiting large request keeps small grants off the front
    pool.front_reserved = pool.size(500 * KB)
    assert pool.alloc(250 * KB) is None
    small = pool.alloc(90 * KB)
    assert small is not None and small[0] >= 500 * KB
    for r in (s1, s2, small):
        pool.release(r)
    pool.release((s2[0] - 100 * KB, s2[0]))
    assert pool.free == [(0, pool.nbytes)]  # every release merged back
    assert pool.free_bytes() == pool.nbytes
    assert pool.alloc(pool.nbytes + 1) is None and pool.alloc(0) is None
    assert pool.view((256, 512)).numel() == 256
