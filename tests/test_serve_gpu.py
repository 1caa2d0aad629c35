"""Serving loop on the GPU: device-built parameters equal the host bookkeeping, Philox prefixes
equal the host bijection, and every request's samples are identical alone and in a mix."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SMALL = {"c16": "ring16_d20_t24_k8", "c24": "ring24_d24_t60_k10", "c32": "ring32_d37_t79_k14"}


@pytest.fixture(scope="module")
def runners():
    from dcs245_classical_sampling_b200.serve import CircuitRunner
    from dcs245_classical_sampling_b200.workloads import build_workload
    out = {}
    for i, (name, wl) in enumerate(SMALL.items()):
        out[name] = CircuitRunner(name, build_workload(wl), key=0x5EED0000 + i, max_samples=16)
    return out


def test_device_items_equal_host_bookkeeping(runners):
    from dcs245_classical_sampling_b200 import _lib
    lib = _lib.load()
    for name, run in runners.items():
        eng = run.engine
        rng = np.random.default_rng(1)
        xs = [rng.integers(0, 2, eng.n).astype(np.uint8) for _ in range(5)]
        masks = torch.tensor([sum(int(b) << q for q, b in enumerate(x)) for x in xs], dtype=torch.int64).cuda()
        L, S = run.dc.nslices, run.dc.nsteps
        params = torch.empty(len(xs) * L * S * _lib.PARAM_DTYPE.itemsize // 8, dtype=torch.int64, device="cuda")
        coefs = torch.empty(2 * len(xs) * L, dtype=torch.float64, device="cuda")
        xors = torch.empty(len(xs) * L, dtype=torch.int64, device="cuda")
        run.dc.build(lib, masks, len(xs), params, coefs, xors, torch.cuda.current_stream().cuda_stream)
        P = params.cpu().numpy().view(_lib.PARAM_DTYPE).reshape(len(xs), L, S)
        C = coefs.cpu().numpy().reshape(len(xs), L, 2)
        X = xors.cpu().numpy().view(np.uint64).reshape(len(xs), L)
        for i, x in enumerate(xs):
            _, items = eng.params.items(x)
            assert len(items) == L
            for l, (coef, prm, xo) in enumerate(items):
                for f in prm.dtype.names:
                    np.testing.assert_array_equal(P[i, l][f], prm[f], err_msg=f"{name} {f}")
                assert complex(*C[i, l]) == coef
                assert int(X[i, l]) == xo


def test_device_philox_equals_host_bijection(runners):
    from dcs245_classical_sampling_b200 import _lib
    lib = _lib.load()
    run = runners["c24"]
    req = torch.tensor([0, 1, 7, 123456], dtype=torch.int32, device="cuda")
    idx = torch.tensor([0, 5, 63, 2], dtype=torch.int32, device="cuda")
    x = torch.empty(4, dtype=torch.int64, device="cuda")
    u = torch.empty(4, dtype=torch.float64, device="cuda")
    closed = run.dc.closed
    _lib.check(lib.dcs_philox_prefixes(_lib.ptr(req), _lib.ptr(idx), 4, run.key, _lib.ptr(closed),
                                       int(closed.numel()), _lib.ptr(x), _lib.ptr(u),
                                       torch.cuda.current_stream().cuda_stream))
    cl = closed.cpu().tolist()
    for i, (r, j) in enumerate(zip(req.cpu().tolist(), idx.cpu().tolist())):
        c = (ctypes.c_uint32 * 4)(r, j, 0, 0)
        lib.dcs_philox4x32_10_host(c, run.key & 0xffffffff, run.key >> 32)
        bits = (c[1] << 32) | c[0]
        want_x = sum(((bits >> jj) & 1) << q for jj, q in enumerate(cl))
        assert int(x[i]) == want_x
        want_u = ((((c[3] << 32) | c[2]) >> 11) * 2.0 ** -53)
        assert float(u[i]) == want_u


def _records(reqs):
    return {(r.rid, i): rec for r in reqs for i, (rec, x) in r.records.items()}


def test_results_identical_alone_and_in_the_mix(runners):
    from dcs245_classical_sampling_b200.serve import Request, Server
    rng = np.random.default_rng(3)
    names = list(SMALL)
    reqs = [Request(rid, names[rid % 3], int(rng.integers(1, 9)), 0.0) for rid in range(12)]
    mixed = Server(runners).run([Request(r.rid, r.circuit, r.nsamples, 0.0) for r in reqs], realtime=False)
    mix = _records(mixed)
    assert all(r.finish is not None for r in mixed)
    for r in reqs:
        alone = _records(Server(runners).run([Request(r.rid, r.circuit, r.nsamples, 0.0)], realtime=False))
        for i in range(r.nsamples):
            a, m = alone[(r.rid, i)], mix[(r.rid, i)]
            assert a["status"] == 0 and m["status"] == 0
            assert a["index"] == m["index"]
            for f in ("cdf_lower", "cdf_upper", "selected_weight", "total_exact"):
                assert a[f] == pytest.approx(m[f], rel=1e-12, abs=1e-300), f


def test_served_samples_match_the_engine_api(runners):
    """A served sample equals engine.block(x) + draw_checked(u) on the same prefix and uniform."""
    from dcs245_classical_sampling_b200.sampling import draw_checked
    from dcs245_classical_sampling_b200.serve import Request, Server
    run = runners["c32"]
    out = Server({"c32": run}).run([Request(900, "c32", 3, 0.0)], realtime=False)[0]
    import ctypes as ct
    from dcs245_classical_sampling_b200 import _lib
    lib = _lib.load()
    for i, (rec, xmask) in out.records.items():
        x = np.array([(xmask >> q) & 1 for q in range(run.engine.n)], np.uint8)
        c = (ct.c_uint32 * 4)(900, i, 0, 0)
        lib.dcs_philox4x32_10_host(c, run.key & 0xffffffff, run.key >> 32)
        u = ((((c[3] << 32) | c[2]) >> 11) * 2.0 ** -53)
        v, _ = run.engine.block(x)
        d = draw_checked(v, u, hashes=False)
        assert d["A_index"] == rec["index"] or d["cdf_tie"] or rec["tie"]


def test_graph_replay_equals_direct_launches():
    """The batch captured as a CUDA graph (per batch size) gives the same records bit for bit."""
    from dcs245_classical_sampling_b200.serve import CircuitRunner, Request, Server
    from dcs245_classical_sampling_b200.workloads import build_workload
    wl = build_workload(SMALL["c24"])
    direct = CircuitRunner("c24", wl, key=0x5EED0101, max_samples=16)
    graph = CircuitRunner("c24", wl, key=0x5EED0101, max_samples=16, graphs=True)

    def reqs():
        return [Request(rid, "c24", n, 0.0) for rid, n in enumerate([3, 5, 3, 8, 5])]

    a = _records(Server({"c24": direct}).run(reqs(), realtime=False))
    b = _records(Server({"c24": graph}).run(reqs(), realtime=False))
    assert graph._graph  # at least one batch size was captured and replayed
    assert a.keys() == b.keys()
    for key in a:
        assert a[key] == b[key], key


def test_pool_admission_alone_and_in_the_mix():
    """The 32- and 48-qubit serving circuits (2^14 and 2^17 blocks) share one table pool that holds
    at most 9 of the 48-qubit circuit's 128 MiB work items, so its batches are admitted with as
    many items as the pool grants at launch.  Every request's records are the same alone and in
    the mix, and every granted region returns to the pool."""
    from dcs245_classical_sampling_b200.serve import CircuitRunner, Request, Server, TablePool
    from dcs245_classical_sampling_b200.workloads import build_workload
    pool = TablePool(int(1.2 * 2 ** 30), "cuda")
    runners = {"c32": CircuitRunner("c32", build_workload("ring32_d37_t79_k14"), key=0x5EED0201, max_samples=16,
                                    pool=pool),
               "c48": CircuitRunner("c48", build_workload("ring48_d55_t177_k17"), key=0x5EED0202, max_samples=16,
                                    pool=pool)}
    assert runners["c48"].item_bytes == 8 << 24 and runners["c48"].table_bytes() == 0
    rng = np.random.default_rng(8)
    reqs = [Request(rid, ("c32", "c48")[rid % 2], int(rng.integers(1, 13)), 0.0) for rid in range(8)]
    mixed = Server(runners, pool).run([Request(r.rid, r.circuit, r.nsamples, 0.0) for r in reqs], realtime=False)
    assert pool.free == [(0, pool.nbytes)]
    mix = _records(mixed)
    for r in reqs:
        alone = _records(Server(runners, pool).run([Request(r.rid, r.circuit, r.nsamples, 0.0)], realtime=False))
        for i in range(r.nsamples):
            a, m = alone[(r.rid, i)], mix[(r.rid, i)]
            assert a["status"] == 0 and m["status"] == 0
            assert a["index"] == m["index"]
            for f in ("cdf_lower", "cdf_upper", "selected_weight", "total_exact"):
                assert a[f] == pytest.approx(m[f], rel=1e-12, abs=1e-300), f
    assert pool.free == [(0, pool.nbytes)]


def test_pool_refuses_a_circuit_larger_than_the_budget():
    from dcs245_classical_sampling_b200.serve import CircuitRunner, TablePool
    from dcs245_classical_sampling_b200.workloads import build_workload
    pool = TablePool(64 << 20, "cuda")
    with pytest.raises(ValueError, match="exceeds the HBM budget"):
        CircuitRunner("c48", build_workload("ring48_d55_t177_k17"), key=1, max_samples=4, pool=pool)
    with pytest.raises(ValueError, match="exceeds the HBM budget"):
        CircuitRunner("c48", build_workload("ring48_d55_t177_k17"), key=1, max_samples=4, hbm_budget=64 << 20)
