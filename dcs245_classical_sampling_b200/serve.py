"""Device-resident serving loop: sampling requests against several circuits at once.

Requests ask for 1..64 samples of one circuit.  Per circuit a ``CircuitRunner`` owns an engine
(contraction tables sized from its share of the HBM budget), a CUDA stream and the circuit's
static parameter tables on the device.  A batch of samples runs entirely on the device:

  Philox4x32-10 prefixes + uniforms -> per-(sample, slice) parameters (dcs_build_items)
  -> contraction (per-step batched kernels, or the fused kernel for large tables)
  -> slice accumulation -> Walsh-Hadamard/phase/U_open tail -> FP64 CDF draw

and only the draw records (96 bytes per sample) come back.  The ``Server`` does continuous
batching: arriving requests are admitted into their circuit's active set; whenever a runner's
previous batch has finished it takes the next samples round-robin over the active requests of
its circuit (one sample of each in turn, up to its slot count), so work of different requests
shares launches, a large request is split over many batches instead of holding the runner, and
the runners of different circuits overlap on the device through their streams.  A sample's
result depends only on (circuit, request id, sample index, key), never on what it was batched
with.

Admission by HBM budget: with a ``TablePool`` the contraction tables are not owned by the
runners.  The pool holds the budget's device memory; a batch is launched only when the pool
grants it a region for at least one work item (slice) of its circuit, and the region returns
to the pool when the batch's records are back, so memory that one circuit frees admits the
work of another (the 64-qubit circuit's 128 GiB table is granted per batch, not held).  Large
regions are granted from the front of the pool and small ones from the back, and while a
large request waits no small batch takes memory from the front.

Latency of a request = completion time - arrival time (host clock); p50/p99 over requests.
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .engine import InplaceConditionalBlockGPU


class DeviceCircuit:
    """Static tables of one circuit for dcs_build_items (from the engine's host bookkeeping)."""

    def __init__(self, engine, device):
        sp = engine.params
        p = engine.plan
        S = sp.nsteps
        fsel = np.zeros((S, 8), np.float64)
        xq = np.full(S, -1, np.int32)
        fixidx = np.full(S, -1, np.int32)
        ffull_ref = sp.full_vectors(np.zeros(p.n, np.int64))  # reference vertices do not depend on x
        for j in range(S):
            q = int(sp.keep[sp.vert[j]])
            if q < p.n:
                for b in (0, 1):
                    row = sp.U[q, b]
                    fsel[j, 4 * b:4 * b + 4] = [row[0].real, row[0].imag, row[1].real, row[1].imag]
                xq[j] = q
            else:
                f = ffull_ref[q]
                fsel[j, 0:4] = fsel[j, 4:8] = [f[0].real, f[0].imag, f[1].real, f[1].imag]
        for a, j in enumerate(sp.fixed_pos):
            fixidx[j] = a
        nfixed = len(sp.fixed_pos)
        fwords = (S + 31) // 32
        F = np.zeros((max(1, nfixed), fwords), np.uint32)
        for a in range(nfixed):
            for t in np.flatnonzero(sp.F[a]):
                F[a, t >> 5] |= np.uint32(1 << (t & 31))
        tail = np.array([int(x) for x in sp.tail] + [0], np.uint64)
        # slices: x-independent coefficients (slices are reference vertices) and flips
        _, items = sp.items(np.zeros(p.n, np.uint8))
        # items skip zero coefficients; recover each kept slice's flips from its bits
        import itertools
        flips, coefs, freeflips = [], [], []
        ff = ffull_ref
        for bits in itertools.product((0, 1), repeat=sp.nslice):
            bits = np.array(bits, np.int64)
            coef = complex(np.prod([ff[s][b] for s, b in zip(p.slices, bits)])) if sp.nslice else 1 + 0j
            par = sum(int(bits[p.slices.index(a)]) * int(bits[p.slices.index(b)]) for a, b in p.slice_edges)
            coef *= (-1) ** par
            if not coef:
                continue
            fl = (bits @ sp.nbr) & 1 if sp.nslice else np.zeros(p.N, np.int64)
            flips.append(fl[sp.vert].astype(np.uint8))
            coefs.append(coef)
            freeflips.append(sum(int(fl[q]) << jj for jj, q in enumerate(sp.open_red)))
        self.nslices = len(coefs)
        assert self.nslices == len(items)
        # the plan-specialised kernels divide f0 out of the free steps' weights: every weight row
        # a prefix can select (slices flip only f1) must pass the engine's check
        rows = np.zeros(2 * S, _lib.PARAM_DTYPE)
        for b in (0, 1):
            rows["f0r"][b::2], rows["f0i"][b::2] = fsel[:, 4 * b], fsel[:, 4 * b + 1]
            rows["f1r"][b::2], rows["f1i"][b::2] = fsel[:, 4 * b + 2], fsel[:, 4 * b + 3]
        self.unit_ok = all(engine.unit_weights_ok(rows[b::2]) for b in (0, 1))
        self.nsteps, self.nfixed = S, nfixed
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.fsel = dev(fsel)
        self.xq = dev(xq)
        self.fixidx = dev(fixidx)
        self.flip = dev(np.stack(flips).astype(np.uint8))
        self.F = dev(F)
        self.tail = dev(tail.view(np.int64))
        self.coef = dev(np.array([[c.real, c.imag] for c in coefs], np.float64).reshape(-1))
        self.freeflip = dev(np.array(freeflips, np.uint64).view(np.int64))
        self.closed = dev(np.array([q for q in range(p.n) if q not in set(p.open_full)], np.int32))

    def build(self, lib, xbits, nsamples, params, coefs, xors, stream):
        _lib.check(lib.dcs_build_items(
            _lib.ptr(self.fsel), _lib.ptr(self.xq), _lib.ptr(self.fixidx), _lib.ptr(self.flip), _lib.ptr(self.F),
            _lib.ptr(self.tail), _lib.ptr(self.coef), _lib.ptr(self.freeflip), self.nsteps, self.nfixed,
            self.nslices, _lib.ptr(xbits), nsamples, _lib.ptr(params), _lib.ptr(coefs), _lib.ptr(xors), stream))


class TablePool:
    """One device buffer of `nbytes` (the HBM budget for contraction tables), granted to batches
    as byte regions.  Regions of `large` bytes or more are granted first-fit from the front,
    smaller ones from the back; freed regions merge with their neighbours.  `front_reserved`
    bytes at the front are kept from small grants (set while a large request waits)."""

    ALIGN = 256

    def __init__(self, nbytes, device, large=1 << 34):
        self.nbytes = int(nbytes) // self.ALIGN * self.ALIGN
        self.device = torch.device(device) if not isinstance(device, torch.device) else device
        self.buf = torch.empty(self.nbytes, dtype=torch.uint8, device=self.device)
        self.free = [(0, self.nbytes)]  # sorted, disjoint (start, end)
        self.large = int(large)
        self.front_reserved = 0

    def size(self, nbytes):
        return -(-int(nbytes) // self.ALIGN) * self.ALIGN

    def alloc(self, nbytes):
        """A region (start, end) of at least `nbytes`, or None if no free run is large enough."""
        size = self.size(nbytes)
        if size <= 0 or size > self.nbytes:
            return None
        if size >= self.large:
            for i, (s, e) in enumerate(self.free):
                if e - s >= size:
                    if s + size == e:
                        del self.free[i]
                    else:
                        self.free[i] = (s + size, e)
                    return (s, s + size)
            return None
        for i in range(len(self.free) - 1, -1, -1):
            s, e = self.free[i]
            if e - max(s, self.front_reserved) >= size:
                if e - size == s:
                    del self.free[i]
                else:
                    self.free[i] = (s, e - size)
                return (e - size, e)
        return None

    def release(self, region):
        self.free.append(tuple(region))
        self.free.sort()
        merged = []
        for a, b in self.free:
            if merged and merged[-1][1] == a:
                merged[-1] = (merged[-1][0], b)
            else:
                merged.append((a, b))
        self.free = merged

    def free_bytes(self):
        return sum(e - s for s, e in self.free)

    def view(self, region):
        s, e = region
        return self.buf[s:e]


@dataclass
class Batch:
    samples: list            # (request id, sample index)
    event: torch.cuda.Event
    host: torch.Tensor       # pinned draw records
    xbits: torch.Tensor      # pinned prefix masks
    launched: float
    region: tuple = None     # pool region holding the batch's tables


class CircuitRunner:
    """One circuit: engine, stream, device tables, in-flight batch buffers."""

    def __init__(self, name, workload, key, max_samples, device=0, mode=None, hbm_budget=None, graphs=False,
                 pool=None):
        """graphs=True: the device work of a batch (prefixes, parameters, contraction, accumulation,
        tail, draw) is captured once per batch size as a CUDA graph and replayed.
        pool: a TablePool that grants the batch's tables per batch (admission by HBM budget);
        without one the runner owns tables of `hbm_budget` bytes at most (default: one batch)."""
        self.name, self.key = name, int(key)
        self.graphs = bool(graphs)
        self._graph = {}
        self.pool = pool
        if pool is not None and self.graphs:
            raise ValueError("CUDA graphs capture fixed table addresses: use runner-owned tables (no pool)")
        w = workload
        self.device = torch.device("cuda", device)
        self.engine = InplaceConditionalBlockGPU(w["graph"], w["unitaries"], w["n"], w["order"],
                                                 w["parity_operations"], w["open_vertices"])
        big = self.engine.plan.maxslots >= 30
        self.mode = mode or ("fused" if big else "device")
        L = len(self.engine.params.items(np.zeros(w["n"], np.uint8))[1])
        entry = 8 << self.engine.plan.maxslots
        if self.mode == "fused":
            items = 1
        elif pool is not None:
            items = max_samples * L
        else:
            fit = int(hbm_budget // entry) if hbm_budget is not None else max_samples * L
            items = max(1, min(max_samples * L, fit))
        if pool is not None and pool.size(entry) > pool.nbytes:
            raise ValueError(f"{name}: one work item's table ({entry / 2**30:.3g} GiB) exceeds the HBM budget "
                             f"({pool.nbytes / 2**30:.3g} GiB)")
        if pool is None and hbm_budget is not None and entry > hbm_budget:
            raise ValueError(f"{name}: one work item's table ({entry / 2**30:.3g} GiB) exceeds the HBM budget "
                             f"({hbm_budget / 2**30:.3g} GiB)")
        self.engine.alloc(np.complex64, device=device, mode=self.mode, items=items,
                          external_table=pool is not None)
        self.item_bytes = self.engine.table_item_bytes()
        self.lib = _lib.load()
        self.dc = DeviceCircuit(self.engine, self.device)
        assert self.dc.nslices == L
        if self.mode == "fused" and self.engine.jit and not self.dc.unit_ok:
            self.engine.set_fused_config(jit=False)  # weights the plan-specialised kernels cannot take
        self.max_samples = max_samples if self.mode == "fused" else max(1, min(max_samples, items // L) or 1)
        self.k = self.engine.k
        self.stream = torch.cuda.Stream(self.device)
        M = self.max_samples
        dev = self.device
        self.d_ids = torch.empty(2 * M, dtype=torch.int32, device=dev)
        self.d_x = torch.empty(M, dtype=torch.int64, device=dev)
        self.d_u = torch.empty(M, dtype=torch.float64, device=dev)
        self.d_params = torch.empty(M * L * self.dc.nsteps * _lib.PARAM_DTYPE.itemsize // 8, dtype=torch.int64,
                                    device=dev)
        self.d_coefs = torch.empty(2 * M * L, dtype=torch.float64, device=dev)
        self.d_xors = torch.empty(M * L, dtype=torch.int64, device=dev)
        self.d_begin = torch.empty(4 * M * L + 8, dtype=torch.int32, device=dev)
        self.d_out = torch.empty((M, 1 << self.k), dtype=torch.complex128, device=dev)
        self.d_res = torch.empty(M * _lib.DRAW_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.d_scratch = torch.empty(self.lib.dcs_draw_scratch_bytes(self.k, M), dtype=torch.uint8, device=dev)

    def table_bytes(self):
        """Device bytes of the tables the runner owns (0 with a pool: tables are granted per batch)."""
        t = self.engine.table
        return 0 if self.pool is not None or t is None else t.numel() * t.element_size()

    def grant(self, n):
        """Tables for a batch of n samples: with a pool, the largest region of up to n x slices work
        items it grants now, bound to the engine (None if not even one item fits); without a pool,
        the runner's own tables."""
        if self.pool is None:
            return ()
        L = self.dc.nslices
        want = n * L if self.mode != "fused" else 1
        items = want
        while items >= 1:
            region = self.pool.alloc(items * self.item_bytes)
            if region is not None:
                self.engine.bind_table(self.pool.view(region), items)
                return region
            items //= 2
        return None

    def _chunks(self, n):
        """Launch chunks of engine.items work items and, per chunk, the item ranges of its blocks."""
        L, cap = self.dc.nslices, self.engine.items
        items = n * L
        chunks, begins = [], []
        for c0 in range(0, items, cap):
            cn = min(cap, items - c0)
            b0, b1 = c0 // L, (c0 + cn - 1) // L
            bl = [0] + [min((b + 1) * L, c0 + cn) - c0 for b in range(b0, b1 + 1)]
            chunks.append((c0, cn, b0, b1 - b0 + 1, len(begins)))
            begins.extend(bl)
        return chunks, begins

    def _device_work(self, n, chunks):
        """Every device step of a batch of n samples after the id upload, on self.stream, with
        fixed buffers only (so that it can be captured as a CUDA graph)."""
        eng, lib = self.engine, self.lib
        st = self.stream.cuda_stream
        _lib.check(lib.dcs_philox_prefixes(_lib.ptr(self.d_ids), _lib.ptr(self.d_ids) + 4 * n, n, self.key,
                                           _lib.ptr(self.dc.closed), int(self.dc.closed.numel()),
                                           _lib.ptr(self.d_x), _lib.ptr(self.d_u), st))
        self.dc.build(lib, self.d_x, n, self.d_params, self.d_coefs, self.d_xors, st)
        out = self.d_out[:n]
        out.zero_()
        entry = _lib.PARAM_DTYPE.itemsize
        nm = eng._nmax() + 1
        for c0, cn, b0, nb, boff in chunks:
            eng._reset_items(cn)
            eng._run_steps(_lib.ptr(self.d_params) + c0 * eng.nsteps * entry, cn)
            _lib.check(lib.dcs_accumulate_batched(
                eng.dcode, _lib.ptr(eng.table), eng.table_stride, eng.plan.terminal_rank,
                eng.term_runs.ctypes.data, eng.term_nruns, eng.tbasis.ctypes.data,
                _lib.ptr(self.d_xors) + 8 * c0, _lib.ptr(self.d_coefs) + 16 * c0,
                _lib.ptr(self.d_begin) + 4 * boff, nb, eng.params.shift, _lib.ptr(eng.scale),
                _lib.ptr(eng.maxbits[nm - 1:]), nm, _lib.ptr(out[b0:b0 + nb]), self.k, cn, st))
        _lib.check(lib.dcs_block_tail(_lib.ptr(out), self.k, eng.adj_hi.ctypes.data, eng.u_open.ctypes.data, n, st))
        _lib.check(lib.dcs_draw(_lib.ptr(out), self.k, n, _lib.ptr(self.d_u), _lib.ptr(self.d_scratch),
                                _lib.ptr(self.d_res), st))

    def _replay(self, n, chunks):
        g = self._graph.get(n)
        if g is None:
            # one direct run first (kernel attributes, allocator), then the capture
            self._device_work(n, chunks)
            self.stream.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=self.stream):
                self._device_work(n, chunks)
            self._graph[n] = g
        g.replay()

    def precapture(self, sizes):
        """Capture the batch graphs of the given batch sizes ahead of serving (graphs=True)."""
        if not self.graphs:
            return
        with torch.cuda.stream(self.stream):
            for n in sizes:
                if n in self._graph or not 0 < n <= self.max_samples:
                    continue
                chunks, begins = self._chunks(n)
                self.d_begin[:len(begins)].copy_(torch.tensor(begins, dtype=torch.int32), non_blocking=False)
                self.d_ids[:2 * n].zero_()
                self._replay(n, chunks)
        self.stream.synchronize()

    def launch(self, samples, region=()):
        """Enqueue one batch (list of (request id, sample index)) on the tables of `region` (from
        grant); returns a Batch."""
        n = len(samples)
        assert 0 < n <= self.max_samples
        chunks, begins = self._chunks(n)
        with torch.cuda.stream(self.stream):
            ids = torch.tensor([s[0] for s in samples] + [s[1] for s in samples] + begins,
                               dtype=torch.int32).pin_memory()
            self.d_begin[:len(begins)].copy_(ids[2 * n:], non_blocking=True)
            self.d_ids[:2 * n].copy_(ids[:2 * n], non_blocking=True)
            if self.graphs:
                self._replay(n, chunks)
            else:
                self._device_work(n, chunks)
            host = torch.empty(n * _lib.DRAW_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
            host.copy_(self.d_res[:n * _lib.DRAW_DTYPE.itemsize], non_blocking=True)
            hx = torch.empty(n, dtype=torch.int64).pin_memory()
            hx.copy_(self.d_x[:n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self._hold = ids  # the pinned upload must outlive its copy
        return Batch(list(samples), ev, host, hx, time.perf_counter(), region or None)


@dataclass
class Request:
    rid: int
    circuit: str
    nsamples: int
    arrival: float
    done: int = 0
    finish: float = None
    records: dict = field(default_factory=dict)


class Server:
    """Continuous batching over several CircuitRunners (see the module docstring).

    pool: the TablePool the runners were built with, if any (batches then launch only when it
    grants their tables, and give them back when their records are in)."""

    def __init__(self, runners, pool=None):
        self.runners = dict(runners)
        self.pool = pool

    @staticmethod
    def _pick(active, m):
        """Up to m samples round-robin over the active requests [request, next index] (one of each
        in turn); returns the samples and the new next indices, without changing `active`."""
        take, nxt = [], {id(a): a[1] for a in active}
        progress = True
        while len(take) < m and progress:
            progress = False
            for a in active:
                r = a[0]
                if nxt[id(a)] < r.nsamples and len(take) < m:
                    take.append((r.rid, nxt[id(a)]))
                    nxt[id(a)] += 1
                    progress = True
        return take, nxt

    def run(self, requests, realtime=True, poll_sleep=0.0005):
        """Serve `requests` (arrival times in seconds from start).  Returns the requests with
        their per-sample draw records and completion times."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        by_id = {r.rid: r for r in reqs}
        pending = collections.deque(reqs)
        active = {c: [] for c in self.runners}
        inflight = {c: None for c in self.runners}
        t0 = time.perf_counter()
        remaining = len(reqs)
        while remaining:
            now = time.perf_counter() - t0
            while pending and (pending[0].arrival <= now or not realtime):
                r = pending.popleft()
                active[r.circuit].append([r, 0])
            progressed = False
            for c, run in self.runners.items():
                b = inflight[c]
                if b is not None and b.event.query():
                    recs = b.host.numpy().view(_lib.DRAW_DTYPE)
                    xs = b.xbits.numpy()
                    tnow = time.perf_counter() - t0
                    for (rid, idx), rec, x in zip(b.samples, recs, xs):
                        r = by_id[rid]
                        r.records[idx] = (rec.copy(), int(x))
                        r.done += 1
                        if r.done == r.nsamples:
                            r.finish = tnow
                            remaining -= 1
                    if b.region is not None:
                        self.pool.release(b.region)
                    inflight[c] = None
                    progressed = True
            for c, run in self.runners.items():
                if inflight[c] is not None or not active[c]:
                    continue
                take, nxt = self._pick(active[c], run.max_samples)
                region = run.grant(len(take))
                if region is None:  # no HBM for this circuit now: wait for a batch to give some back
                    if self.pool is not None and run.item_bytes >= self.pool.large:
                        self.pool.front_reserved = self.pool.size(run.item_bytes)
                    continue
                if self.pool is not None and run.item_bytes >= self.pool.large:
                    self.pool.front_reserved = 0
                if run.pool is not None and run.mode != "fused":  # the granted items bound the batch
                    cap = max(1, run.engine.items // run.dc.nslices)
                    if cap < len(take):
                        take, nxt = self._pick(active[c], cap)
                for a in active[c]:
                    a[1] = nxt[id(a)]
                active[c] = [a for a in active[c] if a[1] < a[0].nsamples]
                inflight[c] = run.launch(take, region)
                progressed = True
            if not progressed:
                if pending and realtime:
                    time.sleep(min(poll_sleep, max(0.0, pending[0].arrival - (time.perf_counter() - t0))))
                else:
                    time.sleep(poll_sleep)
        return reqs


def poisson_requests(rate_hz, duration_s, mix, seed=0, max_samples=64, rid0=0):
    """Poisson arrivals; circuit chosen by `mix` {name: weight}; 1..max_samples samples each."""
    rng = np.random.default_rng(seed)
    names = list(mix)
    w = np.array([mix[n] for n in names], np.float64)
    w /= w.sum()
    out, t, rid = [], 0.0, rid0
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t > duration_s:
            break
        out.append(Request(rid, names[rng.choice(len(names), p=w)], int(rng.integers(1, max_samples + 1)), t))
        rid += 1
    return out


def latency_stats(reqs):
    lat = np.array([(r.finish - r.arrival) * 1e3 for r in reqs if r.finish is not None])
    return {"requests": int(len(lat)), "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None}
