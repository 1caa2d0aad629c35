"""The reference's gather engine on the B200: drop-in for ``ConditionalBlockGPU``
(``source/sampling/conditional_block_gpu.py:25-177``), whose executor is the two-table gather
kernel ``scan_step_scaled`` (``source/dcs_rankwidth/gpu_kernel.py:58-170``).

The reference's production engine is the in-place one (``engine.InplaceConditionalBlockGPU``); this
engine keeps its second one: same constructor, ``alloc(dtype, device)``, ``block(x_bits, w=None,
part=0, parts=1) -> (vector, meta)``, attributes (``rmax``, ``work``, ``steps``, ``tables``,
``combos``, ``terminal_basis``, ``rank_profile``) and errors.  The plan is the gather form
(``plan.build_gather_plan``, bit-exact with ``scan_plan.make_plan``).  Per block, every slice runs all
its steps on the device (``dcs_gather_steps``: FP64 sums, renormalisation on the device, no host
sync), then the slice accumulation and the Walsh-Hadamard/phase/U_open tail are the in-place
engine's kernels (the terminal entries are the first 2^terminal_rank of the final table).  Tables:
two of 2^rmax entries per work item, complex64 or complex128 (the reference's complex128 route needs a
file it does not ship; here both storages run the same kernel).
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from .engine import DeviceBlock, SliceParams, pack_runs
from .plan import build_block_plan, build_gather_plan


class ConditionalBlockGPU:
    """Drop-in for the reference's gather engine (see the module docstring)."""

    def __init__(self, graph, unitaries, n, order, parity_operations, open_vertices):
        bp = self.plan = build_block_plan(graph, unitaries, n, order, parity_operations, open_vertices)
        gp = self.gplan = build_gather_plan(bp)
        # the reference's attribute surface (conditional_block_gpu.py:25-69)
        self.N_full, self.n, self.N = bp.N_full, bp.n, bp.N
        self.open_full, self.open_red = bp.open_full, bp.open_red
        self.slices, self.slice_edges, self.nbrs_in_keep = bp.slices, bp.slice_edges, bp.nbrs_in_keep
        self.relabel, self.keep, self.U_full = bp.relabel, bp.keep, bp.U_full
        self.edges, self.order, self.fixed, self.fut, self.stop = bp.edges, bp.order, bp.fixed, bp.fut, bp.stop
        self.steps, self.rank_profile, self.tables, self.combos = gp.steps, gp.rank_profile, gp.tables, gp.combos
        self.rmax, self.work = gp.rmax, gp.work
        self.terminal_basis = gp.terminal_basis
        self.terminal_rank = len(gp.terminal_basis)
        self.open_edges = bp.open_edges
        self.params = SliceParams(bp)
        self.k = len(bp.open_full)
        self._alloc = False

    def alloc(self, dtype=np.complex64, device=0, fp64_kernel_path=None, items=None, hbm_budget=None):
        """Two tables of 2^rmax entries per work item (conditional_block_gpu.py:71-90,
        gpu_kernel.py:111-123); items: work items (slices) per launch, default as many slices as fit
        in 85% of free device memory.  fp64_kernel_path is accepted for the reference's signature and
        unused: complex128 runs the same kernel."""
        if np.dtype(dtype) not in (np.dtype(np.complex64), np.dtype(np.complex128)):
            raise ValueError(dtype)
        if not torch.cuda.is_available():
            raise RuntimeError("ConditionalBlockGPU needs a CUDA device")
        self.lib = _lib.load()
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self.use_fp64 = np.dtype(dtype) == np.dtype(np.complex128)
        self.dcode = _lib.C128 if self.use_fp64 else _lib.C64
        tdtype = torch.complex128 if self.use_fp64 else torch.complex64
        entry = 16 if self.use_fp64 else 8
        size = 1 << self.rmax
        nslice = 1 << len(self.slices)
        if items is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget = int(hbm_budget if hbm_budget is not None else 0.85 * free)
            items = max(1, min(nslice, budget // (2 * size * entry)))
        self.items = int(items)
        self.stride = size
        self.tab = [torch.zeros(self.items * size, dtype=tdtype, device=self.device) for _ in range(2)]
        # per-step descriptors (host) and their byte tables and kernel combinations (device)
        S = len(self.steps)
        self.dsteps = np.zeros(S, dtype=_lib.GATHER_STEP_DTYPE)
        words = []
        off = 0
        for j, st in enumerate(self.steps):
            T = self.tables[j].reshape(-1)
            C = np.asarray(self.combos[j], np.uint64)
            d = self.dsteps[j]
            d["beta"], d["r_in"], d["r_out"], d["free_"] = st.beta, st.r_in, st.r_out, int(st.free)
            d["nbytes"], d["ncombos"] = self.tables[j].shape[0], len(C)
            d["table_off"], d["combo_off"] = off, off + T.size
            words.extend([T, C])
            off += T.size + C.size
        self.words = torch.from_numpy(np.concatenate(words).view(np.int64)).to(self.device)
        self.nm = S + 1
        self.maxbits = torch.zeros(self.items * self.nm, dtype=torch.int64, device=self.device)
        self.scale = torch.zeros(self.items * _lib.SCALE_DTYPE.itemsize // 8, dtype=torch.int64, device=self.device)
        self.one_bits = (int(np.array([1.0], np.float64).view(np.int64)[0]) if self.use_fp64
                         else int(np.array([1.0], np.float32).view(np.uint32)[0]))
        self.term_runs, self.term_nruns = pack_runs(list(range(self.terminal_rank)))
        self.tbasis = np.array(self.terminal_basis + [0], dtype=np.uint64)
        adj = np.zeros(max(1, self.k), dtype=np.uint32)
        for a, b in self.open_edges:
            lo, hi = (a, b) if a < b else (b, a)
            adj[lo] |= np.uint32(1 << hi)
        self.adj_hi = adj
        u = np.zeros((max(1, self.k), 8), dtype=np.float64)
        for q, orig in enumerate(self.open_full):
            m = np.asarray(self.U_full[orig], np.complex128)
            u[q] = [m[0, 0].real, m[0, 0].imag, m[0, 1].real, m[0, 1].imag,
                    m[1, 0].real, m[1, 0].imag, m[1, 1].real, m[1, 1].imag]
        self.u_open = u
        self._alloc = True

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def block(self, x_bits, w=None, part=0, parts=1):
        """Scaled conditional amplitudes of one prefix (conditional_block_gpu.py:128-177)."""
        if not self._alloc:
            self.alloc()
        start = time.perf_counter()
        count, items = self.params.items(x_bits, w, part, parts)
        lib, st = self.lib, self._stream()
        out = torch.zeros((1, 1 << self.k), dtype=torch.complex128, device=self.device)
        flags = torch.zeros(self.items, dtype=torch.int64, device=self.device)
        S = len(self.steps)
        final = self.tab[S & 1]  # step s reads table s % 2
        sw = _lib.SCALE_DTYPE.itemsize // 8
        for c0 in range(0, len(items), self.items):
            chunk = items[c0:c0 + self.items]
            cn = len(chunk)
            host = np.concatenate([it[1] for it in chunk]).view(np.int64)
            coefs = np.array([[it[0].real, it[0].imag] for it in chunk], np.float64).reshape(-1)
            xors = np.array([it[2] for it in chunk], np.uint64)
            blob = torch.from_numpy(np.concatenate([host, coefs.view(np.int64), xors.view(np.int64),
                                                    np.array([0, cn], np.int64)])).to(self.device)
            o1, o2, o3 = host.size, host.size + coefs.size, host.size + coefs.size + xors.size
            begin = blob[o3:].to(torch.int32)
            mb = self.maxbits[: cn * self.nm].view(cn, self.nm)
            mb.zero_()
            mb[:, 0] = self.one_bits
            self.scale[: cn * sw].zero_()
            self.tab[0].view(self.items, self.stride)[:cn, 0] = 1  # empty environment (gpu_kernel.py:132)
            _lib.check(lib.dcs_gather_steps(self.dcode, _lib.ptr(self.tab[0]), _lib.ptr(self.tab[1]), self.stride,
                                            self.dsteps.ctypes.data, _lib.ptr(self.words), _lib.ptr(blob), S, 0, S,
                                            _lib.ptr(self.maxbits), self.nm, _lib.ptr(self.scale), cn, st))
            _lib.check(lib.dcs_accumulate_batched(
                self.dcode, _lib.ptr(final), self.stride, self.terminal_rank, self.term_runs.ctypes.data,
                self.term_nruns, self.tbasis.ctypes.data, _lib.ptr(blob) + 8 * o2, _lib.ptr(blob) + 8 * o1,
                _lib.ptr(begin), 1, self.params.shift, _lib.ptr(self.scale), _lib.ptr(self.maxbits[self.nm - 1:]),
                self.nm, _lib.ptr(out.view(torch.float64)), self.k, cn, st))
            flags[:cn] |= self.scale[: cn * sw].view(cn, sw)[:, 2]
        _lib.check(lib.dcs_block_tail(_lib.ptr(out), self.k, self.adj_hi.ctypes.data, self.u_open.ctypes.data, 1, st))
        if bool(((flags & 1) != 0).any()):
            raise ArithmeticError("Nonfinite prefix table")
        torch.cuda.current_stream(self.device).synchronize()
        meta = {"seconds": time.perf_counter() - start, "part": part, "parts": parts, "slices_evaluated": count,
                "prefix_dtype": "complex128" if self.use_fp64 else "complex64", "rmax": self.rmax,
                "terminal_rank": self.terminal_rank, "work_per_slice": self.work, "open_vertices": self.open_full,
                "vector_scale": "sqrt(2^(n-k)); sum all complex parts before probabilities"}
        return out[0].as_subclass(DeviceBlock), meta
