"""Conditional-block engine on the B200: the drop-in for the reference's
``InplaceConditionalBlockGPU`` (``source/sampling/conditional_block_inplace_gpu.py``,
``source/sampling/conditional_block_gpu.py``).

Same constructor ``(graph, unitaries, n, order, parity_operations, open_vertices)``, same
``alloc(dtype, device)`` and ``block(x_bits, w=None, part=0, parts=1) -> (vector, meta)``,
same errors.  The returned vector is a complex128 torch tensor on the engine's device
(``DeviceBlock``: ``np.asarray`` and ``cupy.asnumpy`` copy it to the host, as the reference's
worker does), scaled by sqrt(2^(n-k)), index bit j <-> ``open_vertices[j]``.

Execution modes (``alloc(..., mode=...)``):

* ``"plain"``  — one launch per vertex step and a host read of the step's max after each
  launch (the reference's control flow, ``kernel_opt/inplace_gpu.py:107-124``);
* ``"device"`` — the renormalisation stays on the device; all steps of all slices are
  enqueued without host synchronisation, several slices (work items) per launch when the
  HBM budget allows (default);
* ``"fused"``  — like ``device`` but several vertex steps per pass over the table
  (coset-tiled fused kernels; complex128 tables run the plan-specialised register-run kernels
  compiled in FP64, which is how the complex128 audit recontraction runs at full size).

Host work per block is the reference's bookkeeping (local vectors, slice coefficients,
offset bits), vectorised over slices; the device does every pass over the tables.
"""
from __future__ import annotations

import itertools
import math
import time

import numpy as np
import torch

from . import _lib
from .plan import (KIND_GROW, W_T, build_block_plan, deposit_runs, orbit_kind, slot_mask)

LN2 = math.log(2.0)

# Fused plan of complex128 tables (plan-specialised kernels in FP64): 2^12-entry tiles of 16-byte
# entries (64 KB of shared memory, two CTAs per SM), 3 contiguous low bits (128-byte rows),
# register runs of local dimension 4, groups of fewest table bytes.
FP64_FUSED_CONFIG = {"max_dim": 12, "low": 3, "max_steps": 24, "variant": 12, "pairs": False, "grouping": "bytes",
                     "group_cost": 1 << 30, "max_extra": 1}
# shapes tried in order when a group of the plan fits no run of that shape (small plans)
FP64_FALLBACK_CONFIGS = ({"low": 4, "grouping": "greedy"}, {"variant": 4}, {"variant": 4, "low": 4, "grouping": "greedy"},
                         {"variant": 4, "low": 2}, {"variant": 4, "low": 1, "grouping": "greedy"})


def device_steps(steps):
    """OrbitStep list -> dcs_step array (host)."""
    out = np.zeros(len(steps), dtype=_lib.STEP_DTYPE)
    for i, st in enumerate(steps):
        kind, omit = orbit_kind(st)
        enum = [p for p in st.active_in if p not in omit]
        runs = deposit_runs(slot_mask(enum))
        if len(runs) > _lib.MAX_RUNS:
            raise ValueError(f"step {i}: {len(runs)} deposit runs exceed {_lib.MAX_RUNS}")
        r = out[i]
        r["K"], r["Ka"], r["beta"] = st.K, st.Ka, st.beta
        r["pivot_bit"] = (1 << st.pivot) if kind == KIND_GROW else 0
        r["in_mask"], r["out_mask"] = slot_mask(st.active_in), slot_mask(st.active_out)
        r["kind"], r["m"], r["nruns"], r["free_"] = kind, len(enum), len(runs), int(st.free)
        for j, (src, dst, ln) in enumerate(runs):
            r["runs"][j] = src | (dst << 8) | (ln << 16)
    return out


def raise_for_flags(flags):
    """The errors an item's scale flags report: bit 2, a generated kernel's bounded wait between
    tiles gave up (the block is invalid); bit 0, a nonfinite table (the reference's error)."""
    flags = np.asarray(flags)
    if np.any(flags & 4):
        raise RuntimeError("a group kernel's wait between tiles gave up; the block is invalid")
    if np.any(flags & 1):
        raise ArithmeticError("Nonfinite in-place environment")


def pack_runs(slots):
    runs = deposit_runs(slot_mask(slots))
    arr = np.zeros(max(1, len(runs)), dtype=np.uint32)
    for j, (src, dst, ln) in enumerate(runs):
        arr[j] = src | (dst << 8) | (ln << 16)
    return arr, len(runs)


class SliceParams:
    """Vectorised reference bookkeeping: per (prefix, slice) item, the per-step weights,
    offset bits, slice coefficient and scatter xor (conditional_block_gpu.py:136-157,
    inplace_gpu.py:111-114)."""

    def __init__(self, plan):
        p = self.plan = plan
        self.nsteps = len(p.steps)
        self.vert = np.array([st.v for st in p.steps], dtype=np.int64)         # reduced labels
        self.free = np.array([st.free for st in p.steps], dtype=bool)
        self.keep = np.array(p.keep, dtype=np.int64)
        self.nslice = len(p.slices)
        # reference vertices' bra . U (x-independent), data vertices' two rows
        U = np.stack([np.asarray(p.U_full[q], np.complex128) for q in range(p.N_full)])
        self.U = U
        self.is_data = np.arange(p.N_full) < p.n
        # neighbour-flip matrix: slice s -> kept vertices flipped
        self.nbr = np.zeros((self.nslice, p.N), dtype=np.uint8)
        for si, s in enumerate(p.slices):
            for v in p.nbrs_in_keep[s]:
                self.nbr[si, v] ^= 1
        # fixed positions: offset contributions (bits of fut) before `stop` and the tail
        fixed_pos = [j for j, st in enumerate(p.steps) if not st.free]
        self.fixed_pos = np.array(fixed_pos, dtype=np.int64)
        self.fixed_vert = self.vert[self.fixed_pos] if fixed_pos else np.zeros(0, np.int64)
        F = np.zeros((len(fixed_pos), self.nsteps), dtype=np.uint8)
        tail = np.zeros(len(fixed_pos), dtype=object)
        for a, j in enumerate(fixed_pos):
            fj = p.fut[j]
            # bits at positions > j inside the step range; bits >= stop go to the final offset
            for t in range(j + 1, self.nsteps):
                if (fj >> t) & 1:
                    F[a, t] = 1
            tail[a] = fj >> p.stop
        self.F = F
        self.tail = tail
        self.open_red = np.array(p.open_red, dtype=np.int64)
        self.shift = (p.N_full - p.n + len(p.open_full)) * 0.5 * LN2

    def full_vectors(self, x_bits, w=None):
        """local_vectors for every full-graph vertex (scan_plan.py:108-120), shape (N_full, 2)."""
        p = self.plan
        f = np.empty((p.N_full, 2), dtype=np.complex128)
        x = np.asarray(x_bits, dtype=np.int64)[: p.n]
        f[: p.n] = self.U[np.arange(p.n), x]
        if p.N_full > p.n:
            refs = np.arange(p.n, p.N_full)
            if isinstance(w, dict):
                bras = np.stack([np.asarray(w[q], np.complex128) for q in refs])
            else:
                bras = np.broadcast_to(W_T if w is None else np.asarray(w, np.complex128), (len(refs), 2))
            f[p.n:] = np.einsum("ri,rij->rj", bras, self.U[refs])
        return f

    def items(self, x_bits, w=None, part=0, parts=1):
        """-> (count, list of slice items): each item = (coef, params (nsteps) PARAM_DTYPE, xor)."""
        p = self.plan
        ff = self.full_vectors(x_bits, w)
        out = []
        count = 0
        for idx, bits in enumerate(itertools.product((0, 1), repeat=self.nslice)):
            if idx % parts != part:
                continue
            count += 1
            bits = np.array(bits, dtype=np.int64)
            coef = complex(np.prod([ff[s][b] for s, b in zip(p.slices, bits)])) if self.nslice else 1 + 0j
            par = sum(int(bits[p.slices.index(a)]) * int(bits[p.slices.index(b)]) for a, b in p.slice_edges)
            coef *= (-1) ** par
            if not coef:
                continue
            flips = (bits @ self.nbr) & 1 if self.nslice else np.zeros(p.N, dtype=np.int64)
            f = ff[self.keep].copy()
            f[:, 1] *= 1 - 2 * flips
            params = np.zeros(self.nsteps, dtype=_lib.PARAM_DTYPE)
            fs = f[self.vert]
            params["f0r"], params["f0i"] = fs[:, 0].real, fs[:, 0].imag
            params["f1r"], params["f1i"] = fs[:, 1].real, fs[:, 1].imag
            xor_tail = 0
            if len(self.fixed_pos):
                y = (np.abs(f[self.fixed_vert, 0]) > 1e-12) == 0
                params["y"][self.fixed_pos] = y.astype(np.int32)
                ov = (y.astype(np.int64) @ self.F.astype(np.int64)) & 1
                params["ov"] = ov.astype(np.int32)
                for a in np.flatnonzero(y):
                    xor_tail ^= int(self.tail[a])
            freeflip = 0
            for j, q in enumerate(self.open_red):
                if flips[q]:
                    freeflip |= 1 << j
            out.append((coef, params, xor_tail ^ freeflip))
        return count, out


class DeviceBlock(torch.Tensor):
    """What ``block`` returns: the complex128 block as a CUDA tensor that host code can copy the
    way the reference's worker copies CuPy arrays (``host = cp.asnumpy(v)``,
    production/worker.py:109): ``np.asarray(v)`` returns a host copy (so does ``cupy.asnumpy``,
    through ``__cuda_array_interface__``, or a NumPy-backed stand-in of it).  Operations on it
    return plain tensors."""

    __torch_function__ = torch._C._disabled_torch_function_impl

    def __array__(self, dtype=None, copy=None):
        host = torch.Tensor.cpu(self).numpy()
        return host if dtype is None else host.astype(dtype, copy=False)


class InplaceConditionalBlockGPU:
    """Drop-in for the reference engine of the same name (see module docstring)."""

    def __init__(self, graph, unitaries, n, order, parity_operations, open_vertices):
        self.plan = plan = build_block_plan(graph, unitaries, n, order, parity_operations, open_vertices)
        # reference attribute surface (conditional_block_gpu.py:25-69)
        self.N_full, self.n, self.N = plan.N_full, plan.n, plan.N
        self.open_full, self.open_red = plan.open_full, plan.open_red
        self.slices, self.slice_edges, self.nbrs_in_keep = plan.slices, plan.slice_edges, plan.nbrs_in_keep
        self.relabel, self.keep, self.U_full = plan.relabel, plan.keep, plan.U_full
        self.edges, self.order, self.fixed, self.fut = plan.edges, plan.order, plan.fixed, plan.fut
        self.stop, self.rmax, self.work = plan.stop, plan.rmax, plan.work
        self.open_edges = plan.open_edges
        self.terminal_basis = plan.terminal_basis
        self.terminal_rank = plan.terminal_rank
        self.params = SliceParams(plan)
        self._alloc = False

    # ------------------------------------------------------------------ allocation
    def alloc(self, dtype=np.complex64, device=0, fp64_kernel_path=None, mode=None, items=None,
              hbm_budget=None, jit=None, storage=None, external_table=False):
        """Allocate device buffers (conditional_block_inplace_gpu.py:18-34).

        dtype: complex64 (FP32 arithmetic) or complex128 (FP64 arithmetic).
        mode: "plain", "device" or "fused" (default: fused for complex64 tables of 2^26 entries
        and more, device otherwise).
        items: concurrent work items (slices) per launch; default = as many slices as fit
        in the HBM budget (default 85% of free device memory).
        jit: in fused mode with register runs, run the groups as plan-specialised kernels
        compiled for this plan with NVRTC (jit.py); default: the tuned setting of this plan and
        device (autotune_cache.json), else off.
        storage: "float16" stores each entry as two IEEE binary16 components (4 bytes), combines
        them in FP64 and rounds every stored value FP64 -> FP32 -> binary16: the reference's
        approximate half-storage tier (kernel_opt/inplace_half_gpu.py:37-78), which halves the
        table of complex64; complex64 dtype and the "device" / "plain" executors only.
        external_table: allocate no table; the caller lends one per batch with bind_table (up to
        `items` work items), e.g. from a device-memory pool shared by several engines."""
        if np.dtype(dtype) not in (np.dtype(np.complex64), np.dtype(np.complex128)):
            raise ValueError(dtype)
        if storage not in (None, "float16"):
            raise ValueError(f"storage {storage!r}")
        half = storage == "float16"
        if half and np.dtype(dtype) != np.dtype(np.complex64):
            raise ValueError("Half storage exports complex64; use baseline executor for complex128")
        if mode is None:  # fused passes pay off once the tables are far larger than a tile
            mode = ("fused" if np.dtype(dtype) == np.dtype(np.complex64) and self.plan.maxslots >= 26 and not half
                    else "device")
        if mode not in ("plain", "device", "fused"):
            raise ValueError(mode)
        if mode == "fused" and half:
            raise ValueError("the fused executors store complex64 or complex128 tables")
        if mode == "fused" and np.dtype(dtype) == np.dtype(np.complex128) and jit is False:
            raise ValueError("complex128 fused tables run the plan-specialised kernels only (jit)")
        self.lib = _lib.load()
        if not torch.cuda.is_available():
            raise RuntimeError("InplaceConditionalBlockGPU needs a CUDA device")
        self.device = torch.device("cuda", device)
        torch.cuda.set_device(self.device)
        self.mode = mode
        self.inplace_fp64 = self.use_fp64 = np.dtype(dtype) == np.dtype(np.complex128)
        self.half = half
        self.inplace_storage = "float16-components" if half else np.dtype(dtype).name
        self.dcode = _lib.H16 if half else (_lib.C128 if self.use_fp64 else _lib.C64)
        plan = self.plan
        self.inplace_steps = plan.steps
        self.inplace_maxslots = plan.maxslots
        self.inplace_rmax = plan.inplace_rmax
        self.inplace_terminal_basis = dict(zip(plan.terminal_slots, plan.terminal_basis))
        self.dsteps = device_steps(plan.steps)
        # free steps: the plan-specialised kernels divide f0 out of their weights
        self.free_steps = ~np.isin(self.dsteps["kind"], (4, 5))  # DCS_KIND_FIXED, DCS_KIND_FIXED_SHRINK
        self.nsteps = len(plan.steps)
        tdtype = torch.complex128 if self.use_fp64 else torch.complex64
        entry = 16 if self.use_fp64 else (4 if half else 8)
        table_entries = 1 << plan.maxslots
        nslice_items = 1 << len(plan.slices)
        if items is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget = int((hbm_budget if hbm_budget is not None else 0.85 * free))
            items = max(1, min(nslice_items, budget // (table_entries * entry)))
        self.items = int(items)
        if mode == "fused" and self.use_fp64:
            # complex128: 16-byte entries, so tiles of 2^12 entries (64 KB) and two CTAs per SM
            self.fused_config = dict(FP64_FUSED_CONFIG)
            self.jit, self.jit_minb, self.jit_threads = True, 2, 256
            self.fplan = self._build_fplan()
            self.items = 1
        elif mode == "fused":
            from .autotune import cached
            cfg = cached(plan, torch.cuda.get_device_name(self.device)) or {}
            self.fused_config = {"max_dim": cfg.get("max_dim", 13), "low": cfg.get("low", 4),
                                 "max_steps": cfg.get("max_steps", 24), "variant": cfg.get("variant", 0),
                                 "pairs": cfg.get("pairs", False), "grouping": cfg.get("grouping", "greedy"),
                                 "group_cost": cfg.get("group_cost", 1 << 30), "max_extra": cfg.get("max_extra", 1),
                                 "prefetch_kb": cfg.get("prefetch_kb", 0),
                                 "group_variant": {int(g): int(v) for g, v in (cfg.get("group_variant") or {}).items()}}
            self.jit = bool(cfg.get("jit", False) if jit is None else jit)
            self.jit_minb = cfg.get("minb")
            self.jit_threads = cfg.get("threads") or 256
            self.jit_group_cfg = {int(g): tuple(c) for g, c in (cfg.get("group_cfg") or {}).items()}
            self.fplan = self._build_fplan()
            self.items = 1
        self.entry_bytes = entry
        self.table_dtype = torch.float16 if half else tdtype
        self.items_cap = self.items
        if external_table:
            self.table = None
        elif half:  # (re, im) binary16 pairs
            self.table = torch.empty(self.items * table_entries * 2, dtype=torch.float16, device=self.device)
        else:
            self.table = torch.empty(self.items * table_entries, dtype=tdtype, device=self.device)
        self.table_stride = table_entries
        self.maxbits = torch.zeros(self.items * (self._nmax() + 1), dtype=torch.int64, device=self.device)
        self.scale = torch.zeros(self.items * _lib.SCALE_DTYPE.itemsize // 8, dtype=torch.int64,
                                 device=self.device)
        self.d_params = torch.zeros(self.items * self.nsteps * _lib.PARAM_DTYPE.itemsize // 8, dtype=torch.int64,
                                    device=self.device)
        self.one_bits = (np.array([1.0], np.float64).view(np.int64)[0] if self.use_fp64 or half
                         else int(np.array([1.0], np.float32).view(np.uint32)[0]))
        self.term_runs, self.term_nruns = pack_runs(plan.terminal_slots)
        self.tbasis = np.array(plan.terminal_basis + [0], dtype=np.uint64)
        k = len(plan.open_full)
        self.k = k
        adj = np.zeros(max(1, k), dtype=np.uint32)
        for a, b in plan.open_edges:
            lo, hi = (a, b) if a < b else (b, a)
            adj[lo] |= np.uint32(1 << hi)
        self.adj_hi = adj
        u = np.zeros((max(1, k), 8), dtype=np.float64)
        for q, orig in enumerate(plan.open_full):
            m = np.asarray(plan.U_full[orig], np.complex128)
            u[q] = [m[0, 0].real, m[0, 0].imag, m[0, 1].real, m[0, 1].imag,
                    m[1, 0].real, m[1, 0].imag, m[1, 1].real, m[1, 1].imag]
        self.u_open = u
        self._alloc = True
        self.buf = True

    def table_item_bytes(self):
        """Device bytes of one work item's table."""
        return self.table_stride * self.entry_bytes

    def bind_table(self, buf, items):
        """Run the next batches on `items` work items' tables in `buf` (a device uint8 tensor of at
        least items * table_item_bytes() bytes, 256-byte aligned), at most the capacity given
        to alloc.  The engine keeps no other reference to the memory."""
        items = int(items)
        if not 0 < items <= self.items_cap:
            raise ValueError(f"{items} work items outside 1..{self.items_cap}")
        need = items * self.table_item_bytes()
        if buf.dtype != torch.uint8 or buf.numel() < need or buf.data_ptr() % 256 or buf.device != self.device:
            raise ValueError("bind_table needs a 256-byte aligned uint8 device buffer of items x table bytes")
        self.table = buf[:need].view(self.table_dtype)
        self.items = items

    def _mb(self):
        nm = self._nmax() + 1
        return self.maxbits[: self.items * nm].view(self.items, nm)

    def _sc(self):
        w = _lib.SCALE_DTYPE.itemsize // 8
        return self.scale[: self.items * w].view(self.items, w)

    def _nmax(self):
        return len(self.fplan.groups) if self.mode == "fused" else self.nsteps

    def _build_fplan(self):
        """The fused plan of fused_config; with self.jit and register runs, its groups run as
        plan-specialised kernels (jit.py) compiled for this plan."""
        from .fused import build_fused_plan
        fp = build_fused_plan(self.plan, **self.fused_config, fp64=self.use_fp64)
        if self.use_fp64 and not all(int(v) & 4 for v in fp.groups["variant"]):
            # small tiles may not fit register runs of dimension 4: the next shapes that do
            for alt in FP64_FALLBACK_CONFIGS:
                cfg = {**self.fused_config, **alt}
                fp = build_fused_plan(self.plan, **cfg, fp64=True)
                if all(int(v) & 4 for v in fp.groups["variant"]):
                    self.fused_config = cfg
                    break
            else:
                raise ValueError("complex128 fused tables: this plan has groups that fit no register run; "
                                 "use mode='device'")
        if getattr(self, "jit", False) and fp.tile_runs is not None:
            from .jit import JitPlan
            fp.jit = JitPlan(self.plan, fp, self.lib, minb=getattr(self, "jit_minb", None),
                             threads=getattr(self, "jit_threads", 256),
                             group_cfg=getattr(self, "jit_group_cfg", None))
        return fp

    def set_fused_config(self, jit=None, minb=None, threads=None, group_cfg=None, **cfg):
        """Rebuild the fused plan with another tile shape (max_dim, low, max_steps, variant, pairs,
        prefetch_kb); jit=True/False switches the plan-specialised group kernels on or off; minb:
        CTAs per SM their registers are sized for (default: 2 with variant bit 0, else 3);
        threads: per CTA of those kernels (default 256); group_cfg: {group: (minb, prefetch_kb)}
        for single groups (dropped when the shape changes and none is given)."""
        if self.mode != "fused":
            raise ValueError("set_fused_config needs mode='fused'")
        if self.use_fp64 and (jit is False or not cfg.get("variant", 4) & 4):
            raise ValueError("complex128 fused tables run the plan-specialised register-run kernels only")
        if jit is not None:
            self.jit = bool(jit)
        if minb is not None:
            self.jit_minb = int(minb)
        if threads is not None:
            self.jit_threads = int(threads)
        if group_cfg is not None:
            self.jit_group_cfg = {int(g): tuple(c) for g, c in group_cfg.items()}
        elif cfg or minb is not None:
            self.jit_group_cfg = {}
        if cfg and "group_variant" not in cfg:
            cfg["group_variant"] = {}  # per-group variants belong to one shape
        self.fused_config = {**self.fused_config, **cfg}
        self.fplan = self._build_fplan()
        self.maxbits = torch.zeros(self.items * (len(self.fplan.groups) + 1), dtype=torch.int64, device=self.device)

    def tune_groups(self, x_bits=None, save=True, **kw):
        """Choose per group of the fused plan the plan-specialised kernel variant (CTAs per SM,
        staging of the next tile's first-run entries) with the shortest launch (autotune.tune_groups)."""
        from . import autotune as at
        if self.mode != "fused" or self.fplan.jit is None:
            raise ValueError("tune_groups needs mode='fused' with the plan-specialised kernels")
        x = np.zeros(self.n, np.uint8) if x_bits is None else x_bits
        _, items = self.params.items(x)
        prm = torch.from_numpy(items[0][1].view(np.int64).copy()).to(self.device)
        return at.tune_groups(self, prm, save=save and not self.use_fp64, **kw)

    def autotune(self, x_bits=None, candidates=None, jit=None):
        """Time the fused tile-shape candidates on this engine's table and keep the fastest
        (jit: as plan-specialised group kernels; default: the engine's setting)."""
        from . import autotune as at
        if self.mode != "fused":
            return None
        if self.use_fp64:
            raise ValueError("the autotuner times complex64 tables")
        x = np.zeros(self.n, np.uint8) if x_bits is None else x_bits
        _, items = self.params.items(x)
        prm = torch.from_numpy(items[0][1].view(np.int64).copy()).to(self.device)
        jit = self.jit if jit is None else bool(jit)
        if self.fplan.jit is not None:
            self.fplan.jit.close()
        self.jit_group_cfg = {}
        rep = at.tune(self, prm, jit=jit, **({"candidates": candidates} if candidates else {}))
        self.jit = jit
        self.jit_minb = rep["best"].get("minb")
        self.jit_threads = rep["best"].get("threads") or 256
        self.fused_config = {k: rep["best"][k] for k in at.PLAN_KEYS}
        self.scale = torch.zeros(self.items * _lib.SCALE_DTYPE.itemsize // 8, dtype=torch.int64,
                                 device=self.device)
        return rep

    # ------------------------------------------------------------------ execution
    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _reset_items(self, n_items):
        mb = self._mb()
        mb[:n_items].zero_()
        mb[:n_items, 0] = self.one_bits
        self._sc()[:n_items].zero_()
        # empty environment = 1 at address 0 of every item (inplace_gpu.py:108)
        if getattr(self, "half", False):
            t = self.table.view(self.items, self.table_stride, 2)
            t[:n_items, 0, 0] = 1
            t[:n_items, 0, 1] = 0
        else:
            self.table.view(self.items, self.table_stride)[:n_items, 0] = 1

    def prepare(self, x_list, w=None, part=0, parts=1):
        """Host bookkeeping for a batch of prefixes and ONE host->device upload.

        Work items are the (prefix, slice) pairs with a nonzero slice coefficient, in prefix
        order then slice order; they run `self.items` at a time."""
        work, counts = [], []
        for b, x in enumerate(x_list):
            cnt, items = self.params.items(x, w, part, parts)
            counts.append(cnt)
            work.extend((b, c, p, xo) for c, p, xo in items)
        n = len(work)
        chunks = []
        begin_all = []
        for c0 in range(0, n, self.items):
            chunk = work[c0:c0 + self.items]
            blocks_in = []
            for it in chunk:
                if not blocks_in or blocks_in[-1] != it[0]:
                    blocks_in.append(it[0])
            begin = [0]
            for bb in blocks_in:
                begin.append(begin[-1] + sum(1 for it in chunk if it[0] == bb))
            chunks.append((c0, len(chunk), blocks_in[0], len(blocks_in), len(begin_all)))
            begin_all.extend(begin)
        unit_ok = [all(self.unit_weights_ok(it[2]) for it in work[c0:c0 + cn]) if self.mode == "fused" else True
                   for c0, cn, _, _, _ in chunks]
        host_params = (np.concatenate([it[2] for it in work]) if n else
                       np.zeros(1, _lib.PARAM_DTYPE)).view(np.int64)
        coefs = np.zeros(2 * max(1, n), np.float64)
        xors = np.zeros(max(1, n), np.uint64)
        for i, (_, c, _, xo) in enumerate(work):
            coefs[2 * i], coefs[2 * i + 1] = c.real, c.imag
            xors[i] = xo
        blob = np.concatenate([host_params, coefs.view(np.int64), xors.view(np.int64),
                               np.asarray(begin_all or [0], np.int64)])
        pinned = torch.from_numpy(blob).pin_memory()
        dev = torch.empty(blob.size, dtype=torch.int64, device=self.device)
        dev.copy_(pinned, non_blocking=True)
        o1 = host_params.size
        o2 = o1 + coefs.size
        o3 = o2 + xors.size
        return {"n_items": n, "chunks": chunks, "unit_ok": unit_ok, "counts": counts, "nblocks": len(x_list),
                "dev": dev,
                "pinned": pinned, "params": dev[:o1], "coefs": dev[o1:o2].view(torch.float64),
                "xors": dev[o2:o3], "begin": dev[o3:].to(torch.int32), "h2d_bytes": blob.nbytes}

    def unit_weights_ok(self, params):
        """Whether an item's step weights (a dcs_param array) can run the plan-specialised kernels,
        which divide f0 out of every free step: f0 != 0 there, and |f1 / f0| <= 2^32 so that a
        group of steps stays inside the FP32 range between renormalisations."""
        p = params[self.free_steps]
        a0 = np.hypot(p["f0r"], p["f0i"])
        return bool(np.all(a0 > 0) and np.all(np.hypot(p["f1r"], p["f1i"]) <= 2.0 ** 32 * a0))

    def _run_steps(self, params_ptr, n_items, unit_ok=True):
        lib, st = self.lib, self._stream()
        nm = self._nmax() + 1
        if self.mode == "fused":
            f = self.fplan
            if not unit_ok and f.fp64:
                raise ValueError("complex128 fused tables need step weights with f0 != 0 at every free step")
            if unit_ok:
                _lib.check(f.launch(lib, _lib.ptr(self.table), params_ptr, 0, len(f.groups), _lib.ptr(self.maxbits),
                                    _lib.ptr(self.scale), st))
            else:  # library kernels take the weights as they are
                _lib.check(f.launch_library(lib, _lib.ptr(self.table), params_ptr, 0, len(f.groups),
                                            _lib.ptr(self.maxbits), _lib.ptr(self.scale), st))
            return
        if self.mode == "plain":
            mb = self._mb()
            for s in range(self.nsteps):
                _lib.check(lib.dcs_slice_steps_batched(
                    self.dcode, _lib.ptr(self.table), self.table_stride, self.dsteps.ctypes.data, params_ptr,
                    self.nsteps, self.nsteps, s, 1, _lib.ptr(self.maxbits), _lib.ptr(self.scale), n_items, st))
                bits = mb[:n_items, s + 1].cpu().numpy()  # host sync per step, as the reference
                m2 = (bits.view(np.float64) if self.use_fp64 or self.half
                      else bits.astype(np.uint32).view(np.float32))
                if not np.all(np.isfinite(m2)):
                    raise ArithmeticError("Nonfinite in-place environment")
                if np.all(m2 == 0):
                    break  # the remaining steps act on zero tables (the reference returns None here)
            return
        _lib.check(lib.dcs_slice_steps_batched(
            self.dcode, _lib.ptr(self.table), self.table_stride, self.dsteps.ctypes.data, params_ptr,
            self.nsteps, self.nsteps, 0, self.nsteps, _lib.ptr(self.maxbits), _lib.ptr(self.scale), n_items, st))

    def enqueue(self, prep, out, flags=None):
        """Device work for a prepared batch into `out` ((nblocks, 2^k) complex128): contraction of
        every work item, accumulation, tail.  No host synchronisation (except in "plain" mode).
        flags: optional (self.items,) int64 device tensor that collects the items' scale flags
        (bit 0: a nonfinite table).  Returns the number of library kernel launches."""
        lib = self.lib
        nm = self._nmax() + 1
        entry = _lib.PARAM_DTYPE.itemsize
        launches = 0
        out.zero_()
        for ci, (c0, cn, b0, nb, boff) in enumerate(prep["chunks"]):
            self._reset_items(cn)
            self._run_steps(_lib.ptr(prep["params"]) + c0 * self.nsteps * entry, cn, prep["unit_ok"][ci])
            launches += len(self.fplan.groups) if self.mode == "fused" else self.nsteps
            flat = out[b0:b0 + nb].view(torch.float64)
            _lib.check(lib.dcs_accumulate_batched(
                self.dcode, _lib.ptr(self.table), self.table_stride, self.plan.terminal_rank,
                self.term_runs.ctypes.data, self.term_nruns, self.tbasis.ctypes.data,
                _lib.ptr(prep["xors"]) + 8 * c0, _lib.ptr(prep["coefs"]) + 16 * c0,
                _lib.ptr(prep["begin"]) + 4 * boff, nb, self.params.shift, _lib.ptr(self.scale),
                _lib.ptr(self.maxbits[nm - 1:]), nm, _lib.ptr(flat), self.k, cn, self._stream()))
            launches += 2
            if flags is not None:
                flags[:cn] |= self._sc()[:cn, 2]
        _lib.check(lib.dcs_block_tail(_lib.ptr(out), self.k, self.adj_hi.ctypes.data, self.u_open.ctypes.data,
                                      prep["nblocks"], self._stream()))
        launches += 2 if self.k <= 12 else 4
        return launches

    def _flags_tensor(self):
        return torch.zeros(self.items, dtype=torch.int64, device=self.device)

    def check_scale_flags(self, n_items=None):
        """Raise the reference's ArithmeticError if the last chunk saw a nonfinite table."""
        raise_for_flags(self._sc()[: n_items or self.items, 2].cpu().numpy())

    def _run(self, x_list, w=None, part=0, parts=1):
        prep = self.prepare(x_list, w, part, parts)
        out = torch.empty((len(x_list), 1 << self.k), dtype=torch.complex128, device=self.device)
        flags = self._flags_tensor()
        self.enqueue(prep, out, flags)
        raise_for_flags(flags.cpu().numpy())  # one small device->host read per call
        return out, prep

    def block(self, x_bits, w=None, part=0, parts=1):
        """Scaled conditional amplitudes of one prefix (conditional_block_gpu.py:128-177)."""
        if not self._alloc:
            self.alloc()
        start = time.perf_counter()
        out, prep = self._run([x_bits], w, part, parts)
        torch.cuda.current_stream(self.device).synchronize()
        return out[0].as_subclass(DeviceBlock), self._meta(time.perf_counter() - start, part, parts,
                                                           prep["counts"][0])

    def _meta(self, seconds, part, parts, count):
        return {"seconds": seconds, "part": part, "parts": parts, "slices_evaluated": count,
                "prefix_dtype": "complex128" if self.use_fp64 else "complex64", "rmax": self.rmax,
                "terminal_rank": self.terminal_rank, "work_per_slice": self.work,
                "open_vertices": self.open_full,
                "vector_scale": "sqrt(2^(n-k)); sum all complex parts before probabilities"}

    def blocks(self, x_list, w=None):
        """Blocks of many prefixes; (prefix, slice) work items share launches.

        Returns a complex128 tensor (len(x_list), 2^k) on the device (no launch for none)."""
        if not self._alloc:
            self.alloc()
        x_list = list(x_list)
        if not x_list:
            return torch.zeros((0, 1 << self.k), dtype=torch.complex128, device=self.device)
        out, _ = self._run(x_list, w)
        return out


class HalfConditionalBlockGPU(InplaceConditionalBlockGPU):
    """Drop-in for the reference's half-storage engine (sampling/conditional_block_half_gpu.py:11-35):
    binary16 tables with FP64 arithmetic (``alloc(storage="float16")``), and the block's meta
    annotated with the storage, as the reference's worker and verifier expect
    (production/worker.py:86, production/verify.py:460-462)."""

    HALF_META = {"intermediate_storage": "float16 real/imaginary components",
                 "local_arithmetic": "FP64 then float32-to-float16 rounded storage",
                 "coherent_accumulation": "complex128",
                 "approximation_scope": "Whole-vector quality requires independent FP64 validation"}

    def alloc(self, dtype=np.complex64, device=0, fp64_kernel_path=None, mode=None, items=None,
              hbm_budget=None, jit=None, storage="float16"):
        if storage != "float16":
            raise ValueError("HalfConditionalBlockGPU stores float16 components")
        return super().alloc(dtype=dtype, device=device, fp64_kernel_path=fp64_kernel_path, mode=mode,
                             items=items, hbm_budget=hbm_budget, storage="float16")

    def block(self, *args, **kwargs):
        vector, meta = super().block(*args, **kwargs)
        meta.update(self.HALF_META)
        return vector, meta
