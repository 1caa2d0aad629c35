"""ORACLE (test infrastructure): ctypes wrapper of the C/OpenMP executor restatement.

Used only by tests and by bench.py's CPU-baseline leg; built into oracle/_ref/ by `build()`.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref"
LIB = OUT / "liboracle_inplace.so"


def build():
    src = HERE / "inplace_omp.c"
    if LIB.exists() and LIB.stat().st_mtime >= src.stat().st_mtime:
        return LIB
    OUT.mkdir(exist_ok=True)
    # -march=native is host-specific: the box that runs the baseline rebuilds if the load fails
    subprocess.run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", str(LIB), str(src),
                    "-lm"], check=True)
    return LIB


def load():
    try:
        lib = ctypes.CDLL(str(build()))
    except OSError:
        LIB.unlink(missing_ok=True)
        lib = ctypes.CDLL(str(build()))
    lib.oracle_run_steps.restype = ctypes.c_double
    lib.oracle_run_steps.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.oracle_threads.restype = ctypes.c_int
    return lib


def encode(plan_steps):
    """OrbitStep-like dicts/objects -> (N,8) uint64 step words."""
    from dcs245_classical_sampling_b200.plan import orbit_kind, slot_mask, KIND_GROW
    out = np.zeros((len(plan_steps), 8), np.uint64)
    for i, st in enumerate(plan_steps):
        kind, omit = orbit_kind(st)
        out[i] = [kind, st.K, st.Ka, st.beta, (1 << st.pivot) if kind == KIND_GROW else 0,
                  slot_mask([p for p in st.active_in if p not in omit]), slot_mask(st.active_out), 0]
    return out


def encode_params(params):
    """PARAM_DTYPE records -> (N,6) float64."""
    return np.stack([params["f0r"], params["f0i"], params["f1r"], params["f1i"],
                     params["ov"].astype(np.float64), params["y"].astype(np.float64)], axis=1).copy()


def run_steps(lib, steps_u64, params_f64, E, first=0, count=None):
    count = len(steps_u64) - first if count is None else count
    return lib.oracle_run_steps(steps_u64.ctypes.data, params_f64.ctypes.data, first, count, E.ctypes.data)


_KIND = {"grow": 0, "replace": 3, "fixed": 4, "fixed_shrink": 5}


def encode_oracle_steps(steps):
    """The oracle engine's step dicts (block_ref.compile_plan) -> (N,8) uint64 step words of
    oracle_run_steps: kind code (inplace_gpu.py:74-82), K, Ka, beta, grow pivot bit, the
    enumerated slots (active_in without the orbit's role slots) and the active_out mask."""
    def mask(slots):
        m = 0
        for p in slots:
            m |= 1 << int(p)
        return m
    out = np.zeros((len(steps), 8), np.uint64)
    for i, st in enumerate(steps):
        kind = st["kind"]
        omit = ()
        if kind == "mix":
            code, omit = (1, (st["pivot_a"],)) if st["Ka"] else (2, ())
        elif kind == "shrink":
            code, omit = (6, (st["pivot"], st["pivot_a"])) if st["Ka"] else (7, (st["pivot"],))
        else:
            code = _KIND[kind]
            if kind in ("replace", "fixed_shrink"):
                omit = (st["pivot"],)
        enum = [p for p in st["active_in"] if p not in omit]
        out[i] = [code, st["K"], st["Ka"], st["beta"], (1 << st["pivot"]) if kind == "grow" else 0,
                  mask(enum), mask(st["active_out"]), 0]
    return out


class CpuSampler:
    """A complete CPU sample (block + draw) of the oracle engine with the C/OpenMP executor for the
    vertex steps: the reference's block() control flow (conditional_block_gpu.py:128-177) with
    execute_inplace's steps (inplace_plan.py:90-135) in C, then draw_checked in NumPy
    (sampling_protocol.py:44-88).  The CPU comparator of the small workloads."""

    def __init__(self, engine, lib=None):
        from oracle.block_ref import _addr
        self.eng = engine
        self.lib = lib or load()
        self.words = encode_oracle_steps(engine.steps)
        self.E = np.zeros(1 << engine.maxslots, np.complex128)
        last = engine.steps[-1]["active_out"] if engine.steps else ()
        self.terminal = _addr(last).astype(np.int64)

    def block(self, x_bits):
        import math
        from oracle.block_ref import tail
        e = self.eng
        k = len(e.open_full)
        total = np.zeros(1 << k, np.complex128)
        for coef, f, yfix, flips in e.slice_inputs(x_bits):
            if not coef:
                continue
            params = np.zeros((len(e.steps), 6))
            offset = 0
            for s, st in enumerate(e.steps):  # offset bits as execute() tracks them
                j = st["j"]
                params[s, 4] = (offset >> j) & 1
                offset &= ~(1 << j)
                y = int(yfix[st["v"]]) if not st["free"] else 0
                if y:
                    offset ^= e.fut[j]
                params[s, 5] = y
                f0, f1 = complex(f[st["v"]][0]), complex(f[st["v"]][1])
                params[s, :4] = f0.real, f0.imag, f1.real, f1.imag
            self.E[:] = 0
            self.E[0] = 1
            ls = run_steps(self.lib, self.words, params, self.E)
            env = self.E[self.terminal]
            if not np.any(env):
                continue
            freeflip = sum(int(flips[q]) << j for j, q in enumerate(e.open_red))
            idx = e.syndrome_map ^ np.uint64((offset >> e.stop) ^ freeflip)
            c = coef * math.exp(ls - (e.N_full - e.n + k) * 0.5 * math.log(2.0))
            total[idx.astype(np.int64)] += env * c
        tail(total, k, e.phase, [e.U_full[q] for q in e.open_full])
        return total

    def sample(self, x_bits, uniform):
        from oracle.sampler_ref import draw
        v = self.block(x_bits)
        return draw(v, uniform)
