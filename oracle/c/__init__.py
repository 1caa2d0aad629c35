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
