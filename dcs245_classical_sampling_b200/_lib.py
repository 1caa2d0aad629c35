"""ctypes binding of ``libdcs245.so`` (the C ABI in ``include/dcs245.h``).

The struct layouts are mirrored as NumPy structured dtypes; ``load()`` checks them against
``dcs_struct_size`` so that a header change cannot silently corrupt kernel arguments.
There is no fallback: if the library is missing or fails to load, ``load()`` raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libdcs245.so"

C64, C128, H16 = 0, 1, 2  # table storage: complex64, complex128, two binary16 components
MAX_RUNS = 28
E_ARG, E_CUDA, E_NONFINITE, E_CDF = -1, -2, -3, -4
DRAW_SEQUENTIAL = 1  # dcs_draw_ex flag: numpy's sequential CDF pass for every block

STEP_DTYPE = np.dtype([
    ("K", "<u8"), ("Ka", "<u8"), ("beta", "<u8"), ("pivot_bit", "<u8"), ("in_mask", "<u8"),
    ("out_mask", "<u8"), ("kind", "<i4"), ("m", "<i4"), ("nruns", "<i4"), ("free_", "<i4"),
    ("runs", "<u4", (MAX_RUNS,)),
])
PARAM_DTYPE = np.dtype([("f0r", "<f8"), ("f0i", "<f8"), ("f1r", "<f8"), ("f1i", "<f8"),
                        ("ov", "<i4"), ("y", "<i4")])
SCALE_DTYPE = np.dtype([("logscale", "<f8"), ("exponent_sum", "<i8"), ("flags", "<u4"), ("pad", "<u4"),
                        ("phase", "<f8")])
GROUP_DTYPE = np.dtype([
    ("first", "<i4"), ("count", "<i4"), ("tile_dim", "<i4"), ("low_bits", "<i4"),
    ("coset_m", "<i4"), ("ncoset_runs", "<i4"), ("step_tile_off", "<i4"), ("variant", "<i4"),
    ("out_mask", "<u8"), ("basis", "<u8", (16,)), ("coset_runs", "<u4", (MAX_RUNS,)),
])
TILE_STEP_DTYPE = np.dtype([("cskip", "<u8"), ("tK", "<u4"), ("tKa", "<u4"), ("tpiv", "<u4"), ("tbeta", "<u4"),
                            ("sK", "<u1"), ("sKa", "<u1"), ("nins", "<u1"), ("rb1", "<u1"), ("rb2", "<u1"),
                            ("rk1", "<u1"), ("rk2", "<u1"), ("rmix", "<u1"), ("ins", "<u1", (16,)), ("mhi", "<u4"),
                            ("pair", "<u1"),
                            ("pnins", "<u1"), ("swapB", "<u1"), ("swapA", "<u1"), ("pmhi", "<u4"), ("tau1", "<u4"),
                            ("tau2", "<u4"), ("pins", "<u1", (16,)), ("s1e", "<u1", (4,)), ("s2e", "<u1", (4,)),
                            ("ptab", "<u2"), ("run_len", "<u1"), ("rdead", "<u1")])
TILE_RUN_DTYPE = np.dtype([("nins", "<u1"), ("count", "<u1"), ("r", "<u1"), ("pad", "<u1"), ("ins", "<u1", (16,)),
                           ("mhi", "<u4"), ("off", "<u2", (16,))])
DRAW_DTYPE = np.dtype([
    ("index", "<i8"), ("tie", "<i4"), ("status", "<i4"), ("total_cdf", "<f8"), ("total_exact", "<f8"),
    ("selected_weight", "<f8"), ("cdf_lower", "<f8"), ("cdf_upper", "<f8"), ("cdf_lower_exact", "<f8"),
    ("cdf_upper_exact", "<f8"), ("uniform", "<f8"), ("tv53", "<f8"), ("weight_l2", "<f8"),
])
GATHER_STEP_DTYPE = np.dtype([("beta", "<u8"), ("table_off", "<u8"), ("combo_off", "<u8"), ("r_in", "<i4"),
                              ("r_out", "<i4"), ("nbytes", "<i4"), ("ncombos", "<i4"), ("free_", "<i4"),
                              ("pad", "<i4")])
STRUCTS = [STEP_DTYPE, PARAM_DTYPE, SCALE_DTYPE, GROUP_DTYPE, TILE_STEP_DTYPE, DRAW_DTYPE, TILE_RUN_DTYPE,
           GATHER_STEP_DTYPE]

_P = ctypes.c_void_p
_I = ctypes.c_int
_U64 = ctypes.c_uint64
_D = ctypes.c_double

# name: (restype, argtypes)
SIGNATURES = {
    "dcs_abi_version": (_I, []),
    "dcs_prefix_cut_ranks": (_I, [_P, _I, _P, _I, _P]),
    "dcs_last_error": (ctypes.c_char_p, []),
    "dcs_sm_count": (_I, []),
    "dcs_struct_size": (ctypes.c_size_t, [_I]),
    "dcs_inplace_step": (_I, [_I, _P, _U64, _P, _I, _I, _I, _U64, _U64, _I, _U64, _I, _D, _D, _D, _D, _I, _D,
                              _P, _I, _P]),
    "dcs_slice_steps": (_I, [_I, _P, _P, _P, _I, _I, _I, _P, _P, _P]),
    "dcs_slice_steps_batched": (_I, [_I, _P, _U64, _P, _P, _U64, _I, _I, _I, _P, _P, _I, _P]),
    "dcs_fused_groups": (_I, [_P, _P, _I, _P, _I, _P, _P, _I, _I, _P, _P, _P]),
    "dcs_fused_runs": (_I, [_P, _P, _I, _P, _I, _P, _P, _P, _I, _I, _P, _P, _P]),
    "dcs_accumulate_batched": (_I, [_I, _P, _U64, _I, _P, _I, _P, _P, _P, _P, _I, _D, _P, _P, _U64, _P, _I, _I,
                                    _P]),
    "dcs_block_tail": (_I, [_P, _I, _P, _P, _I, _P]),
    "dcs_gather_steps": (_I, [_I, _P, _P, _U64, _P, _P, _P, _U64, _I, _I, _P, _U64, _P, _I, _P]),
    "dcs_draw_scratch_bytes": (ctypes.c_size_t, [_I, _I]),
    "dcs_draw": (_I, [_P, _I, _I, _P, _P, _P, _P]),
    "dcs_draw_ex": (_I, [_P, _I, _I, _P, ctypes.c_uint, _P, _P, _P]),
    "dcs_draw_static": (_I, [_P, _I, _P, _P, _P]),
    "dcs_overlap": (_I, [_P, _P, _U64, _P, _P, _P]),
    "dcs_philox_prefixes": (_I, [_P, _P, _I, _U64, _P, _I, _P, _P, _P]),
    "dcs_philox4x32_10_host": (None, [_P, ctypes.c_uint32, ctypes.c_uint32]),
    "dcs_build_items": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _P, _I, _P, _P, _P, _P]),
    "dcs_jit_compile": (_I, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _I,
                             ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_size_t), ctypes.c_char_p, ctypes.c_size_t]),
    "dcs_jit_free": (None, [_P]),
    "dcs_jit_load": (_I, [_P, ctypes.POINTER(_P)]),
    "dcs_jit_unload": (_I, [_P]),
    "dcs_jit_kernel": (_I, [_P, ctypes.c_char_p, ctypes.c_size_t, _I, ctypes.POINTER(_P), ctypes.POINTER(_I)]),
    "dcs_jit_launch": (_I, [_P, ctypes.c_uint, _I, ctypes.c_size_t, _P, _P, _P, _P, _P]),
}


class DCSError(RuntimeError):
    """A failed library call (the message is the library's last error)."""

    def __init__(self, code, msg):
        super().__init__(f"{msg} (code {code})")
        self.code = code


_lib = None


def load():
    """Load and check the library.  Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH.name} is not built; run `python -m dcs245_classical_sampling_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.dcs_abi_version() != 1:
        raise ImportError("libdcs245.so ABI version mismatch")
    for i, dt in enumerate(STRUCTS):
        if lib.dcs_struct_size(i) != dt.itemsize:
            raise ImportError(f"struct {i} layout mismatch: C {lib.dcs_struct_size(i)} vs Python {dt.itemsize}")
    _lib = lib
    return lib


def check(rc):
    if rc != 0:
        msg = _lib.dcs_last_error().decode(errors="replace") if _lib is not None else "library not loaded"
        raise DCSError(rc, msg)


def ptr(t):
    """Device (or host) address of a torch tensor / numpy array for the C ABI."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def exported_symbols():
    return list(SIGNATURES)
