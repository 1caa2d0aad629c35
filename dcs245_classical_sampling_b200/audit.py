"""Audit of a complex64 block against a complex128 recontraction (the c_y overlap).

``audit_vector_pair`` has the keys and errors of the reference's function
(``source/review/full_vector_audit_certificate.py:15-43``); the three inner products run on
the device (``dcs_overlap``, compensated FP64 sums) and only four doubles come back.
``normalized_conditional_overlap_abs`` is c_y = |<ref, approx>| / (|approx| |ref|).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib

_scratch = {}


def _dev(v, device):
    if isinstance(v, torch.Tensor):
        t = v if v.is_cuda else v.to(device)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(v, np.complex128))).to(device)
    return t.to(torch.complex128).contiguous()


def overlap_sums(reference_scaled, approximate_vector, device=None):
    """(<ref,ref>, <ap,ap>, <ref,ap>) as Python floats/complex."""
    lib = _lib.load()
    device = device or (reference_scaled.device if isinstance(reference_scaled, torch.Tensor) else "cuda")
    ref = _dev(reference_scaled, device)
    ap = _dev(approximate_vector, device)
    if ref.dim() != 1 or ref.shape != ap.shape or not ref.numel():
        raise ValueError("Need two nonempty full vectors with identical shape")
    key = str(ref.device)
    if key not in _scratch:
        _scratch[key] = torch.empty(16384 + 64, dtype=torch.uint8, device=ref.device)
    out = torch.empty(4, dtype=torch.float64, device=ref.device)
    _lib.check(lib.dcs_overlap(_lib.ptr(ref), _lib.ptr(ap), ref.numel(), _lib.ptr(out), _lib.ptr(_scratch[key]),
                               torch.cuda.current_stream(ref.device).cuda_stream))
    rr, aa, re, im = out.cpu().tolist()
    return rr, aa, complex(re, im)


def audit_vector_pair(reference_scaled, approximate_vector, audit_id):
    """Reference-compatible audit record (full_vector_audit_certificate.py:15-43)."""
    rr, aa, cross = overlap_sums(reference_scaled, approximate_vector)
    if not math.isfinite(rr) or not math.isfinite(aa) or not math.isfinite(abs(cross)):
        raise ValueError("Nonfinite vector values; do not filter this audit")
    if aa <= 0:
        raise ValueError("Invalid norm; supply the actual declared fallback if used")
    n = (reference_scaled.numel() if isinstance(reference_scaled, torch.Tensor) else len(reference_scaled))
    score = float(abs(cross) / math.sqrt(aa))
    overlap = min(1.0, score / math.sqrt(rr)) if rr > 0 else None
    weight = min(score, 1.0)
    return {"audit_id": audit_id, "vector_length": n, "reference_scaled_mass": rr, "approximate_input_mass": aa,
            "normalized_conditional_overlap_abs": overlap,
            "normalized_conditional_fidelity": overlap ** 2 if overlap is not None else None,
            "uncapped_overlap_witness": score, "clipped_weight": weight, "loss": 1 - weight,
            "reference_arithmetic": "complex128 numerical reference; not an interval-arithmetic proof"}


def relative_l2(reference, approx):
    """||approx - ref|| / ||ref|| after removing the global phase (parity slicing fixes amplitudes
    only up to a phase, parity_slicing.py:10)."""
    rr, aa, cross = overlap_sums(reference, approx)
    # min over phases of ||ap e^{i phi} - ref||^2 = aa + rr - 2 |<ref, ap>|
    return math.sqrt(max(0.0, aa + rr - 2 * abs(cross)) / rr) if rr > 0 else float("nan")
