"""ORACLE (test infrastructure): restatement of the reference sampler, law vector and audit.

* ``draw``           <- ``source/sampling/sampling_protocol.py:44-88`` (draw_checked)
* ``cdf_law_vector`` <- ``source/production/protocol_common.py:48-70``
* ``audit_pair``     <- ``source/review/full_vector_audit_certificate.py:15-43``
* ``assemble``       <- ``source/sampling/sampling_protocol.py:91-100``
* ``protocol``       <- ``source/sampling/sampling_protocol.py:14-41`` (PCG64 schedule)
"""
from __future__ import annotations

import math

import numpy as np


def draw(amplitudes, uniform):
    """Sequential FP64 CDF, last value forced to 1, searchsorted(side='right'), fsum interval."""
    v = np.asarray(amplitudes, dtype=np.complex128)
    if v.ndim != 1 or not len(v) or len(v) & (len(v) - 1):
        raise ValueError("Expected a power-of-two one-dimensional amplitude vector")
    if not np.isfinite(v).all() or not 0 <= uniform < 1:
        raise ValueError("Nonfinite vector or invalid uniform")
    w = v.real * v.real + v.imag * v.imag
    cdf = np.cumsum(w)
    total = float(cdf[-1])
    if not total > 0 or not math.isfinite(total):
        raise ArithmeticError("Numerically zero/nonfinite block")
    cdf = cdf / total
    cdf[-1] = 1.0
    idx = int(np.searchsorted(cdf, uniform, side="right"))
    if idx >= len(w) or w[idx] <= 0:
        raise ArithmeticError("CDF produced an invalid outcome")
    mass = math.fsum(w.tolist())
    pre = math.fsum(w[:idx].tolist())
    lo, hi = pre / mass, (pre + float(w[idx])) / mass
    if not lo <= uniform < hi:
        raise ArithmeticError("Independent accurately summed CDF interval disagrees")
    ends = np.ceil(cdf * 2.0 ** 53)
    grid = np.diff(ends, prepend=0.0) / 2.0 ** 53
    tv = float(0.5 * np.sum(np.abs(grid - w / mass)))
    return {"A_index": idx, "uniform": float(uniform), "scaled_mass_cdf": total,
            "scaled_mass_fsum": mass, "selected_scaled_weight": float(w[idx]),
            "selected_conditional_probability": float(w[idx] / mass),
            "cdf_lower_numpy": float(cdf[idx - 1]) if idx else 0.0, "cdf_upper_numpy": float(cdf[idx]),
            "cdf_lower_fsum": lo, "cdf_upper_fsum": hi,
            "uniform_to_nearest_boundary": min(uniform - lo, hi - uniform),
            "finite_53bit_draw_TV_against_computed_normalized_weights": tv}


def cdf_law_vector(amplitudes):
    """Amplitudes whose probabilities are the 53-bit grid counts of the sampler's CDF."""
    a = np.asarray(amplitudes, dtype=np.complex128)
    w = a.real * a.real + a.imag * a.imag
    cdf = np.cumsum(w)
    total = float(cdf[-1])
    if not total > 0:
        raise ArithmeticError("Zero conditional vector")
    cdf = cdf / total
    cdf[-1] = 1.0
    ends = np.ceil(cdf * 2.0 ** 53).astype(np.uint64)
    counts = np.diff(np.concatenate(([np.uint64(0)], ends)))
    assert int(counts.sum(dtype=np.uint64)) == 1 << 53
    ph = np.ones(len(a), complex)
    nz = np.abs(a) > 0
    ph[nz] = a[nz] / np.abs(a[nz])
    return ph * np.sqrt(counts.astype(float) / 2.0 ** 53), counts


def audit_pair(reference_scaled, approximate):
    """normalized_conditional_overlap_abs = |<ref, approx>| / (|approx| |ref|), capped at 1."""
    ref = np.asarray(reference_scaled, np.complex128)
    ap = np.asarray(approximate, np.complex128)
    rm = float(np.vdot(ref, ref).real)
    am = float(np.vdot(ap, ap).real)
    score = float(abs(np.vdot(ref, ap)) / math.sqrt(am))
    return {"normalized_conditional_overlap_abs": min(1.0, score / math.sqrt(rm)) if rm > 0 else None,
            "uncapped_overlap_witness": score, "clipped_weight": min(score, 1.0),
            "reference_scaled_mass": rm, "approximate_input_mass": am}


def assemble(input_bits, free, index, ring=None):
    bits = [int(b) for b in input_bits]
    for j, q in enumerate(free):
        bits[q] = (index >> j) & 1
    ring = list(range(len(bits))) if ring is None else list(ring)
    orig = [0] * len(bits)
    for q, actual in enumerate(ring):
        orig[actual] = bits[q]
    return "".join(map(str, bits)), "".join(map(str, orig[::-1]))


def protocol(seed, count, n, free):
    """PCG64 per sample: branch uniform, closed bits (uint8), draw uniform (mixture weight 1)."""
    closed = [q for q in range(n) if q not in free]
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for sid in range(count):
        bu = float(rng.random())
        x = np.zeros(n, np.uint8)
        x[closed] = rng.integers(0, 2, len(closed), dtype=np.uint8)
        du = float(rng.random())
        out.append({"sample_id": sid, "branch_uniform": bu, "draw_uniform": du,
                    "input_data_bits": "".join(map(str, x))})
    return out
