"""Sampler interface of the reference (``source/sampling/sampling_protocol.py``) on the GPU.

* ``draw_checked(amplitudes, uniform)`` — same arguments, same result keys and errors as the
  reference (:44-88); the CDF work runs on the device (``dcs_draw``) and the SHA-256 hashes of
  the weights and amplitudes are taken on the host from one device-to-host copy, as the
  reference's record requires.  Extra key ``cdf_tie``: the parallel FP64 CDF could not
  certify that NumPy's sequential CDF selects the same index, so the device ran the exact
  sequential pass instead (the index is NumPy's either way).
* ``draw_many(blocks, uniforms)`` — the device-only fast path for a batch of blocks: returns
  the per-block result records without hashes and with one small device-to-host copy.
* ``make_protocol`` / ``assemble_output`` — the reference's PCG64 schedule and bit mapping
  (:14-41, :91-100), host-side, unchanged in behaviour.
"""
from __future__ import annotations

import hashlib

import numpy as np
import torch

from . import _lib

REPLAY_SCOPE = ("Full CDF checked in memory; hashes/interval retained. Independent regeneration "
                "requires rerunning the frozen block contraction.")


class _Scratch:
    def __init__(self):
        self.buf = {}

    def get(self, device, nbytes):
        key = (device, 0)
        t = self.buf.get(key)
        if t is None or t.numel() < nbytes:
            t = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=device)
            self.buf[key] = t
        return t


_scratch = _Scratch()


def _as_device_blocks(amplitudes, device=None):
    if isinstance(amplitudes, torch.Tensor):
        v = amplitudes
        if not v.is_cuda:
            v = v.to(device or "cuda")
    else:
        v = torch.from_numpy(np.ascontiguousarray(np.asarray(amplitudes, dtype=np.complex128))).to(device or "cuda")
    if v.dtype != torch.complex128:
        v = v.to(torch.complex128)
    return v.contiguous()


def draw_many(blocks, uniforms, device=None):
    """Device draw for a batch: blocks (B, 2^k) complex128 (torch, device), uniforms (B,) float64.

    Returns a NumPy structured array (DRAW_DTYPE) with one record per block."""
    lib = _lib.load()
    v = _as_device_blocks(blocks, device)
    if v.dim() == 1:
        v = v.unsqueeze(0)
    B, n = v.shape
    if n < 1 or n & (n - 1):
        raise ValueError("Expected a power-of-two one-dimensional amplitude vector")
    k = n.bit_length() - 1
    u = torch.as_tensor(np.asarray(uniforms, dtype=np.float64).reshape(B), device=v.device)
    res = torch.empty(B * _lib.DRAW_DTYPE.itemsize, dtype=torch.uint8, device=v.device)
    scratch = _scratch.get(v.device, lib.dcs_draw_scratch_bytes(k, B))
    stream = torch.cuda.current_stream(v.device).cuda_stream
    _lib.check(lib.dcs_draw(_lib.ptr(v), k, B, _lib.ptr(u), _lib.ptr(scratch), _lib.ptr(res), stream))
    return res.cpu().numpy().view(_lib.DRAW_DTYPE)


def draw_checked(amplitudes, uniform, hashes=True):
    """Reference-compatible checked draw (sampling_protocol.py:44-88)."""
    if isinstance(amplitudes, torch.Tensor):
        if amplitudes.dim() != 1:
            raise ValueError("Expected a power-of-two one-dimensional amplitude vector")
        n = amplitudes.shape[0]
    else:
        a = np.asarray(amplitudes)
        if a.ndim != 1:
            raise ValueError("Expected a power-of-two one-dimensional amplitude vector")
        n = a.shape[0]
    if not n or n & (n - 1):
        raise ValueError("Expected a power-of-two one-dimensional amplitude vector")
    if not 0 <= uniform < 1:
        raise ValueError("Nonfinite vector or invalid uniform")
    v = _as_device_blocks(amplitudes)
    r = draw_many(v.unsqueeze(0), [uniform], device=v.device)[0]
    if r["status"] == _lib.E_ARG:
        raise ValueError("Nonfinite vector or invalid uniform")
    if r["status"] != 0 or r["index"] < 0:
        raise ArithmeticError("Numerically zero/nonfinite block: do not replace the query")
    index = int(r["index"])
    lo, hi = float(r["cdf_lower_exact"]), float(r["cdf_upper_exact"])
    if not lo <= uniform < hi:
        raise ArithmeticError("Independent accurately summed CDF interval disagrees; do not resample")
    mass = float(r["total_exact"])
    out = {"A_index": index, "uniform": float(uniform), "scaled_mass_cdf": float(r["total_cdf"]),
           "scaled_mass_fsum": mass, "selected_scaled_weight": float(r["selected_weight"]),
           "selected_conditional_probability": float(r["selected_weight"] / mass),
           "cdf_lower_numpy": float(r["cdf_lower"]), "cdf_upper_numpy": float(r["cdf_upper"]),
           "cdf_lower_fsum": lo, "cdf_upper_fsum": hi,
           "uniform_to_nearest_boundary": min(uniform - lo, hi - uniform),
           "independent_cdf_check_passed": True,
           "finite_53bit_draw_TV_against_computed_normalized_weights": float(r["tv53"]),
           "cdf_tie": bool(r["tie"])}
    if hashes:
        host = v.cpu().numpy()
        weights = np.asarray(host.real * host.real + host.imag * host.imag, dtype="<f8", order="C")
        out["weights_sha256"] = hashlib.sha256(weights.tobytes()).hexdigest()
        out["amplitudes_sha256"] = hashlib.sha256(host.astype("<c16", copy=False).tobytes()).hexdigest()
    out["replay_scope"] = REPLAY_SCOPE
    return out


def make_protocol(seed, count, n, free_vertices, mixture_weight=1.0):
    """PCG64 prefix / uniform schedule (sampling_protocol.py:14-41), host-side."""
    free = list(map(int, free_vertices))
    if len(set(free)) != len(free) or not all(0 <= q < n for q in free):
        raise ValueError("Free vertices must be distinct data indices")
    if not 0 <= mixture_weight <= 1 or count < 1:
        raise ValueError("Invalid mixture weight or sample count")
    closed = [q for q in range(n) if q not in free]
    rng = np.random.Generator(np.random.PCG64(seed))
    records = []
    for sample_id in range(count):
        before = rng.bit_generator.state
        branch_u = float(rng.random())
        expensive = branch_u < mixture_weight
        x = np.zeros(n, np.uint8)
        if expensive:
            x[closed] = rng.integers(0, 2, len(closed), dtype=np.uint8)
            draw_u = float(rng.random())
        else:
            x[:] = rng.integers(0, 2, n, dtype=np.uint8)
            draw_u = None
        records.append({"sample_id": sample_id, "conditional_branch": expensive, "branch_uniform": branch_u,
                        "draw_uniform": draw_u, "input_data_bits": "".join(map(str, x)),
                        "rng_before": before, "rng_after": rng.bit_generator.state})
    return {"seed": int(seed), "count": count, "n": n, "free_vertices": free, "closed_vertices": closed,
            "mixture_weight": mixture_weight,
            "rng": "NumPy PCG64; branch float64, uint8 vector bits, conditional float64",
            "numpy_version": np.__version__, "records": records}


def assemble_output(input_bits, free_vertices, A_index, ring=None):
    """Index -> ring bits -> Qiskit bitstring (sampling_protocol.py:91-100)."""
    bits = list(map(int, input_bits))
    if not 0 <= A_index < 1 << len(free_vertices):
        raise ValueError("Conditional index outside free-output range")
    for j, q in enumerate(free_vertices):
        bits[q] = (A_index >> j) & 1
    if ring is None:
        ring = list(range(len(bits)))
    if sorted(ring) != list(range(len(bits))):
        raise ValueError("Invalid ring permutation")
    original = [0] * len(bits)
    for q, actual in enumerate(ring):
        original[actual] = bits[q]
    return "".join(map(str, bits)), "".join(map(str, original[::-1]))
