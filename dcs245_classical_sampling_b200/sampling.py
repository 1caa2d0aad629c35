"""Sampler interface of the reference (``source/sampling/sampling_protocol.py``) on the GPU.

* ``draw_checked(amplitudes, uniform)`` — same arguments, same result keys and errors as the
  reference (:44-88); the CDF work runs on the device (``dcs_draw``) and the SHA-256 hashes of
  the weights and amplitudes are taken on the host from one device-to-host copy, as the
  reference's record requires.  Extra keys: ``cdf_tie`` (the parallel FP64 CDF could not
  certify that NumPy's sequential CDF selects the same index, so the device ran the exact
  sequential pass instead; the index is NumPy's either way) and ``cdf_straddle`` with
  ``cdf_straddle_margin`` (the uniform lies within that margin of an edge of its CDF bin, so a
  block of relative L2 error ``straddle_rel_l2`` could select a neighbouring index: by default
  the complex64 tolerance against the complex128 contraction of the same prefix; see
  ``straddle_margin``).  ``exact_cdf=True`` runs NumPy's sequential CDF for the
  block, so that ``cdf_lower_numpy``, ``cdf_upper_numpy`` and ``scaled_mass_cdf`` are NumPy's
  values bit for bit (otherwise they are the compensated values when no tie was found).
* ``draw_many(blocks, uniforms)`` — the device-only fast path for a batch of blocks: returns
  the per-block result records without hashes and with one small device-to-host copy.
* ``sample_checked(engine, prefixes, uniforms)`` — the per-sample loop of the reference's worker
  (block, host copy, checked draw with hashes: production/worker.py:105-113) with the host work
  of sample i (hashes, record) overlapped with the device work of sample i + 1.
* ``make_protocol`` / ``assemble_output`` — the reference's PCG64 schedule and bit mapping
  (:14-41, :91-100), host-side, unchanged in behaviour; ``make_audit_ids`` — the audit selection
  of ``production/protocol_common.py:22-31``.
"""
from __future__ import annotations

import hashlib

import numpy as np
import torch

from . import _lib

REPLAY_SCOPE = ("Full CDF checked in memory; hashes/interval retained. Independent regeneration "
                "requires rerunning the frozen block contraction.")

# Relative L2 bound of a complex64 block against the complex128 contraction of the same prefix.
COMPLEX64_REL_L2 = 1e-5
# A block within relative L2 error r of another has normalised CDF values within 2r of the
# other's: ||a/|a| - b/|b| || <= 2r, the probability vectors differ by at most twice that in L1,
# and partial sums of two distributions differ by at most half their L1 distance.  At 2^20
# outcomes a CDF bin is ~1e-6 wide, so this worst case covers every draw.
CDF_SHIFT_BOUND = 2 * COMPLEX64_REL_L2
# Standard deviations of the CDF shift that the straddle margin covers (see straddle_margin).
STRADDLE_SIGMAS = 6.0


def straddle_margin(weight_l2, rel_l2=COMPLEX64_REL_L2):
    """Distance to a CDF edge within which another contraction of relative L2 error rel_l2 could
    select a neighbouring index.  With independent per-entry relative errors of rms rel_l2, the
    shift of a partial sum of the probabilities p_j has standard deviation <= 2 rel_l2
    sqrt(sum p_j^2) (each p_j moves by about 2 p_j times its amplitude's relative error); the
    margin is STRADDLE_SIGMAS of that, and never more than the worst case 2 rel_l2."""
    return min(2.0 * rel_l2, STRADDLE_SIGMAS * 2.0 * rel_l2 * float(np.sqrt(max(weight_l2, 0.0))))


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


def draw_many(blocks, uniforms, device=None, exact_cdf=False):
    """Device draw for a batch: blocks (B, 2^k) complex128 (torch, device), uniforms (B,) float64.

    Returns a NumPy structured array (DRAW_DTYPE) with one record per block.  A record whose
    status is not 0 is a block the reference's draw_checked rejects (``check_record`` raises
    its error)."""
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
    _lib.check(lib.dcs_draw_ex(_lib.ptr(v), k, B, _lib.ptr(u), _lib.DRAW_SEQUENTIAL if exact_cdf else 0,
                               _lib.ptr(scratch), _lib.ptr(res), stream))
    return res.cpu().numpy().view(_lib.DRAW_DTYPE)


def check_record(r):
    """Raise the reference's error for a failed device draw record (sampling_protocol.py:54-72)."""
    if r["status"] == _lib.E_ARG:
        raise ValueError("Nonfinite vector or invalid uniform")
    if r["status"] != 0 or r["index"] < 0:
        raise ArithmeticError("Numerically zero/nonfinite block: do not replace the query")
    if not float(r["cdf_lower_exact"]) <= float(r["uniform"]) < float(r["cdf_upper_exact"]):
        raise ArithmeticError("Independent accurately summed CDF interval disagrees; do not resample")


def record_dict(r, straddle_rel_l2=COMPLEX64_REL_L2):
    """draw_checked's result keys (without the hashes) from a checked device record."""
    check_record(r)
    uniform = float(r["uniform"])
    lo, hi = float(r["cdf_lower_exact"]), float(r["cdf_upper_exact"])
    mass = float(r["total_exact"])
    near = min(uniform - lo, hi - uniform)
    margin = straddle_margin(float(r["weight_l2"]), straddle_rel_l2) if straddle_rel_l2 is not None else 0.0
    return {"A_index": int(r["index"]), "uniform": uniform, "scaled_mass_cdf": float(r["total_cdf"]),
            "scaled_mass_fsum": mass, "selected_scaled_weight": float(r["selected_weight"]),
            "selected_conditional_probability": float(r["selected_weight"] / mass),
            "cdf_lower_numpy": float(r["cdf_lower"]), "cdf_upper_numpy": float(r["cdf_upper"]),
            "cdf_lower_fsum": lo, "cdf_upper_fsum": hi,
            "uniform_to_nearest_boundary": near,
            "independent_cdf_check_passed": True,
            "finite_53bit_draw_TV_against_computed_normalized_weights": float(r["tv53"]),
            "cdf_tie": bool(r["tie"]),
            "cdf_straddle": bool(near < margin), "cdf_straddle_margin": margin}


def block_hashes(host):
    """weights_sha256 and amplitudes_sha256 of a host complex128 block (sampling_protocol.py:86-87)."""
    weights = np.asarray(host.real * host.real + host.imag * host.imag, dtype="<f8", order="C")
    return {"weights_sha256": hashlib.sha256(weights.tobytes()).hexdigest(),
            "amplitudes_sha256": hashlib.sha256(host.astype("<c16", copy=False).tobytes()).hexdigest()}


def draw_checked(amplitudes, uniform, hashes=True, exact_cdf=False, straddle_rel_l2=COMPLEX64_REL_L2):
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
    r = draw_many(v.unsqueeze(0), [uniform], device=v.device, exact_cdf=exact_cdf)[0]
    out = record_dict(r, straddle_rel_l2)
    if hashes:
        out.update(block_hashes(v.cpu().numpy()))
    out["replay_scope"] = REPLAY_SCOPE
    return out


def sample_checked(engine, x_list, uniforms, hashes=True, exact_cdf=False, straddle_rel_l2=COMPLEX64_REL_L2,
                   keep_host_blocks=False):
    """Blocks and checked draws of many prefixes, one sample at a time, as the reference's worker
    loop does (production/worker.py:105-113: block, host copy, draw_checked): the same records
    as ``engine.block`` + ``draw_checked(..., hashes)`` for each prefix, in order.

    The device work of sample i + 1 (contraction, tail, draw) is enqueued before the host
    finishes sample i (the host copy's hashes and record), and the host copy runs on a second
    stream, so host and device work overlap.  Returns a list of draw_checked dicts; with
    keep_host_blocks, also the host blocks (complex128 NumPy arrays)."""
    lib = _lib.load()
    n = len(x_list)
    if len(uniforms) != n:
        raise ValueError("one uniform per prefix")
    if not all(0 <= u < 1 for u in uniforms):
        raise ValueError("Nonfinite vector or invalid uniform")
    if n == 0:
        return ([], []) if keep_host_blocks else []
    dev = engine.device
    k = engine.k
    stream = torch.cuda.current_stream(dev)
    copy_stream = torch.cuda.Stream(dev)
    d_u = torch.tensor(np.asarray(uniforms, np.float64), device=dev)
    outs = [torch.empty((1, 1 << k), dtype=torch.complex128, device=dev) for _ in range(2)]
    res = torch.empty((2, _lib.DRAW_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    flags = torch.zeros((2, engine.items), dtype=torch.int64, device=dev)
    scratch = _scratch.get(dev, lib.dcs_draw_scratch_bytes(k, 1))
    host_blk = [torch.empty(1 << k, dtype=torch.complex128).pin_memory() if hashes or keep_host_blocks else None
                for _ in range(2)]
    host_res = [torch.empty(_lib.DRAW_DTYPE.itemsize, dtype=torch.uint8).pin_memory() for _ in range(2)]
    host_flags = [torch.empty(engine.items, dtype=torch.int64).pin_memory() for _ in range(2)]
    copied = [None, None]
    out, blocks = [], []

    def finish(i, slot):
        copied[slot].synchronize()
        from .engine import raise_for_flags
        raise_for_flags(host_flags[slot].numpy())
        rec = record_dict(host_res[slot].numpy().view(_lib.DRAW_DTYPE)[0], straddle_rel_l2)
        if hashes:
            rec.update(block_hashes(host_blk[slot].numpy()))
        rec["replay_scope"] = REPLAY_SCOPE
        out.append(rec)
        if keep_host_blocks:
            blocks.append(host_blk[slot].numpy().copy())

    prep = engine.prepare([x_list[0]])
    pending = None
    for i in range(n):
        slot = i & 1
        if copied[slot] is not None:  # sample i - 2's copies out of this slot are done
            stream.wait_event(copied[slot])
        flags[slot].zero_()
        engine.enqueue(prep, outs[slot], flags=flags[slot])
        _lib.check(lib.dcs_draw_ex(_lib.ptr(outs[slot]), k, 1, _lib.ptr(d_u[i:i + 1]),
                                   _lib.DRAW_SEQUENTIAL if exact_cdf else 0, _lib.ptr(scratch), _lib.ptr(res[slot]),
                                   stream.cuda_stream))
        done = torch.cuda.Event()
        done.record(stream)
        copy_stream.wait_event(done)
        with torch.cuda.stream(copy_stream):
            host_res[slot].copy_(res[slot], non_blocking=True)
            host_flags[slot].copy_(flags[slot], non_blocking=True)
            if host_blk[slot] is not None:
                host_blk[slot].copy_(outs[slot][0], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(copy_stream)
        copied[slot] = ev
        if i + 1 < n:
            prep = engine.prepare([x_list[i + 1]])
        if pending is not None:
            finish(*pending)
        pending = (i, slot)
    finish(*pending)
    return (out, blocks) if keep_host_blocks else out


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


def make_audit_ids(audit_seed, count, workers, per_worker):
    """Audit sample ids chosen before generation (production/protocol_common.py:22-31): an
    independent PCG64 stream picks `per_worker` ids without replacement in each worker's
    stratum (ids w, w + workers, ...).  Returns {worker: sorted ids}."""
    if workers < 1 or per_worker < 1:
        raise ValueError("Invalid worker/audit count")
    rng = np.random.Generator(np.random.PCG64(audit_seed))
    out = {}
    for worker in range(workers):
        ids = list(range(worker, count, workers))
        if len(ids) < per_worker:
            raise ValueError("Too few records in an audit stratum")
        out[worker] = sorted(map(int, rng.choice(ids, size=per_worker, replace=False)))
    return out


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
