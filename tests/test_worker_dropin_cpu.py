"""The engine's block as the reference's worker handles it (production/worker.py:105-113):
``host = cp.asnumpy(v)`` with CuPy or with the NumPy-backed stand-in the reference's own CPU
fixture installs (``cp.asnumpy = np.asarray``, make_synthetic_worker_fixture.py:53-59)."""
import hashlib
import types

import numpy as np
import torch

from dcs245_classical_sampling_b200.engine import DeviceBlock


def test_device_block_copies_to_host_like_a_cupy_array():
    cp = types.SimpleNamespace(asnumpy=np.asarray)  # the reference fixture's stand-in
    base = torch.arange(16, dtype=torch.float64) * (1 + 0.5j)
    v = base.to(torch.complex128).as_subclass(DeviceBlock)
    host = cp.asnumpy(v)
    assert isinstance(host, np.ndarray) and host.dtype == np.complex128 and host.shape == (16,)
    np.testing.assert_array_equal(host, base.numpy())
    # the worker's anchor hash and the draw's amplitude hash are over '<c16' bytes of the host copy
    want = hashlib.sha256(base.numpy().astype("<c16").tobytes()).hexdigest()
    assert hashlib.sha256(host.astype("<c16", copy=False).tobytes()).hexdigest() == want
    assert np.asarray(v, dtype=np.complex64).dtype == np.complex64
    # operations give plain tensors; the block stays a tensor for the library's own calls
    assert type(v * 2) is torch.Tensor and isinstance(v, torch.Tensor)
