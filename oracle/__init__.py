"""ORACLE — test infrastructure only.

A CPU restatement of the reference's contraction-and-sampling path, used to
check the CUDA path.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import anything under ``oracle/``; the
product package never does, and the product fails loudly when its CUDA
library is missing instead of falling back here.

* ``oracle.block_ref``   NumPy complex128 restatement of the plan compiler,
  the one-buffer executor, the slice loop and the Walsh-Hadamard tail.
* ``oracle.sampler_ref`` NumPy/math restatement of the FP64 CDF draw, the
  53-bit law vector and the audit overlap.
* ``oracle/c``           the same executor in C with OpenMP (complex128),
  used as the timed CPU baseline.

Parity is pinned: the restatement is checked against golden vectors produced
by running the reference itself (``tests/golden/make_golden.py``) and against
the reference's own known-answer cases (``sampling_protocol.selftest``,
``test_protocol_cpu.py`` rational grid counts).
"""
