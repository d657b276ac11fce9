"""CPU oracle for the IB-transfer and MAC-multigrid hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``afsi_gpu_b200`` package imports
this directory; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` use it, as the checker and as the timed CPU
restatement of the reference algorithm.  It is never the measured or shipped
path.

Every function is a NumPy (FP64 or FP32) restatement of the afsi-torch 0.28.0
algorithm it names, with the reference ``file:line`` in its docstring.  The
restatement keeps the reference's order of floating-point operations where that
order is observable (binning, the Peskin radical, stencil rows), so integer
outputs are bit-exact and floating-point outputs agree to rounding.

Parity pin: ``tests/golden/*.npz`` were produced by importing the reference
package on CPU (``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py``
checks this oracle against them.
"""
