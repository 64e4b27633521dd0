"""CPU oracle for the split-operator Wigner propagation -- TEST INFRASTRUCTURE ONLY.

This package is a NumPy restatement of the reference's algorithm
(cabrer7/PyWignerCUDA2: GPU_Wigner4D.py, GPU_WignerDirac4D.py,
GPU_WignerDiracKvN4D.py).  Every function cites the reference file:line it
follows.  It exists to check the CUDA product, nothing else: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs
may import it.  The product package never imports it and has no CPU fallback.

Pinning.  The reference has no tests.  Its fractional transform ("FAFT") is an
external, un-vendored CUDA library (loaded by absolute path at
GPU_Wigner4D.py:29-58; no source, no version pin), restated here from its call
sites.  The restatement is pinned against the trace norms printed by the
reference's own notebooks (``instances/WignerDirac4D_64_64/*.ipynb``,
``instances/WignerDiracKvN4D_64_64/*.ipynb``), extracted to
``tests/golden/notebook_norms.json`` by ``tests/golden/make_golden.py``.
The scalar ``GPU_Wigner4D`` path prints no numbers in its notebooks; it shares
the FAFT contract, the rescaling wrappers and the elementwise-kernel
conventions with the pinned Dirac path, but its own step is "parity unpinned"
beyond that.
"""
