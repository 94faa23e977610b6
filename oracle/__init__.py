"""CPU oracle for the fused lattice-Boltzmann step -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (``pylbm_b200``) imports this package. Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it, and only as the
checker or the timed CPU reference -- never as a fallback for the GPU path.

* ``lbm_oracle``: float64 NumPy (or torch, for autograd) restatement of pylbm's array-level
  algorithm (core.py:88-266, karman.py:45-53,88-96), extended with a per-node Guo force field.
  Pinned bit-for-bit against fixtures generated by running pylbm itself
  (``tests/golden/make_golden.py``).
* ``build_ref.py``: compiles pylbm's own CUDA C kernel (backends/cuda/lbm.cu) from the reference
  tree into ``oracle/_ref/`` with a launcher written here, as a GPU parity comparator.
"""
