"""CPU oracle for the band-solve path: TEST INFRASTRUCTURE, NOT PRODUCT.

A plain numpy/scipy float64 restatement of the reference's Kohn-Sham band
solve, used only as the checker: by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline legs of ``bench.py``. Nothing in ``gradwave_b200``
imports it, and the product path never routes through it.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference itself
(gradwave, imported in the build container) on the seeded cells and the
committed ``tests/golden/*.npz`` hold its outputs; ``tests/test_oracle.py``
checks this restatement against them.

Modules:
  ham       - ``BatchedHamiltonian.apply`` (gradwave ``core/batch.py:405-428,480-505``)
  precond   - ``teter_b`` (gradwave ``solvers/precond.py:20-39``)
  davidson  - ``davidson_batched`` (gradwave ``solvers/davidson.py:406-457,528-774``)
  mlp       - float64 forward/backward of the learned preconditioner network
"""
