"""CPU oracle for the TT-rounding / AMEn hot path.

TEST INFRASTRUCTURE ONLY.  This package is a plain FP64 numpy restatement of
the reference algorithms (TT-Toolbox, MATLAB) and exists to *check* the CUDA
library and to time the reference CPU path beside it.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its ``cpu_baseline`` leg and its
``--impl reference`` arm) may import it.  The shipped library never calls it:
the GPU path fails loudly when the CUDA extension is missing.

Every function cites the reference file:line it restates (paths relative to
the TT-Toolbox source tree).

Pinning status
--------------
* ``tt_round`` / ``my_chop2``: the reference has no golden vectors for
  rounding; pinned by mathematical invariants (error bound, exact ranks of
  known-rank inputs, full-tensor comparison at small d) in ``tests/``.
* ``amen_solve2``: pinned at the system level by the reference's known-answer
  fixtures ``tests/tt-solve/*.mat`` (stored solutions and their residuals),
  converted into ``tests/golden/*.npz`` by ``tests/golden/make_golden.py``.
  Iterates are not pinned by the reference (MATLAB is not runnable here).
* ``bfun3``, ``dgmresr_hh``, ``jac_gen``/``jac_apply`` (centre block
  Jacobi): pinned against the reference's own C (``fmex/solve3d.c``) built
  by ``oracle/build_ref.py`` into ``oracle/_ref/`` and called through ctypes
  (``tests/test_oracle_ref.py``).
* ``alstpz_solve``: the reference has no tests or golden vectors for it;
  pinned by convergence of the true residual, the zero-weight enrichment
  leaving the tensor unchanged, and the dense and GMRES local branches
  agreeing (``tests/test_oracle_alstpz.py``).
* ``amen_sum``: the reference has no tests or golden vectors for it; pinned
  by the exact linear combination at tight tolerance (full tensors at small
  d), rank bounds and tolerance-following errors (``tests/test_oracle_amen_sum.py``).
"""
