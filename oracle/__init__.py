"""CPU oracle for the graspcg NCG/NUFFT hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package (``mrirecon_b200``)
imports this package.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may use it, and
only as the checker or as the timed CPU stand-in for the reference.

Contents
--------
``oracle.kb``      Kaiser-Bessel gridding restatement (binning, weights,
                   deapodisation, forward/adjoint NUFFT with SENSE and DCF).
``oracle.nudft``   FP64 direct NUDFT and its true adjoint.
``oracle.tv``      Huber-TV energy/gradient restatement (TVND + ndops).
``oracle.ncg``     Non-linear CG driver restatement (CGSolver + Armijo/Wolfe +
                   FR/PR+/DY directions + Objective), reference schedule.

Parity pinning
--------------
* Binning is pinned bit-for-bit against index tables produced by the
  reference's own ``PTNUFFTAdapter.prepare`` (``tests/golden``).
* ``nudft_forward`` is pinned against the reference's ``_nudft_A``
  (graspcg/tests/test_nufft_precision_gt.py:55-89) on committed fixtures.
  The reference's ``_nudft_AH`` (same file :91-121) is not a true adjoint
  (it multiplies by the (R,K) matrix as if it were (K,R)); the oracle uses
  conj(E)^T instead and the fixtures record both.
* TV and the NCG driver are pinned against the reference's TVND/RegManager
  and CGSolver run on CPU here (fixtures under ``tests/golden``).
"""
