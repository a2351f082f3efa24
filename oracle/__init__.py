"""CPU oracle for the TwoPhaseFlow hot path (CCD operator + variable-density PPE).

TEST INFRASTRUCTURE ONLY.  This package is a plain NumPy/SciPy restatement of
the reference's own CPU algorithms (every function cites the reference file and
line it follows).  It is the checker: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import
it.  The product path (``twophaseflow_b200``) never imports or calls it and has
no CPU fallback.

Parity pinning: ``tests/golden/make_golden.py`` runs the reference itself
(``twophase`` imported from its source tree) on seeded inputs and stores the
outputs as ``tests/golden/*.npz``; ``tests/test_oracle_golden.py`` checks this
restatement against those fixtures.

Third-party arithmetic restated here: SciPy 1.18.1 ``scipy.sparse.linalg.cg``
and ``gmres`` (the reference calls them through ``tp/ppe/gmres_helpers.py``),
LAPACK getrf/getrs via ``scipy.linalg.lu_factor/lu_solve`` (dense CCD solve)
and SuperLU via ``scipy.sparse.linalg.spsolve`` (direct FVM solve).
"""
