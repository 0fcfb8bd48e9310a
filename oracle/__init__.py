"""CPU oracle for the LBM time step -- TEST INFRASTRUCTURE ONLY.

A NumPy restatement of the reference solver's step (``ReferenceSolver`` in
``src/lbm/solver.py:224-292`` and the node physics it calls). It is the
checker for the CUDA path: only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it. The product package never
does, and has no CPU fallback.

Parity pinned: ``tests/test_oracle_golden.py`` checks this oracle against
golden vectors produced by the unmodified reference package
(``tests/golden/make_golden.py``).
"""

from .lbm_oracle import (  # noqa: F401
    OracleDiverged,
    OracleSolver,
    collide,
    equilibrium,
    lowbias32,
    quantize,
    stochastic_round,
    stream_pull,
)
