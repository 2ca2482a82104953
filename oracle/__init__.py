"""CPU oracle for the beamform -> channelize -> detect path.

TEST INFRASTRUCTURE ONLY.  Nothing in ``blade_b200`` imports this package; only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use it, and only as the checker (or, for ``bench.py --impl reference``, as the
timed CPU restatement of the reference's own numpy formulas).

``formulas`` restates, in FP64 numpy, the arithmetic of the reference modules and
of the numpy oracles in the reference's own tests; every function cites the
reference file:line it follows.  ``loops`` restates the same arithmetic as plain
Python loops in the reference kernels' own loop order, for small cases, and is
used to cross-check ``formulas``.
"""
