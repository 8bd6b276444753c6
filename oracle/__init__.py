"""CPU checker for the soliton_solver flow hot path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the thing results are checked against
(or timed beside), never by the product package.  ``flow64`` is an FP64 numpy
restatement of the reference's kernels, pinned to golden vectors produced by the
reference itself (``tests/golden``).
"""
