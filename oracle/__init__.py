"""CPU restatement of the LightHit per-event transport path (test infrastructure).

This package is the checker, not the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it.
Every function restates the reference algorithm in float64 NumPy and cites the
reference file:line it follows. Parity is pinned against fixtures written by
the reference's own float64 route (``tests/golden/``).
"""
