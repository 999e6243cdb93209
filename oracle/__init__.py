"""Test infrastructure: the CPU oracle and the reference-build harness.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs
import this package, always as the checker or the timed baseline.  The product
(``cavalry_b200``) never imports it.
"""
