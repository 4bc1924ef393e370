"""CPU oracle for the DWG reconstruction hot path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package: it is the checker, never the product.
"""
from .oracle import *  # noqa: F401,F403
