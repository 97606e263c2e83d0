"""CPU oracle for the planogram reconstruction path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker.  The product
library (``petl_b200``) never imports it.
"""
from .oracle import *  # noqa: F401,F403
