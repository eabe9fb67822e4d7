"""CPU restatement of necsim-rust's Independent algorithm (test infrastructure).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package: it is the parity checker and the timed CPU
baseline, never part of the product path.
"""
from .pyoracle import *  # noqa: F401,F403
