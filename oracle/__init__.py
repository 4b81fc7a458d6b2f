"""Test infrastructure: the FP64 CPU oracle and the compiled-reference binding.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.  The product never does.
"""
