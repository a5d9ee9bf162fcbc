"""ORACLE — test infrastructure only.

A CPU restatement of the reference crate's LU path (C++, built by
oracle/Makefile into oracle/liboracle.so) and its Python wrapper. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may use it, as the
checker; the product library never links or calls it.
"""
