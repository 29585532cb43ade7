"""Test oracle package (CPU restatement of the reference path).  Only the
test suite, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it."""
