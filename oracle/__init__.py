"""Test oracle for the gtomrln CUDA library (TEST INFRASTRUCTURE ONLY).

See oracle/oracle.py.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this package; the product (gtom_b200/) never does.
"""
