"""Test infrastructure: CPU oracle for the fastPLS model-fitting path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package, always as the checker. The product (fastpls_b200) never does.
"""
