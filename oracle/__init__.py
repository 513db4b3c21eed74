"""ORACLE -- test infrastructure only.

CPU restatements of the reference GLST algorithm (FP64), used as the checker
by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg.
Nothing in the product imports this package.
"""
