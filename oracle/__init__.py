"""Oracle for the sloth_b200 CUDA kernels -- test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs;
never by the sloth_b200 package.
"""
