"""CPU oracle for the locate + link hot path (test infrastructure only).

Loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
leg; never by the product package.  See gt_oracle.cpp for what it restates
and how it is pinned to the reference.
"""
