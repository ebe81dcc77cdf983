"""CPU oracle of the exact-decimal path — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline and the
reference arm) import this package; the product never does.
"""
