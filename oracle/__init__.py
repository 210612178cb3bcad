"""TEST INFRASTRUCTURE ONLY: the CPU oracle of the EMSES particle path.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg
as the checker; never by the product package ctca_b200.
"""
