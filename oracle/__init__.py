"""CPU oracle for charming-b200. TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by
the product path."""
