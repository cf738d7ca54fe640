"""Test oracle for the docking hot path (CPU). Not part of the product: only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference legs import it."""
