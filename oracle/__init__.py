"""Test-only checkers for the delay-and-sum path (CPU FP64 restatement, FP32 CPU
loop, and a wrapper for the reference library built from its sources).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference
legs use this package, as checkers.  Product code never imports it.
"""
