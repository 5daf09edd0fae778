"""Parity checkers for the SDTFE density path (test infrastructure only).

Nothing in the shipped library imports this package; tests/, bench.py's CPU
baseline and __graft_entry__.smoke() use it to check the GPU library.
"""
