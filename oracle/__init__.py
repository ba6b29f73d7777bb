"""CPU oracle for the packed-vector ops hot path (test infrastructure only).

Nothing in the product package imports this; tests/, the smoke check and the
benchmark's CPU-baseline leg load it as the checker.
"""
