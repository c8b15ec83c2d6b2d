"""Test infrastructure only: CPU oracle of ChysX's implicit cloth step.

Nothing in the product package imports this; tests, the smoke check and
bench.py's CPU-baseline / reference arm use it as the checker.
"""
