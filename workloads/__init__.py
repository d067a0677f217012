"""Seeded synthetic workloads with the shapes of the benchmark configurations.

This package imports nothing from ``cusbf_b200``: the reference arm of
``bench.py`` and the golden-fixture script use it without loading the engine's
library.
"""
