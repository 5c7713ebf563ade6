"""B200-native SORD time-stepper (drop-in for Coseis ``cst.sord``).

Use ``from coseis_b200 import sord`` where the reference used ``import cst.sord``.
"""
from . import sord  # noqa: F401
