"""CPU oracle for the zone crossmatch -- TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the CPU-baseline leg of the benchmark use
this package.  The product (``xmatch_b200``) never imports it.
"""
from .oracle import *  # noqa: F401,F403
