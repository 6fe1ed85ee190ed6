"""Test-side checkers for csu_b200 (not product code).

refharness  -- the reference CSU solver compiled from its own sources (oracle/_ref/libcsuref.so)
restated    -- the plain-C restatement of the path (oracle/_build/libcsuoracle.so, csu_oracle.c)
"""
