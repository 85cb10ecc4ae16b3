"""CPU checker for the engine: a restatement of ParaCOSM's matching semantics
(csm_oracle.cpp) and the reference itself compiled from its sources
(ref_build/).  TEST INFRASTRUCTURE ONLY: imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline / reference legs,
never by the product path.
"""
