"""CPU oracle -- test infrastructure only (tests/, __graft_entry__.smoke(),
bench.py's CPU-baseline and reference legs).  Never imported by mercury_b200.

oracle.core wraps liboracle.so, the C restatement of the reference step
(mercury_oracle.c); oracle.ref wraps oracle/_ref/, the reference's own code
compiled from its sources (ref_harness.cpp, Makefile).
"""
