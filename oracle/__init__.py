"""CPU oracle for the replay hot path -- TEST INFRASTRUCTURE ONLY.

`oracle.orc` wraps the plain-C restatement (oracle/liboracle.so) and
`oracle.ref` wraps the reference implementation built from its own sources
(oracle/_ref/libref_shim.so, oracle/_ref/replay_ref).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this package,
as the checker; the product never does.
"""
