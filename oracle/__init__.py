"""Test oracle for conan_b200 (test infrastructure only).

`oracle.cpu` wraps liboracle.so, the FP64 CPU restatement of the reference's
PM path and initial conditions (conan_oracle.cc). `oracle.ref` wraps
_ref/libconan_ref.so, the unmodified reference code compiled from its own
sources, when it has been built. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this package; the product never does.
"""
