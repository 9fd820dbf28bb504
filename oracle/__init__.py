"""Oracle: test infrastructure, never part of the product.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package. It holds (a) the FP64 CPU restatement of the reference's GPU
render path (oracle/rb_oracle.cpp, built into oracle/_build/liboracle.so) and
(b) bindings to drivers around the reference's own code (oracle/ref/, built
into oracle/_ref/ from the reference's sources by oracle/ref/Makefile).
"""
