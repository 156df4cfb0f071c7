"""Test-only checkers for diffsoup_b200.

`oracle.cpu` wraps liboracle.so, the CPU restatement of the reference kernels.
`oracle.ref` wraps oracle/_ref/libdsref*.so, the reference's own CUDA sources
built by oracle/Makefile.  Only tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py may import this package.
"""
