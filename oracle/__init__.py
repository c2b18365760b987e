"""Test infrastructure: the checker the device solver is compared with.

``oracle.port`` binds the CPU restatement in cfd_oracle.c (built to
``oracle/_build/liboracle.so``); ``oracle.reference`` binds the reference
solver itself, compiled from its own sources into ``oracle/_ref/libcfdref.so``
where those sources were available at build time. Only tests, the smoke check
and the CPU-baseline leg of bench.py import this package; the product never
does.
"""
