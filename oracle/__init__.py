"""ORACLE -- test infrastructure only.

CPU checkers for the fine-scale kick: the reference's own PP kernel compiled
from its sources (``build_ref.py``), a C restatement of the reference PM3
(``pm3_oracle.c``) and an FP64 Ewald direct sum (``ewald.c``).  Only the test
suite, the smoke check and the CPU-baseline leg of the benchmark may import
this package; the library in ``cube2_b200`` never does.
"""
