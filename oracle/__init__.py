"""Test infrastructure only: CPU oracles for the FIR projection path.

``oracle.bridge`` loads the C restatement (``oracle/libfir_oracle.so``) and,
when it was built, the compiled FIR sources (``oracle/_ref/libfirref.so``).
Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this package; the product never imports it.
"""
