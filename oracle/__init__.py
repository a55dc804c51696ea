"""Oracles for the electrostatic BEM hot path (test infrastructure only).

``oracle.ref``  -- the reference's own FP64 CPU code compiled from its sources
                   (``oracle/_ref/libkemref.so``, see ``oracle/Makefile``).
``oracle.port`` -- ``kem_oracle.c``, a plain-C restatement of the same path.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
these; the product (``kassiopeia_b200``) never imports them.
"""
