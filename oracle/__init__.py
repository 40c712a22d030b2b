"""Oracle for the PAVES GPU search path — TEST INFRASTRUCTURE ONLY.

* ``oracle.cpu``: ctypes wrapper of ``paves_oracle.c`` (the CPU
  restatement of the reference algorithms, built by ``make -C oracle``).
* ``oracle.refengine``: ctypes wrapper of the reference engine itself,
  compiled from its own sources by ``make -C oracle ref`` into
  ``oracle/_ref/`` (CPU builds, the drop-in build linked against
  libpaves_gpu.so, and the reference's own GPU backend).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
use this package, as the checker or the timed CPU baseline; the product
(``paves_b200``) never imports it.
"""
