"""ORACLE — test infrastructure only.

CPU checkers for the graph-diffusion path. Only the test suite, the smoke check
and the CPU-baseline leg of ``bench.py`` may import this package; the product
libraries never load it.

* ``oracle.port`` — ctypes wrapper of ``diffusion_oracle.c``, the plain-C
  restatement of scl-core's diffusion arithmetic (each function cites the
  reference lines it follows).
* ``oracle.ref``  — ctypes wrapper of scl-core's OWN implementation, compiled
  from the reference sources into ``oracle/_ref/`` by ``oracle/Makefile`` with a
  project-written stand-in for the Highway vector header.
"""
