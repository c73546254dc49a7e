"""CPU oracle for the interleaved block-cyclic FFT / stencil path.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` -- never by the product package.  It wraps
``liboracle.so`` (``zoracle.c``, a plain-C FP64 restatement of StencilFFT's zmodel
pipeline) and, when they were built, the reference's own host layout code in
``_ref/libzref_host_*.so``.
"""
from .oracle import *  # noqa: F401,F403
