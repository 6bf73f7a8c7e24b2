"""Test oracle for the Shack-Hartmann frame (test infrastructure only).

:mod:`oracle.ref` drives the reference's OWN C code for the path, compiled in
place into oracle/_ref/libmaosref.so by oracle/Makefile (with stand-ins for the
absent FFTW and BLAS/LAPACK), and the MAOS-side adapter test library
oracle/_ref/libmaosadapter.so.

Only tests/, __graft_entry__ (build, smoke) and bench.py's CPU-baseline and
reference legs use it.
"""
import os

#: The reference source tree the oracle is compiled from: the MAOS_REF
#: environment variable, else this default.  Only the build recipe and the
#: tests that read the tree itself use it; the built library does not.
REF_TREE = os.environ.get("MAOS_REF", "/root/reference")
