"""Test oracle for the Shack-Hartmann frame (test infrastructure only).

- :mod:`oracle.ref` drives the reference's OWN C code for the path, compiled in
  place into oracle/_ref/libmaosref.so by oracle/Makefile.
- :mod:`oracle.port` binds liboracle.so, a plain-C restatement of the per-frame
  path that follows the reference line by line.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
