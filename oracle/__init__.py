"""Parity oracle for the B200 Datalog engine -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker or the timed CPU
baseline. The product library (``mnmgdatalog_b200``) never imports it.

* ``oracle.cpu``  -- ctypes wrapper over ``liboracle.so``, the C restatement of
  the reference programs (tc.cu, sg.cu, wcc.cu, single_join.cu).
* ``oracle.ops``  -- numpy restatements of the reference's relational idioms
  (thrust sort/unique/set_difference/merge with ``set_cmp``, the hash join).
* ``oracle/_ref`` -- the reference's own programs built from its sources by
  ``oracle/Makefile`` (GPU programs as one MPI rank, and rough/tc_mpi.cpp).
"""
