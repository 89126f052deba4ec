"""CPU oracle for the cupoly_b200 hot path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (``cupoly_b200``) imports this package.  Only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, and only as the checker
or as the timed CPU baseline.

Two restatements of cuPoly's algorithms live here:

* ``oracle.pyoracle``  -- pure-Python big-integer restatement (exact
  definitions plus a bit-exact restatement of cuPoly's hierarchical DGT);
* ``oracle/cpoly_oracle.c`` -- the same integer algorithms in C with
  ``unsigned __int128`` and OpenMP, loaded through ``oracle.coracle``; it
  is the fast checker at full sizes and the timed CPU baseline.
"""
