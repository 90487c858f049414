"""CPU oracle of the igaops matrix-free weighted-quadrature path.

TEST INFRASTRUCTURE ONLY.  This package restates, in plain numpy/scipy, the
reference algorithms of the path (every function cites the reference
file:line it follows).  It is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` import it.  The product (``igaops_b200``) never imports
it and has no CPU path.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every function here
against golden vectors produced by the unmodified reference
(``tests/golden/make_golden.py``, run in a container where the reference
source is mounted, with the ``geomdl`` stand-in of ``oracle/geomdl_shim``).
"""
