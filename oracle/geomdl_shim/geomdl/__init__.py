"""Import-time stand-in for ``geomdl`` (test infrastructure only; see helpers.py).

The reference imports ``geomdl.BSpline`` / ``geomdl.NURBS`` only for type
annotations of CAD constructors that are outside the matrix-free path
(``src/igaops/geometry/patch.py:3,29-34``); the stub modules define empty
``Curve``/``Surface``/``Volume`` classes so that import succeeds.
"""
from . import helpers, BSpline, NURBS  # noqa: F401
