"""Import-time stub: the reference imports ``geomdl.BSpline`` (geometry/patch.py:3)."""


class Surface:
    pass


class Volume:
    pass


class Curve:
    pass
