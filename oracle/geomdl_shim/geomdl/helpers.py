"""Minimal stand-in for the third-party ``geomdl.helpers`` module.

TEST INFRASTRUCTURE ONLY.  The unmodified igaops reference imports
``geomdl`` (``pyproject.toml:29``, ``geomdl>=5.4``, no lock file, so no pinned
version) for B-spline span search and basis-derivative evaluation
(``src/igaops/quadrature/utils/operations.py:86-89``,
``src/igaops/quadrature/utils/template.py:104``).  ``geomdl`` is not installed
in this image and cannot be installed, so this module restates the published
algorithms it implements:

* ``find_span_linear``   -- linear knot-span search (Piegl & Tiller,
  *The NURBS Book*, 2nd ed., Alg. A2.1, linear-search variant): the span is the
  last index ``s`` in ``[p, n-1]`` with ``U[s] <= u``; ``u = U[-1]`` maps to
  the last non-empty span.
* ``basis_function_ders`` -- non-zero basis functions and their derivatives
  up to order ``nd`` at ``u`` (Alg. A2.3), returned as ``ders[k][j]``.
* ``find_multiplicity``  -- number of knots equal to ``u`` within a small
  absolute tolerance.

It is placed on ``sys.path`` only by the golden-fixture generator that imports
the reference; nothing in the product imports it.
"""


def find_span_linear(degree, knot_vector, num_ctrlpts, knot, **kwargs):
    span = degree + 1
    while span < num_ctrlpts and knot_vector[span] <= knot:
        span += 1
    return span - 1


def find_multiplicity(knot, knot_vector, **kwargs):
    tol = kwargs.get("tol", 1e-7)
    return sum(1 for k in knot_vector if abs(knot - k) <= tol)


def basis_function_ders(degree, knot_vector, span, knot, order):
    p = degree
    U = knot_vector
    u = knot
    # ndu[j][r]: basis values (upper triangle) and knot differences (lower)
    ndu = [[1.0 for _ in range(p + 1)] for _ in range(p + 1)]
    left = [1.0] * (p + 1)
    right = [1.0] * (p + 1)
    for j in range(1, p + 1):
        left[j] = u - U[span + 1 - j]
        right[j] = U[span + j] - u
        saved = 0.0
        for r in range(j):
            ndu[j][r] = right[r + 1] + left[j - r]
            temp = ndu[r][j - 1] / ndu[j][r]
            ndu[r][j] = saved + right[r + 1] * temp
            saved = left[j - r] * temp
        ndu[j][j] = saved

    ders = [[0.0 for _ in range(p + 1)] for _ in range(order + 1)]
    for j in range(p + 1):
        ders[0][j] = ndu[j][p]

    a = [[1.0 for _ in range(p + 1)] for _ in range(2)]
    for r in range(p + 1):
        s1, s2 = 0, 1
        a[0][0] = 1.0
        for k in range(1, order + 1):
            d = 0.0
            rk = r - k
            pk = p - k
            if r >= k:
                a[s2][0] = a[s1][0] / ndu[pk + 1][rk]
                d = a[s2][0] * ndu[rk][pk]
            j1 = 1 if rk >= -1 else -rk
            j2 = k - 1 if (r - 1) <= pk else p - r
            for j in range(j1, j2 + 1):
                a[s2][j] = (a[s1][j] - a[s1][j - 1]) / ndu[pk + 1][rk + j]
                d += a[s2][j] * ndu[rk + j][pk]
            if r <= pk:
                a[s2][k] = -a[s1][k - 1] / ndu[pk + 1][r]
                d += a[s2][k] * ndu[r][pk]
            ders[k][r] = d
            s1, s2 = s2, s1

    r = p
    for k in range(1, order + 1):
        for j in range(p + 1):
            ders[k][j] *= r
        r *= p - k
    return ders
