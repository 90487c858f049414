"""igaops_b200: B200 (sm_100a) matrix-free weighted-quadrature hot path.

A drop-in for the matrix-free path of igaops: the same operator API
(MatrixFree, BsplineOperations, SingleFD / MultiFD, LinearSolver, GCRODR)
with every numerical step in hand-written CUDA kernels (libigab200.so).
"""
from .common import Constants, KronProduct, ParametricDirection, combine_arrays, validate_entry
from .quadrature import StandardGauss, WeightedQuadrature
from .operators import BsplineOperations, MatrixFree, MFOperator
from .geometry import GeometryOps, SingleSpline, precompute_coefficients, unit_cube_ctrlpts
from .nurbs import NurbsMFOperator, NurbsOperations

__all__ = [
    "Constants",
    "KronProduct",
    "ParametricDirection",
    "combine_arrays",
    "validate_entry",
    "StandardGauss",
    "WeightedQuadrature",
    "BsplineOperations",
    "MatrixFree",
    "MFOperator",
    "NurbsOperations",
    "NurbsMFOperator",
    "GeometryOps",
    "SingleSpline",
    "precompute_coefficients",
    "unit_cube_ctrlpts",
]
