"""Error and status paths that need no GPU: the convergence manager's
iteration overflow (RuntimeError, src/igaops/solvers/utils/
convergence_manager.py:138-146), argument checks (ValueError), and the map
from C-ABI status codes to Python exceptions."""
import pytest

from igaops_b200 import _lib
from igaops_b200.solvers import ConvergenceManager, GcrodrArgs, SolverArgs


def test_iteration_overflow_raises_runtime_error():
    cm = ConvergenceManager(1e-10, 5)
    cm.update(curr_absolute=1.0, curr_relative=1.0, curr_iteration=5)
    assert not cm.has_converged()
    cm.update(curr_iteration=6)
    with pytest.raises(RuntimeError, match="Maximum iterations"):
        cm.has_converged()


def test_solver_argument_checks():
    with pytest.raises(ValueError):
        SolverArgs(tolerance=2.0, maxiters=10)
    with pytest.raises(ValueError):
        SolverArgs(tolerance=1e-8, maxiters=0)
    with pytest.raises(ValueError):
        GcrodrArgs(tolerance=1e-8, maxiters=10, krylov_size=5, recycled_size=10)


@pytest.mark.parametrize("status,exc", [
    (_lib.IGA_ERR_INVALID_ARG, ValueError),
    (_lib.IGA_ERR_UNSUPPORTED, NotImplementedError),
    (_lib.IGA_ERR_TIMEOUT, TimeoutError),
    (_lib.IGA_ERR_NONFINITE, FloatingPointError),
    (_lib.IGA_ERR_GEOMETRY, ValueError),
    (_lib.IGA_ERR_CUDA, RuntimeError),
])
def test_status_codes_map_to_exceptions(status, exc):
    with pytest.raises(exc):
        _lib.check(status)
    _lib.check(_lib.IGA_OK)
