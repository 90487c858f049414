"""Fast-diagonalisation (FD) preconditioner, applied on the GPU.

* ``SpaceFD``  -- src/igaops/fastdiag/utils/space_precond.py:20-320
* ``SingleFD`` -- src/igaops/fastdiag/preconditioner.py:15-197
  (alias ``SingleFastDiagonalization``)
* ``MultiFD``  -- src/igaops/fastdiag/multi_preconditioner.py:13-103
* ``SpaceTimeFD`` -- src/igaops/fastdiag/utils/time_arrow.py:16-192 (arrowhead)

Setup (per direction: dense 1D Gauss mass/stiffness pencils, Dirichlet rows
removed, generalized symmetric eigenproblem in FP64) is small 1D work done on
the host once, as in the reference.  The apply -- gather the free box,
d mode products with U^T, scale by 1/Lambda, d mode products with U, scatter
-- runs in libigab200 (iga_fd_apply).
"""
from __future__ import annotations

import ctypes
import logging
import math
import threading
from typing import Dict, List, Literal, Optional, Sequence, Tuple

import numpy as np
import scipy.linalg as sclin
import scipy.sparse as sp
import torch

from . import _lib
from ._device import compute_dtype, iga_dtype, like_input, require_cuda, stream_handle, to_device
from .common import Constants, KronProduct, ParametricDirection, combine_arrays, validate_entry
from .quadrature import StandardGauss

logger = logging.getLogger(__name__)


def _tile_kmajor_bf16(Bm: np.ndarray, dev) -> torch.Tensor:
    """BF16 image of the (N x K) matrix Bm padded to multiples of 16 and laid
    out in 8x8 core matrices: core (g, kc) at element (kc*Np/8 + g)*64, each
    core 8 rows of 8 contiguous K elements (the no-swizzle K-major operand
    layout of the tensor-core MMA)."""
    nr, kr = Bm.shape
    Np = -(-nr // 16) * 16
    Kp = -(-kr // 16) * 16
    P = np.zeros((Np, Kp), dtype=np.float32)
    P[:nr, :kr] = Bm
    img = P.reshape(Np // 8, 8, Kp // 8, 8).transpose(2, 0, 1, 3).reshape(-1)
    return torch.from_numpy(np.ascontiguousarray(img)).to(dev).to(torch.bfloat16).contiguous()


# 1D Gauss pencils (mass, stiffness) and their generalized eigenpairs per
# spline (degree, knot vector), kept across preconditioner builds: a serving
# loop builds one preconditioner per request, and requests repeat
# discretisations. Bounded LRU; entries are private copies.
_PENCIL_CACHE: "OrderedDict" = None
_PENCIL_CACHE_MAX = 512


def _cache():
    global _PENCIL_CACHE
    if _PENCIL_CACHE is None:
        from collections import OrderedDict

        _PENCIL_CACHE = OrderedDict()
    return _PENCIL_CACHE


def clear_pencil_cache():
    """Drop the kept 1D pencils and eigenpairs (e.g. to time a cold start)."""
    if _PENCIL_CACHE is not None:
        with _PENCIL_LOCK:
            _PENCIL_CACHE.clear()


_PENCIL_LOCK = threading.Lock()


def _cache_get(key, make):
    # the serving loop sets patches up on several threads: the lookup and
    # the insertion hold the lock, the computation does not (two threads may
    # both compute a missing entry; either result is the same)
    c = _cache()
    with _PENCIL_LOCK:
        hit = c.get(key)
        if hit is not None:
            c.move_to_end(key)
            return hit
    val = make()
    with _PENCIL_LOCK:
        c[key] = val
        if len(c) > _PENCIL_CACHE_MAX:
            c.popitem(last=False)
    return val


def _spline_key(q):
    """Cache key of the Gauss rewrite of rule q, or None when q is itself a
    Gauss-Legendre rule (then its own matrices are used, uncached)."""
    if getattr(q, "quadrature_class", None) == "GAUSS" and getattr(q, "quadrature_type", None) == "legendre":
        return None
    kv = np.ascontiguousarray(np.asarray(q.knotvector, dtype=np.float64))
    return (int(q.degree), kv.tobytes())


def _gauss_pencil(q):
    """Dense 1D Gauss mass and stiffness matrices of rule q's spline."""
    def make():
        (g,) = rewrite_quadrature([q])
        mass = sp.csr_array(g.weights[0] @ g.basis[0]).toarray()
        stiff = sp.csr_array(g.weights[-1] @ g.basis[-1]).toarray()
        return mass, stiff

    key = _spline_key(q)
    if key is None:
        return make()
    return _cache_get(("pencil",) + key, make)


def rewrite_quadrature(quadrule_list):
    """Gauss-Legendre rules on the same splines (fastdiag/utils/template.py:28-45)."""
    if not isinstance(quadrule_list, (list, tuple)):
        raise ValueError("quadrule_list should be iterable")
    out = []
    for q in quadrule_list:
        if getattr(q, "quadrature_class", None) == "GAUSS" and getattr(q, "quadrature_type", None) == "legendre":
            out.append(q)
        else:
            out.append(StandardGauss(degree=q.degree, knotvector=q.knotvector, quadtype="legendre"))
    return out


def _box_complement(n: Sequence[int], lo: Sequence[int], m: Sequence[int]) -> np.ndarray:
    """Sorted flat indices (direction 1 fastest) of the grid n[0] x n[1] x ...
    outside the box lo[d] .. lo[d] + m[d] - 1: the disjoint sets "outside in
    direction d, inside in every slower direction", each an outer sum."""
    nd = len(n)
    stride = [1] * nd
    for d in range(1, nd):
        stride[d] = stride[d - 1] * int(n[d - 1])
    parts = []
    for d in range(nd - 1, -1, -1):
        rng_d = np.arange(int(n[d]), dtype=np.int64)
        out_d = rng_d[(rng_d < lo[d]) | (rng_d >= lo[d] + m[d])]
        if out_d.size == 0:
            continue
        idx = out_d * stride[d]
        for e in range(nd - 1, -1, -1):  # slower: inside the box; faster: all
            if e == d:
                continue
            vals = (np.arange(lo[e], lo[e] + m[e], dtype=np.int64) if e > d
                    else np.arange(int(n[e]), dtype=np.int64)) * stride[e]
            idx = (idx[:, None] + vals[None, :]).reshape(-1)
        parts.append(idx)
    if not parts:
        return np.zeros(0, dtype=np.int64)
    return np.sort(np.concatenate(parts))


class SpaceFD:
    """Spatial FD preconditioner of one patch."""

    def __init__(self):
        self._nonzeros_by_dir: Dict[ParametricDirection, int] = {}
        self._indices_by_dir: Dict[Tuple[int, ParametricDirection], List[int]] = {}
        self._nbDoFsPerNode = 0
        self._space_dirs: List[ParametricDirection] = []
        self._space_free_nodes: List[np.ndarray] = []  # int64 arrays, one per DOF per node
        self._space_free_lists: Optional[List[List[int]]] = None
        self._space_table_dirichlet = np.array([])
        self._space_scalar_coefs: Tuple[float, float] = (0.0, 1.0)
        self._space_eigenvalues: Optional[List[np.ndarray]] = None
        self._eigenvec_by_dir_space: List[List[np.ndarray]] = []
        self._eigenval_by_dir_space: List[List[np.ndarray]] = []
        self._mass_space_corrector: Sequence[float] = []
        self._stiff_space_corrector: Sequence[np.ndarray] = []
        self._boxes: List[Tuple[List[int], List[int]]] = []
        self._dev: Dict[tuple, list] = {}

    # ---- properties (same names as the reference)
    @property
    def space_free_nodes(self) -> List[List[int]]:
        """Free DOFs per DOF-per-node block, as lists (the reference's type;
        converted once on first use -- `free_nodes` is the array form)."""
        if self._space_free_lists is None:
            self._space_free_lists = [a.tolist() for a in self._space_free_nodes]
        return self._space_free_lists

    def free_nodes(self, node: int = 0) -> np.ndarray:
        """Free DOFs of one DOF-per-node block as an int64 array."""
        return self._space_free_nodes[node]

    def dirichlet_nodes(self, node: int = 0) -> np.ndarray:
        """The other DOFs (sorted int64): the complement of the free box,
        built from its faces (indices outside the box in the slowest
        direction, then in the next, ...) instead of a mask over every DOF."""
        lo, mm = self._boxes[node]
        n = [self._nonzeros_by_dir[d] for d in self._space_dirs]
        return _box_complement(n, lo, mm)

    nonzeros_by_dir = property(lambda self: self._nonzeros_by_dir)
    indices_by_dir = property(lambda self: self._indices_by_dir)
    nbDoFsPerNode = property(lambda self: self._nbDoFsPerNode)
    space_dirs = property(lambda self: self._space_dirs)
    space_table_dirichlet = property(lambda self: self._space_table_dirichlet)
    space_scalar_coefs = property(lambda self: self._space_scalar_coefs)
    eigenvec_by_dir_space = property(lambda self: self._eigenvec_by_dir_space)
    eigenval_by_dir_space = property(lambda self: self._eigenval_by_dir_space)
    mass_space_corrector = property(lambda self: self._mass_space_corrector)
    stiff_space_corrector = property(lambda self: self._stiff_space_corrector)

    @property
    def sp_nnz(self):
        return int(np.prod([v for k, v in self._nonzeros_by_dir.items()
                            if k != ParametricDirection.TAU]))

    @property
    def space_eigenvalues(self):
        if self._space_eigenvalues is None:
            self._space_eigenvalues = self.update_space_eigenvalues(self._space_scalar_coefs)
            self._dev.clear()
        return self._space_eigenvalues

    # ---- setup
    def compute_space_eigendecomposition(self, space_quadrule_list, space_table_dirichlet):
        """Per direction and DOF-per-node: eigh(K_d, M_d) of the Gauss pencils
        minus the Dirichlet rows (space_precond.py:124-193)."""
        if not isinstance(space_quadrule_list, (list, tuple)):
            raise ValueError("quadrule_list should be iterable")
        pencils = [_gauss_pencil(q) for q in space_quadrule_list]
        mass = [m for m, _ in pencils]
        stiff = [k for _, k in pencils]
        keys = [_spline_key(q) for q in space_quadrule_list]
        nnz_list = [m.shape[0] for m in mass]
        table = np.asarray(space_table_dirichlet, dtype=bool)
        ndof, ndirs, _ = table.shape
        ndirs = min(ndirs, len(space_quadrule_list))
        dirs = [ParametricDirection(i) for i in range(ndirs)]
        nnz_by_dir, idx_by_dir = {}, {}
        eig_keys = {}
        mcorr, scorr, vecs_all, vals_all, boxes = [], [], [], [], []
        for ii in range(ndof):
            vecs, vals, lo, mm = [], [], [], []
            mcorr.append(1.0)
            scorr.append(np.ones(ndirs))
            for jj, sd in enumerate(dirs):
                nnz = nnz_list[jj]
                a = 1 if table[ii, jj, 0] else 0
                b = nnz - 1 if table[ii, jj, 1] else nnz
                idx = list(range(a, b))
                nnz_by_dir[sd] = nnz
                idx_by_dir[(ii, sd)] = idx
                def eig(jj=jj, idx=idx, nnz=nnz):
                    Bm = mass[jj][np.ix_(idx, idx)]
                    Am = stiff[jj][np.ix_(idx, idx)]
                    if nnz == len(idx):
                        Am = Am + Constants.TINY * Bm  # no Dirichlet row: avoid a null eigenvalue
                    w, V = sclin.eigh(Am, Bm)
                    return np.real(w), np.real(V)

                if keys[jj] is None:
                    w, V = eig()
                    eig_keys[(ii, jj)] = None
                else:
                    w, V = _cache_get(("eig",) + keys[jj] + (a, b), eig)
                    eig_keys[(ii, jj)] = ("eig",) + keys[jj] + (a, b)
                vecs.append(V.copy())
                vals.append(w.copy())
                lo.append(a)
                mm.append(len(idx))
            vecs_all.append(vecs)
            vals_all.append(vals)
            boxes.append((lo, mm))
        self._nonzeros_by_dir = nnz_by_dir
        self._indices_by_dir = idx_by_dir
        self._nbDoFsPerNode = ndof
        self._space_dirs = dirs
        self._space_table_dirichlet = table
        self._eigenvec_by_dir_space = vecs_all
        self._eigenval_by_dir_space = vals_all
        self._mass_space_corrector = mcorr
        self._stiff_space_corrector = scorr
        self._boxes = boxes
        self._eig_keys = eig_keys  # pencil-cache keys of the eigenpairs (None: not cached)
        self._space_free_nodes = self._propagate_nodes_in_space()
        self._space_free_lists = None
        self._space_eigenvalues = None
        self._dev.clear()

    def _propagate_nodes_in_space(self):
        out = [np.zeros(0, dtype=np.int64) for _ in range(self._nbDoFsPerNode)]
        if not (self._indices_by_dir and self._nonzeros_by_dir):
            return out
        nnz = [self._nonzeros_by_dir[d] for d in self._space_dirs][::-1]
        for ii in range(self._nbDoFsPerNode):
            idx = [self._indices_by_dir.get((ii, d), []) for d in self._space_dirs[::-1]]
            out[ii] = KronProduct.kron_nonzero_array(idx, nnz)
        return out

    def update_space_eigenvalues(self, scalar_coefs: Sequence[float]) -> List[np.ndarray]:
        """Lambda = c0 * mass_corr + c1 * sum_d corr_d lambda_d (kron sum),
        floored at 1e-14 * max (space_precond.py:195-236)."""
        out = []
        if len(scalar_coefs) < 2:
            return out
        for ii in range(self._nbDoFsPerNode):
            mixed = combine_arrays(self._eigenval_by_dir_space[ii], self._stiff_space_corrector[ii])
            cur = (scalar_coefs[0] * self._mass_space_corrector[ii] * np.ones_like(mixed)
                   + scalar_coefs[1] * mixed)
            cur = np.maximum(cur, Constants.SAFEGUARD * np.max(cur))
            out.append(cur)
        self._space_scalar_coefs = (float(scalar_coefs[0]), float(scalar_coefs[1]))
        return out

    def add_scalar_space_correctors(self, mass_corrector=None, stiffness_corrector=None):
        def ok(e):
            return isinstance(e, (list, tuple)) and len(e) == self._nbDoFsPerNode

        if mass_corrector is not None and ok(mass_corrector):
            self._mass_space_corrector = mass_corrector
            self._space_eigenvalues = None
            self._dev.clear()  # the device data holds (1 / Lambda)
        if stiffness_corrector is not None and ok(stiffness_corrector):
            self._stiff_space_corrector = stiffness_corrector
            self._space_eigenvalues = None
            self._dev.clear()

    # ---- device data
    def device_data(self, dtype: torch.dtype):
        eig = self.space_eigenvalues
        hit = self._dev.get(dtype)
        if hit is None:
            dev = require_cuda()
            hit = []
            for ii in range(self._nbDoFsPerNode):
                U = [torch.from_numpy(np.ascontiguousarray(u)).to(dev, dtype)
                     for u in self._eigenvec_by_dir_space[ii]]
                inv = torch.from_numpy(1.0 / eig[ii]).to(dev, dtype)
                hit.append((U, inv))
            self._dev[dtype] = hit
        return hit

    def apply_device(self, x: torch.Tensor, y: torch.Tensor, ncols: int = 1, node: int = 0,
                     work: Optional[Tuple[torch.Tensor, torch.Tensor]] = None):
        """y = P^{-1} x for one DOF-per-node block; x, y (N*ncols) with the
        column index fastest; device hot path (no host sync)."""
        U, inv = self.device_data(x.dtype)[node]
        lo, mm = self._boxes[node]
        ndim = len(mm)
        n = [self._nonzeros_by_dir[d] for d in self._space_dirs]
        M = math.prod(mm)
        if work is None:
            work = (torch.empty(M * ncols, dtype=x.dtype, device=x.device),
                    torch.empty(M * ncols, dtype=x.dtype, device=x.device))
        arr = ctypes.c_int32 * ndim
        ptrs = (ctypes.c_void_p * ndim)(*[u.data_ptr() for u in U])
        _lib.check(
            _lib.LIB.iga_fd_apply(iga_dtype(x.dtype), ndim, arr(*n), arr(*lo), arr(*mm), ptrs,
                                  inv.data_ptr(), ncols, x.data_ptr(), y.data_ptr(),
                                  work[0].data_ptr(), work[1].data_ptr(), stream_handle())
        )

    # ---- tensor-core (BF16) apply, 3D, one DOF per node
    def tc_data(self, node: int = 0):
        """Device data of the BF16 tensor-core apply (built once): the tiled
        BF16 images of U_d^T / U_d (kept across builds per spline and box,
        like the eigenpairs), 1/Lambda in FP32 computed on the device from
        the 1D eigenvalues (the host Lambda's arithmetic, in its order), the
        BF16 work tensors and the status word."""
        key = ("tc", node)
        hit = self._dev.get(key)
        if hit is None:
            dev = require_cuda()
            lo, mm = self._boxes[node]
            if len(mm) != 3:
                raise NotImplementedError("the tensor-core FD apply covers 3D patches")
            if max(mm) > 256:
                raise NotImplementedError("the tensor-core FD apply covers free extents <= 256")
            fwd, bwd = [], []
            for jj, U in enumerate(self._eigenvec_by_dir_space[node]):
                ek = getattr(self, "_eig_keys", {}).get((node, jj))
                make = (lambda U=U: (_tile_kmajor_bf16(U.T, dev), _tile_kmajor_bf16(U, dev)))
                f, b = make() if ek is None else _cache_get(("tc_img", str(dev)) + ek, make)
                fwd.append(f)
                bwd.append(b)
            inv = self._inv_lambda_device(node, dev)
            elems = ctypes.c_int64(0)
            _lib.check(_lib.LIB.iga_fd_tc_workspace((ctypes.c_int32 * 3)(*mm), ctypes.byref(elems)))
            work = (torch.zeros(int(elems.value), dtype=torch.bfloat16, device=dev),
                    torch.zeros(int(elems.value), dtype=torch.bfloat16, device=dev))
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            hit = (fwd, bwd, inv, work, status)
            self._dev[key] = hit
        return hit

    def _inv_lambda_device(self, node: int, dev) -> torch.Tensor:
        """1 / Lambda (FP32, direction 1 fastest) for the tensor-core apply,
        formed on the device with the operations of update_space_eigenvalues
        in their order (Kronecker sum by broadcasting, the scalar mix, the
        1e-14 * max floor, the FP64 reciprocal), so it equals the host
        array's conversion bit for bit without forming it on the host."""
        if self._space_eigenvalues is not None:
            return torch.from_numpy(1.0 / self._space_eigenvalues[node]).to(dev, torch.float32)
        vals = self._eigenval_by_dir_space[node]
        corr = self._stiff_space_corrector[node]
        c0, c1 = self._space_scalar_coefs
        nd = len(vals)
        total = None
        for i in range(nd):
            term = torch.from_numpy(np.asarray(vals[i]) * corr[i]).to(dev)
            term = term.reshape([-1 if k == nd - 1 - i else 1 for k in range(nd)])
            total = term if total is None else total + term
        shape = [len(v) for v in vals][::-1]
        mixed = total.expand(shape).reshape(-1)
        const = c0 * self._mass_space_corrector[node]
        cur = const + c1 * mixed
        cur = torch.maximum(cur, Constants.SAFEGUARD * cur.max())
        return (1.0 / cur).to(torch.float32)

    def apply_device_tc(self, x: torch.Tensor, y: torch.Tensor, node: int = 0):
        """y = P^{-1} x with BF16 tensor-core mode products (FP32 accumulation);
        x, y full FP32 or FP64 vectors on the device."""
        fwd, bwd, inv, work, status = self.tc_data(node)
        lo, mm = self._boxes[node]
        n = [self._nonzeros_by_dir[d] for d in self._space_dirs]
        arr = ctypes.c_int32 * 3
        pf = (ctypes.c_void_p * 3)(*[b.data_ptr() for b in fwd])
        pb = (ctypes.c_void_p * 3)(*[b.data_ptr() for b in bwd])
        _lib.check(
            _lib.LIB.iga_fd_apply_tc(iga_dtype(x.dtype), arr(*n), arr(*lo), arr(*mm), pf, pb,
                                     inv.data_ptr(), x.data_ptr(), y.data_ptr(),
                                     work[0].data_ptr(), work[1].data_ptr(), status.data_ptr(),
                                     stream_handle())
        )

    def check_tc_status(self, node: int = 0):
        status = self.tc_data(node)[4]
        st = int(status.item())
        if st:
            status.zero_()
            _lib.check(st)

    def apply(self, array_in):
        dtype = compute_dtype(array_in)
        x = to_device(array_in, dtype)
        tail = tuple(x.shape[1:])
        n1 = self._nbDoFsPerNode
        n2 = x.shape[0] // n1
        k = math.prod(tail) if tail else 1
        xr = x.reshape(n1, n2 * k)
        out = torch.empty_like(xr)
        for ii in range(n1):
            self.apply_device(xr[ii].contiguous(), out[ii], k, ii)
        return like_input(out.reshape((-1,) + tail), array_in)


class SpaceTimeFD:
    """Space-time FD preconditioner in arrowhead form
    (src/igaops/fastdiag/utils/time_arrow.py:16-192, time_template.py:12-140).

    Setup (host, FP64/complex128, as the reference): the time pencil
    (advection W_t = weights[1] @ basis[1], mass M_t = weights[0] @ basis[0])
    of the Gauss-rewritten time rule without the first time DOF (time is
    always constrained at t = 0); generalized eigenvectors of its leading
    block normalised in the mass inner product, completed by the
    mass-orthogonal vector [M_p^{-1}(-m), 1]: U_t^H M_t U_t = I and
    U_t^H W_t U_t = [[diag(D), g], [-g^H, sigma]].
    Apply (device, ``iga_fd_sptime_apply``): space and time mode products
    and the arrowhead solve on the free space-time box."""

    def __init__(self, space_fd: SpaceFD):
        self._space_fd = space_fd
        self._eigenvec_time = np.array([])
        self._eigenblocks_time: List[np.ndarray] = []
        self._advection_time_corrector: Sequence[float] = []
        self._sptm_free_nodes: List[List[int]] = []
        self._nt = 0
        self._dev: Dict[tuple, tuple] = {}

    space_fd = property(lambda self: self._space_fd)
    nbDoFsPerNode = property(lambda self: self._space_fd.nbDoFsPerNode)
    nonzeros_by_dir = property(lambda self: self._space_fd.nonzeros_by_dir)
    indices_by_dir = property(lambda self: self._space_fd.indices_by_dir)
    eigenvec_time = property(lambda self: self._eigenvec_time)
    eigenblocks_time = property(lambda self: self._eigenblocks_time)
    sptm_free_nodes = property(lambda self: self._sptm_free_nodes)
    advection_time_corrector = property(lambda self: self._advection_time_corrector)

    @property
    def tm_nnz(self):
        return self.nonzeros_by_dir.get(ParametricDirection.TAU, 0)

    def compute_time_schurdecomposition(self, time_quadrule):
        q = rewrite_quadrature([time_quadrule])[0]
        Mfull = sp.csr_array(q.weights[0] @ q.basis[0]).toarray()
        Wfull = sp.csr_array(q.weights[1] @ q.basis[1]).toarray()
        nt = Mfull.shape[0]
        idx = list(range(1, nt))
        self.nonzeros_by_dir[ParametricDirection.TAU] = nt
        self.indices_by_dir[(0, ParametricDirection.TAU)] = idx
        Wt = Wfull[np.ix_(idx, idx)]
        Mt = Mfull[np.ix_(idx, idx)]
        k = len(idx) - 1
        Wp, Mp = Wt[:k, :k], Mt[:k, :k]
        D, V = sclin.eig(Wp, Mp)
        for i in range(V.shape[1]):
            nrm = np.sqrt(np.abs(np.vdot(V[:, i], Mp @ V[:, i])))
            V[:, i] = V[:, i] / nrm
        v = np.linalg.solve(Mp, -Mt[:k, k]) if k > 0 else np.zeros(0)
        last = np.append(v, 1.0)
        last = last / np.sqrt(last @ (Mt @ last))
        Ut = np.zeros((k + 1, k + 1), dtype=complex)
        Ut[:k, :k] = V
        Ut[:k, k] = last[:k]
        Ut[k, k] = last[k]
        g = V.conj().T @ (Wt[:k, :] @ last)
        sigma = last @ (Wt @ last)
        self._eigenvec_time = Ut
        self._eigenblocks_time = [np.append(D, sigma), np.ravel(g)]
        self._nt = nt
        self._advection_time_corrector = [1.0] * self.nbDoFsPerNode
        self._sptm_free_nodes = self._propagate_nodes_in_time()
        self._dev.clear()

    def _propagate_nodes_in_time(self):
        nt = self._nt
        Ns = self._space_fd.sp_nnz
        out = []
        for ii in range(self.nbDoFsPerNode):
            sfree = self._space_fd.free_nodes(ii)
            out.append((np.arange(1, nt, dtype=np.int64)[:, None] * Ns + sfree[None, :]).reshape(-1).tolist())
        return out

    def add_scalar_time_correctors(self, advection_corrector=None):
        if (advection_corrector is not None and isinstance(advection_corrector, (list, tuple))
                and len(advection_corrector) == self.nbDoFsPerNode):
            self._advection_time_corrector = advection_corrector
            self._dev.clear()

    def device_data(self, dtype: torch.dtype, node: int = 0):
        sp_fd = self._space_fd
        lam = sp_fd.space_eigenvalues[node]
        key = (dtype, node, id(lam))
        hit = self._dev.get(key)
        if hit is None:
            dev = require_cuda()
            adv = float(self._advection_time_corrector[node])
            Dt, g = self._eigenblocks_time
            gs = adv * g

            def cplx(a):
                a = np.asarray(a, dtype=complex)
                return torch.from_numpy(np.ascontiguousarray(
                    np.stack([a.real, a.imag], axis=-1).reshape(-1))).to(dev)

            U = [torch.from_numpy(np.ascontiguousarray(u)).to(dev, dtype)
                 for u in sp_fd.eigenvec_by_dir_space[node]]
            Ut = self._eigenvec_time
            ut_re = torch.from_numpy(np.ascontiguousarray(Ut.real)).to(dev, dtype)
            ut_im = torch.from_numpy(np.ascontiguousarray(Ut.imag)).to(dev, dtype)
            lo, mm = sp_fd._boxes[node]
            n = [sp_fd.nonzeros_by_dir[d] for d in sp_fd.space_dirs] + [self._nt]
            lo = list(lo) + [1]
            mm = list(mm) + [self._nt - 1]
            M = math.prod(mm)
            work = [torch.empty(M, dtype=dtype, device=dev) for _ in range(3)]
            hit = dict(U=U, ut_re=ut_re, ut_im=ut_im, dt=cplx(adv * Dt),
                       b=cplx(gs) if gs.size else torch.zeros(2, dtype=torch.float64, device=dev),
                       bT=cplx(-np.conj(gs)) if gs.size else torch.zeros(2, dtype=torch.float64, device=dev),
                       lam=torch.from_numpy(np.ascontiguousarray(lam)).to(dev, torch.float64),
                       n=n, lo=lo, m=mm, work=work)
            self._dev = {key: hit}
        return hit

    def apply_device(self, x: torch.Tensor, y: torch.Tensor, transpose: bool = False,
                     node: int = 0):
        """y = P^{-1} x (or P^{-T} x) for one DOF-per-node block; x, y full
        space-time vectors on the device (time slowest)."""
        h = self.device_data(x.dtype, node)
        sd = len(h["U"])
        arr = ctypes.c_int32 * (sd + 1)
        ptrs = (ctypes.c_void_p * sd)(*[u.data_ptr() for u in h["U"]])
        w = h["work"]
        _lib.check(_lib.LIB.iga_fd_sptime_apply(
            iga_dtype(x.dtype), sd, arr(*h["n"]), arr(*h["lo"]), arr(*h["m"]), ptrs,
            h["ut_re"].data_ptr(), h["ut_im"].data_ptr(), h["dt"].data_ptr(),
            (h["bT"] if transpose else h["b"]).data_ptr(), h["lam"].data_ptr(), int(transpose),
            x.data_ptr(), y.data_ptr(), w[0].data_ptr(), w[1].data_ptr(), w[2].data_ptr(),
            stream_handle()))

    def _apply(self, array_in, transpose):
        dtype = compute_dtype(array_in)
        x = to_device(array_in, dtype)
        tail = tuple(x.shape[1:])
        n1 = self.nbDoFsPerNode
        k = math.prod(tail) if tail else 1
        xr = x.reshape(n1, -1, k)
        out = torch.empty_like(xr)
        for ii in range(n1):
            for c in range(k):
                xc = xr[ii, :, c].contiguous()
                yc = torch.empty_like(xc)
                self.apply_device(xc, yc, transpose, ii)
                out[ii, :, c] = yc
        return like_input(out.reshape((-1,) + tail), array_in)

    def apply(self, array_in):
        return self._apply(array_in, False)

    def apply_transpose(self, array_in):
        return self._apply(array_in, True)


class SpaceTimeQZFD(SpaceTimeFD):
    """Space-time FD preconditioner in the QZ ("legacy") form
    (src/igaops/fastdiag/utils/time_legacy.py:16-170): the time pencil
    (advection W_t, mass M_t; same matrices as the arrowhead form) is
    reduced by the complex generalized Schur decomposition
    W_t = Q S Z^H, M_t = Q T Z^H (scipy.linalg.qz on the host, as the
    reference); the apply is, on the free space-time box,
        x -> (U_s^T per space direction) -> (Q^H in time)
          -> per spatial eigen-index j: solve (adv S + lam_j T) y = . (upper
             triangular, complex) -> (Z in time) -> (U_s) -> real part,
    and the transpose uses Z^T, the lower-triangular (adv S + lam_j T)^T and
    conj(Q).  Device: ``iga_fd_sptime_qz_apply``."""

    def __init__(self, space_fd: SpaceFD):
        super().__init__(space_fd)
        self._schur = None  # (S, T, Q, Z)

    schur_adv = property(lambda self: self._schur[0])
    schur_mass = property(lambda self: self._schur[1])
    schur_VSL = property(lambda self: self._schur[2])
    schur_VSR = property(lambda self: self._schur[3])

    def compute_time_schurdecomposition(self, time_quadrule):
        q = rewrite_quadrature([time_quadrule])[0]
        Mfull = sp.csr_array(q.weights[0] @ q.basis[0]).toarray()
        Wfull = sp.csr_array(q.weights[1] @ q.basis[1]).toarray()
        nt = Mfull.shape[0]
        idx = list(range(1, nt))
        self.nonzeros_by_dir[ParametricDirection.TAU] = nt
        self.indices_by_dir[(0, ParametricDirection.TAU)] = idx
        Wt = Wfull[np.ix_(idx, idx)]
        Mt = Mfull[np.ix_(idx, idx)]
        self._schur = sclin.qz(Wt, Mt, output="complex")
        self._nt = nt
        self._advection_time_corrector = [1.0] * self.nbDoFsPerNode
        self._sptm_free_nodes = self._propagate_nodes_in_time()
        self._dev.clear()

    def device_data(self, dtype: torch.dtype, node: int = 0):
        sp_fd = self._space_fd
        lam = sp_fd.space_eigenvalues[node]
        key = (dtype, node, id(lam))
        hit = self._dev.get(key)
        if hit is None:
            dev = require_cuda()
            S, T, Q, Z = self._schur

            def cplx(a):
                a = np.asarray(a, dtype=complex)
                return torch.from_numpy(np.ascontiguousarray(
                    np.stack([a.real, a.imag], axis=-1).reshape(-1))).to(dev)

            def part(a):
                return torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype)

            U = [torch.from_numpy(np.ascontiguousarray(u)).to(dev, dtype)
                 for u in sp_fd.eigenvec_by_dir_space[node]]
            lo, mm = sp_fd._boxes[node]
            n = [sp_fd.nonzeros_by_dir[d] for d in sp_fd.space_dirs] + [self._nt]
            lo = list(lo) + [1]
            mm = list(mm) + [self._nt - 1]
            M = math.prod(mm)
            work = [torch.empty(M, dtype=dtype, device=dev) for _ in range(3)]
            hit = dict(U=U, q_re=part(Q.real), q_im=part(Q.imag), z_re=part(Z.real),
                       z_im=part(Z.imag), S=cplx(S), T=cplx(T),
                       adv=float(self._advection_time_corrector[node]),
                       lam=torch.from_numpy(np.ascontiguousarray(lam)).to(dev, torch.float64),
                       n=n, lo=lo, m=mm, work=work)
            self._dev = {key: hit}
        return hit

    def apply_device(self, x: torch.Tensor, y: torch.Tensor, transpose: bool = False,
                     node: int = 0):
        h = self.device_data(x.dtype, node)
        sd = len(h["U"])
        arr = ctypes.c_int32 * (sd + 1)
        ptrs = (ctypes.c_void_p * sd)(*[u.data_ptr() for u in h["U"]])
        w = h["work"]
        _lib.check(_lib.LIB.iga_fd_sptime_qz_apply(
            iga_dtype(x.dtype), sd, arr(*h["n"]), arr(*h["lo"]), arr(*h["m"]), ptrs,
            h["q_re"].data_ptr(), h["q_im"].data_ptr(), h["z_re"].data_ptr(),
            h["z_im"].data_ptr(), h["S"].data_ptr(), h["T"].data_ptr(), h["adv"],
            h["lam"].data_ptr(), int(transpose), x.data_ptr(), y.data_ptr(), w[0].data_ptr(),
            w[1].data_ptr(), w[2].data_ptr(), stream_handle()))


class SingleFastDiagonalization:
    """Facade of the reference (fastdiag/preconditioner.py:15-197)."""

    def __init__(self, preconditioner_type: Literal["spatial", "spacetime"]):
        self._preconditioner_type = validate_entry(preconditioner_type, ["spatial", "spacetime"])
        self._space_fd: Optional[SpaceFD] = None
        self._sptime_fd = None

    @property
    def preconditioner_type(self):
        return self._preconditioner_type

    @property
    def space_preconditioner(self) -> SpaceFD:
        if self._space_fd is None:
            raise RuntimeError("Space preconditioner not defined.")
        return self._space_fd

    @property
    def sptm_preconditioner(self):
        if self._preconditioner_type == "spatial" or self._sptime_fd is None:
            raise RuntimeError("Space-time preconditioner not defined.")
        return self._sptime_fd

    def compute_space_eigendecomposition(self, space_quadrule_list, space_table_dirichlet):
        fd = SpaceFD()
        fd.compute_space_eigendecomposition(space_quadrule_list, space_table_dirichlet)
        self._space_fd = fd

    def compute_time_schurdecomposition(self, time_quadrule, use_arrowhead: bool = True):
        if self._preconditioner_type == "spatial" or self._space_fd is None:
            raise RuntimeError("Space-time preconditioner not defined.")
        fd = (SpaceTimeFD if use_arrowhead else SpaceTimeQZFD)(self._space_fd)
        fd.compute_time_schurdecomposition(time_quadrule)
        self._sptime_fd = fd

    def update_space_eigenvalues(self, scalar_coefs: Sequence[float]):
        fd = self.space_preconditioner
        fd._space_eigenvalues = fd.update_space_eigenvalues(scalar_coefs)
        fd._dev.clear()
        if self._sptime_fd is not None:
            self._sptime_fd._dev.clear()

    def add_scalar_space_time_correctors(self, mass_corrector=None, stiffness_corrector=None,
                                         advection_corrector=None):
        if self._space_fd is not None:
            self._space_fd.add_scalar_space_correctors(mass_corrector=mass_corrector,
                                                       stiffness_corrector=stiffness_corrector)
        if self._sptime_fd is not None:
            self._sptime_fd.add_scalar_time_correctors(advection_corrector=advection_corrector)

    def apply(self, array_in):
        if self._preconditioner_type == "spatial":
            return self.space_preconditioner.apply(array_in)
        return self.sptm_preconditioner.apply(array_in)

    def apply_transpose(self, array_in):
        if self._preconditioner_type == "spatial":
            return self.space_preconditioner.apply(array_in)  # symmetric
        return self.sptm_preconditioner.apply_transpose(array_in)


SingleFD = SingleFastDiagonalization


class MultiFastDiagonalization:
    """Block-diagonal FD over consecutive slices, one block per patch
    (src/igaops/fastdiag/multi_preconditioner.py:13-103).

    ``apply`` / ``apply_transpose`` run each patch's device apply on its
    slice (FP64 / FP32, the reference's arithmetic); ``apply_device_tc``
    applies every 3D patch at once with the BF16 tensor-core kernels -- six
    launches for all patches (``iga_fd_tc_batch_apply``)."""

    def __init__(self, list_preconditioner: List[SingleFastDiagonalization]):
        if list_preconditioner is None or len(list_preconditioner) < 1:
            raise RuntimeError("Empty list of preconditioners")
        if not all(isinstance(m, SingleFastDiagonalization) for m in list_preconditioner):
            raise RuntimeError("All elements should be preconditioners")
        self._list = list(list_preconditioner)
        self._preconditioner_type = self._list[0].preconditioner_type
        for fd in self._list:
            if fd.preconditioner_type != self._preconditioner_type:
                raise RuntimeError("Preconditioners should be of the same type")
        self._tc: Dict[torch.dtype, dict] = {}

    @property
    def preconditioner_type(self):
        return self._preconditioner_type

    def _sizes(self):
        out = []
        for p in self._list:
            fd = p.space_preconditioner
            tm = 1
            if self._preconditioner_type == "spacetime":
                tm = p.sptm_preconditioner.tm_nnz
            out.append(int(fd.nbDoFsPerNode * fd.sp_nnz * tm))
        return out

    def _apply_func(self, array_in, name):
        dtype = compute_dtype(array_in)
        x = to_device(array_in, dtype)
        sizes = self._sizes()
        if sum(sizes) != x.shape[0]:
            raise RuntimeError("array size does not match the preconditioner blocks")
        out = torch.empty_like(x)
        start = 0
        for p, n in zip(self._list, sizes):
            out[start:start + n] = getattr(p, name)(x[start:start + n])
            start += n
        return like_input(out, array_in)

    def apply(self, array_in):
        return self._apply_func(array_in, "apply")

    def apply_transpose(self, array_in):
        return self._apply_func(array_in, "apply_transpose")

    # ---- all patches at once on the tensor cores (3D, one DOF per node)
    def _tc_table(self, io_dtype: torch.dtype):
        hit = self._tc.get(io_dtype)
        if hit is not None:
            return hit
        if self._preconditioner_type != "spatial":
            raise NotImplementedError("the tensor-core FD apply covers spatial preconditioners")
        dev = require_cuda()
        P = len(self._list)
        i32 = ctypes.c_int32 * (3 * P)
        n, lo, m = i32(), i32(), i32()
        Bf = (ctypes.c_void_p * (3 * P))()
        Bb = (ctypes.c_void_p * (3 * P))()
        inv = (ctypes.c_void_p * P)()
        w0 = (ctypes.c_void_p * P)()
        w1 = (ctypes.c_void_p * P)()
        offs = (ctypes.c_int64 * P)()
        keep = []
        start = 0
        for i, (p, size) in enumerate(zip(self._list, self._sizes())):
            sp = p.space_preconditioner
            if sp.nbDoFsPerNode != 1:
                raise NotImplementedError("the tensor-core FD apply covers one DOF per node")
            fwd, bwd, invl, work, _ = sp.tc_data(0)
            keep.append((fwd, bwd, invl, work))
            lo_i, mm = sp._boxes[0]
            nn = [sp.nonzeros_by_dir[d] for d in sp.space_dirs]
            for d in range(3):
                n[3 * i + d], lo[3 * i + d], m[3 * i + d] = int(nn[d]), int(lo_i[d]), int(mm[d])
                Bf[3 * i + d] = fwd[d].data_ptr()
                Bb[3 * i + d] = bwd[d].data_ptr()
            inv[i] = invl.data_ptr()
            w0[i] = work[0].data_ptr()
            w1[i] = work[1].data_ptr()
            offs[i] = start
            start += size
        nbytes = ctypes.c_int64(0)
        _lib.check(_lib.LIB.iga_fd_tc_batch_table_bytes(P, ctypes.byref(nbytes)))
        table = torch.empty(int(nbytes.value) + 256, dtype=torch.uint8, device=dev)
        base = (table.data_ptr() + 255) // 256 * 256
        grid = (ctypes.c_int32 * 6)()
        smem = ctypes.c_int64(0)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.check(_lib.LIB.iga_fd_tc_batch_prepare(P, n, lo, m, Bf, Bb, inv, w0, w1, offs,
                                                    iga_dtype(io_dtype), status.data_ptr(), base,
                                                    grid, ctypes.byref(smem)))
        hit = dict(table=table, base=base, grid=grid, smem=int(smem.value), keep=keep,
                   status=status, ntot=start)
        self._tc[io_dtype] = hit
        return hit

    def apply_device_tc(self, x: torch.Tensor, y: torch.Tensor):
        """y = blockdiag(P_p^{-1}) x with BF16 tensor-core mode products for
        every patch in one set of launches; x, y device vectors (FP32/FP64)."""
        t = self._tc_table(x.dtype)
        if x.numel() != t["ntot"] or y.numel() != t["ntot"]:
            raise ValueError("vector size does not match the preconditioner blocks")
        _lib.check(_lib.LIB.iga_fd_tc_batch_apply(iga_dtype(x.dtype), len(self._list), t["base"],
                                                  t["grid"], t["smem"], x.data_ptr(),
                                                  y.data_ptr(), t["ntot"], None,
                                                  stream_handle()))

    def check_tc_status(self):
        for t in self._tc.values():
            st = int(t["status"].item())
            if st:
                t["status"].zero_()
                _lib.check(st)


MultiFD = MultiFastDiagonalization
