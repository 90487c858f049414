"""GPU parity of the fast-diagonalisation apply and the geometry precompute
(oracle / golden fixtures of the reference)."""
import numpy as np
import pytest
import torch

from oracle import fd as ofd
from oracle import mf as omf
from tests._golden import FixtureRule, load, rules as golden_rules
from tests._problems import rel_err, rules

pytestmark = pytest.mark.gpu


def test_fd_apply_matches_reference_golden(cuda):
    from igaops_b200.fastdiag import SingleFD

    d = load("fastdiag")
    q = rules(1, 3, 4, kind="gauss")[0]
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition([q] * 3, d["table"])
    fd.add_scalar_space_time_correctors(stiffness_corrector=[d["corr"]])
    fd.update_space_eigenvalues(d["scalar_coefs"])
    sp = fd.space_preconditioner
    assert np.array_equal(np.asarray(sp.space_free_nodes[0]), d["free"])
    assert rel_err(sp.space_eigenvalues[0], d["eig"]) < 1e-12
    assert rel_err(fd.apply(d["v"]), d["Pv"]) < 1e-12
    assert rel_err(fd.apply(d["V"]), d["PV"]) < 1e-12
    # float32 apply
    v32 = torch.from_numpy(d["v"]).float().cuda()
    assert rel_err(fd.apply(v32).double().cpu().numpy(), d["Pv"]) < 1e-5


@pytest.mark.parametrize("ndim,p,ne", [(1, 3, 6), (2, 2, 9), (2, 3, 64), (3, 3, 10), (3, 5, 7)])
@pytest.mark.parametrize("table_kind", ["all", "mixed", "none"])
def test_fd_apply_matches_oracle(cuda, ndim, p, ne, table_kind):
    from igaops_b200.fastdiag import SingleFD, rewrite_quadrature

    rl = rules(ndim, p, ne)
    table = np.ones((1, ndim, 2), dtype=bool)
    if table_kind == "mixed":
        table[0, 0, 0] = False
        table[0, -1, 1] = False
    elif table_kind == "none":
        table[:] = False
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, table)
    fd.update_space_eigenvalues([0.3, 1.0])
    ofdd = ofd.setup(rewrite_quadrature(rl), table, scalar_coefs=(0.3, 1.0))
    rng = np.random.default_rng(ne)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    for x in (rng.standard_normal(N), rng.standard_normal((N, 2))):
        ref = ofd.apply(ofdd, x)
        assert rel_err(fd.apply(x), ref) < 1e-11


def test_geometry_matches_reference_golden(cuda):
    from igaops_b200.geometry import GeometryOps, SingleSpline, precompute_coefficients

    d = load("geometry")
    q = FixtureRule(d, "rule")
    spl = SingleSpline(d["ctrlpts"], np.array([]), [q] * 3).evaluate_spline()
    assert rel_err(spl.jac, d["jac"]) < 1e-13
    assert rel_err(spl.det_jac, d["det_jac"]) < 1e-12
    assert rel_err(spl.inv_jac, d["inv_jac"]) < 1e-12
    assert rel_err(spl.qp_phy, d["qp_phy"]) < 1e-14
    co = precompute_coefficients([q] * 3, d["ctrlpts"])
    C = np.einsum("il...,jl...->ij...", d["inv_jac"], d["inv_jac"]) * d["det_jac"]
    assert rel_err(co["stiffness"].cpu().numpy(), C) < 1e-12
    assert rel_err(co["mass"].cpu().numpy(), d["det_jac"]) < 1e-12
    det, inv = GeometryOps.inverse_rectangular_matrix(d["jac"])
    assert rel_err(det, d["det_jac"]) < 1e-12 and rel_err(inv, d["inv_jac"]) < 1e-12


@pytest.mark.parametrize("p,ne", [(2, 7), (3, 16), (5, 9)])
def test_greville_unit_cube_is_the_identity_map(cuda, p, ne):
    """Known answer: the Greville control net of the unit cube maps the
    parametric cube onto itself, so det J = 1 and the stiffness coefficients
    det J J^+ J^+T = I at every quadrature point (to rounding)."""
    from igaops_b200 import precompute_coefficients, unit_cube_ctrlpts

    rl = rules(3, p, ne)
    co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=0.0))
    det = co["mass"].cpu().numpy()
    C = co["stiffness"].cpu().numpy()
    assert np.max(np.abs(det - 1.0)) < 1e-13
    assert np.max(np.abs(C - np.eye(3)[:, :, None])) < 1e-13


def test_geometry_rejects_degenerate(cuda):
    from igaops_b200.geometry import SingleSpline

    q = rules(1, 2, 3)[0]
    n = q.nbctrlpts ** 2
    flat = np.zeros((2, n))  # all control points at the origin: det J = 0
    with pytest.raises((ZeroDivisionError, ValueError)):
        SingleSpline(flat, np.array([]), [q, q]).evaluate_spline()


@pytest.mark.parametrize("name", ["2d_wq2", "3d_wq2", "3d_wq1", "3d_gauss", "st_01", "st_00", "st_10"])
@pytest.mark.parametrize("op", ["u_v", "gradu_gradv", "gradu_v", "u_gradv"])
def test_matvec_matches_reference_golden(cuda, name, op):
    """GPU operators fed the reference's own 1D factors reproduce the
    reference's outputs (FP64, 1e-12)."""
    from igaops_b200 import BsplineOperations

    d = load("matvec")
    ndim = 2 if name.startswith("2d") else 3
    rl = golden_rules(d, name, ndim)
    td = tuple(int(t) for t in d[f"{name}_td"])
    td = None if td[0] < 0 else td
    fn = getattr(BsplineOperations, f"compute_mf_scalar_{op}")
    c = d[f"{name}_{op}_c"]
    assert rel_err(fn(rl, c, d[f"{name}_x"], time_ders=td), d[f"{name}_{op}_y"]) < 1e-12
    if f"{name}_{op}_Y" in d:
        assert rel_err(fn(rl, c, d[f"{name}_X"], time_ders=td), d[f"{name}_{op}_Y"]) < 1e-12


def test_lmode_matches_reference_golden(cuda):
    from igaops_b200 import MatrixFree

    d = load("matvec")
    mats = [d[f"lm_M{k}"] for k in range(3)]
    assert rel_err(MatrixFree.apply(mats, d["lm_v"]), d["lm_y"]) < 1e-13
    assert rel_err(MatrixFree.apply(mats, d["lm_vt"], is_transpose=True), d["lm_yt"]) < 1e-13


@pytest.mark.parametrize("p,ne,table_kind", [(2, 3, "all"), (3, 13, "mixed"), (3, 96, "all"),
                                              (2, 40, "none")])
def test_fd_apply_tensor_cores_bf16(cuda, p, ne, table_kind):
    """BF16 tcgen05 mode products: relative error of the BF16 apply <= 1e-2
    (2-norm) against the FP64 oracle, before any refinement."""
    from igaops_b200.fastdiag import SingleFD, rewrite_quadrature

    rl = rules(3, p, ne)
    table = np.ones((1, 3, 2), dtype=bool)
    if table_kind == "mixed":
        table[0, 0, 0] = False
        table[0, 2, 1] = False
    elif table_kind == "none":
        table[:] = False
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, table)
    spfd = fd.space_preconditioner
    rng = np.random.default_rng(ne)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    ref = ofd.apply(ofd.setup(rewrite_quadrature(rl), table), x)
    for dt in (torch.float64, torch.float32):
        xd = torch.from_numpy(x).to("cuda", dt)
        yd = torch.empty_like(xd)
        spfd.apply_device_tc(xd, yd)
        spfd.check_tc_status()
        got = yd.double().cpu().numpy()
        err2 = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err2 < 1e-2, err2
        free = np.asarray(spfd.space_free_nodes[0])
        mask = np.ones(N, dtype=bool)
        mask[free] = False
        assert np.all(got[mask] == 0.0)


def _bf16(a):
    """Round to BF16 (nearest, ties to even), returned as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _bf16_apply(fd, x):
    """The tensor-core apply's arithmetic in numpy (all-Dirichlet box): the
    input, the eigenvector images and every intermediate rounded to BF16
    where the kernel rounds them, 1/Lambda in FP32, products accumulated in
    FP64 (the tensor cores accumulate in FP32), the last product in FP32."""
    n, m = fd.n, [U.shape[0] for U in fd.U]
    box = (slice(1, 1 + m[2]), slice(1, 1 + m[1]), slice(1, 1 + m[0]))
    T = _bf16(x.reshape(n[2], n[1], n[0])[box])
    U1, U2, U3 = (_bf16(U) for U in fd.U)
    T = _bf16(np.einsum("cba,ai->cbi", T, U1))
    T = _bf16(np.einsum("cbi,bj->cji", T, U2))
    T = np.einsum("cji,ck->kji", T, U3)
    inv = (1.0 / fd.eig).astype(np.float32).astype(np.float64).reshape(m[2], m[1], m[0])
    T = _bf16(T.astype(np.float32).astype(np.float64) * inv)
    T = _bf16(np.einsum("kji,ai->kja", T, U1))
    T = _bf16(np.einsum("kja,bj->kba", T, U2))
    T = np.einsum("kba,ck->cba", T, U3).astype(np.float32).astype(np.float64)
    y = np.zeros(n[2] * n[1] * n[0])
    y.reshape(n[2], n[1], n[0])[box] = T
    return y


@pytest.mark.parametrize("p,ne", [(2, [254, 3, 5]), (2, [4, 254, 2]), (3, [5, 6, 253]),
                                  (2, [1, 3, 5]), (3, [1, 1, 2]), (3, 12)])
def test_fd_apply_tensor_cores_extreme_extents(cuda, p, ne):
    """The largest free extent the tensor-core apply takes (254 + padding =
    256: K = N = 256 in the products of that direction, the column split
    into 128 + 128) in each direction, and single free indices (m = 1,
    K = N = 16): the apply equals a numpy emulation of its BF16 arithmetic
    within 3e-3 (2-norm; the emulation accumulates in FP64, the tensor
    cores in FP32, so an intermediate may round to the neighbouring BF16
    value), and the FP64 oracle within 2e-2 (BF16; a 1 x 3 x 5 box has
    too few terms to average the roundings out: 1.2 %)."""
    from igaops_b200.fastdiag import SingleFD, rewrite_quadrature

    rl = rules(3, p, ne)
    table = np.ones((1, 3, 2), dtype=bool)
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, table)
    spfd = fd.space_preconditioner
    assert max(spfd._boxes[0][1]) <= 256
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = np.random.default_rng(N).standard_normal(N)
    ofdd = ofd.setup(rewrite_quadrature(rl), table)
    ref = ofd.apply(ofdd, x)
    emu = _bf16_apply(ofdd, x)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    spfd.apply_device_tc(xd, yd)
    spfd.check_tc_status()
    got = yd.cpu().numpy()
    assert np.linalg.norm(got - emu) / np.linalg.norm(emu) < 3e-3
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-2


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("offset", [0, 1, 2, 3])
def test_fd_apply_tc_reads_only_the_free_box(cuda, dt, offset):
    """The tensor-core apply gathers its input in aligned 16-byte blocks,
    which also hold entries outside the free box: with NaN in every entry
    outside the box and the vector starting at any element offset (so at
    every alignment), the result equals, bit for bit, the apply of a clean,
    aligned copy; the box rows have odd lengths so that blocks straddle
    row ends."""
    from igaops_b200.fastdiag import SingleFD

    rl = rules(3, 3, [10, 7, 12])
    table = np.ones((1, 3, 2), dtype=bool)
    table[0, 1, 1] = False
    fd = SingleFD("spatial")
    fd.compute_space_eigendecomposition(rl, table)
    spfd = fd.space_preconditioner
    N = int(np.prod([q.nbctrlpts for q in rl]))
    free = spfd.free_nodes(0)
    rng = np.random.default_rng(7)
    clean = np.zeros(N)
    clean[free] = rng.standard_normal(free.size)
    dirty = np.full(N, np.nan)
    dirty[free] = clean[free]
    xa = torch.from_numpy(clean).to("cuda", dt)
    ya = torch.empty_like(xa)
    spfd.apply_device_tc(xa, ya)
    buf = torch.full((N + 8,), float("nan"), dtype=dt, device="cuda")
    buf[offset:offset + N] = torch.from_numpy(dirty).to("cuda", dt)
    xv = buf[offset:offset + N]
    yv = torch.empty_like(xa)
    spfd.apply_device_tc(xv, yv)
    spfd.check_tc_status()
    assert torch.isfinite(yv).all()
    assert torch.equal(yv, ya)


def test_multifd_matches_per_patch_oracle(cuda):
    """MultiFD: block-diagonal apply over consecutive patch slices equals the
    oracle applied patch by patch (FP64 1e-11); the batched tensor-core apply
    of all patches equals each patch's own tensor-core apply."""
    from igaops_b200.fastdiag import MultiFD, SingleFD, rewrite_quadrature

    specs = [(2, 4), (3, 5), (3, 3)]
    fds, oracles, sizes = [], [], []
    for k, (p, ne) in enumerate(specs):
        rl = rules(3, p, ne + k)
        table = np.ones((1, 3, 2), dtype=bool)
        fd = SingleFD("spatial")
        fd.compute_space_eigendecomposition(rl, table)
        fds.append(fd)
        oracles.append(ofd.setup(rewrite_quadrature(rl), table))
        sizes.append(int(np.prod([q.nbctrlpts for q in rl])))
    mfd = MultiFD(fds)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(sum(sizes))
    got = mfd.apply(x)
    start = 0
    for o, n in zip(oracles, sizes):
        assert rel_err(got[start:start + n], ofd.apply(o, x[start:start + n])) < 1e-11
        start += n
    xd = torch.from_numpy(x).float().cuda()
    yd = torch.empty_like(xd)
    mfd.apply_device_tc(xd, yd)
    mfd.check_tc_status()
    start = 0
    for fd, n in zip(fds, sizes):
        ys = torch.empty(n, dtype=torch.float32, device="cuda")
        fd.space_preconditioner.apply_device_tc(xd[start:start + n].contiguous(), ys)
        assert torch.equal(ys, yd[start:start + n])
        start += n
    with pytest.raises(RuntimeError):
        MultiFD([])


def test_fd_tc_inverse_eigenvalues_on_device_equal_host(cuda):
    """The tensor-core data forms 1/Lambda on the device from the 1D
    eigenvalues (no host Lambda array): bit for bit the host array's FP32
    conversion, with and without a stiffness corrector, and the applies
    agree bit for bit; a second set-up of the same spline reuses the
    cached BF16 eigenvector images."""
    from igaops_b200.fastdiag import SingleFD

    rl = rules(3, 3, [9, 7, 11])
    table = np.ones((1, 3, 2), dtype=bool)
    rng = np.random.default_rng(3)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = torch.from_numpy(rng.standard_normal(N)).cuda()
    for corr in (None, [np.array([1.0, 0.7, 1.3])]):
        host = SingleFD("spatial")
        host.compute_space_eigendecomposition(rl, table)
        dev = SingleFD("spatial")
        dev.compute_space_eigendecomposition(rl, table)
        if corr is not None:
            host.space_preconditioner.add_scalar_space_correctors(stiffness_corrector=corr)
            dev.space_preconditioner.add_scalar_space_correctors(stiffness_corrector=corr)
        host.update_space_eigenvalues([0.0, 1.0])  # host Lambda formed first
        hs, ds = host.space_preconditioner, dev.space_preconditioner
        assert ds._space_eigenvalues is None
        inv_h = hs.tc_data()[2]
        inv_d = ds.tc_data()[2]
        assert ds._space_eigenvalues is None  # never formed on the host
        assert torch.equal(inv_h, inv_d)
        for a, b in zip(hs.tc_data()[0] + hs.tc_data()[1], ds.tc_data()[0] + ds.tc_data()[1]):
            assert a.data_ptr() == b.data_ptr()  # the cached images
        yh, yd = torch.empty_like(x), torch.empty_like(x)
        hs.apply_device_tc(x, yh)
        ds.apply_device_tc(x, yd)
        assert torch.equal(yh, yd)
