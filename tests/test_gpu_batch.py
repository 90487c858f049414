"""Many patches in one launch: the multi-patch matvec and tensor-core FD
apply against the single-patch kernels, the segmented Krylov kernels against
numpy, and the batched mixed-precision FGMRES against the oracle's FP64
operator (true relative residual < 1e-10 per patch) and the plain FP64 path.
"""
import numpy as np
import pytest
import torch

from oracle import mf as omf
from tests._problems import rel_err, rules

pytestmark = pytest.mark.gpu

SPECS = [(2, 6, 0.0), (3, 7, 0.05), (4, 5, 0.1), (3, 9, 0.08), (2, 11, 0.02)]


def _patches(specs=SPECS):
    from igaops_b200 import precompute_coefficients, unit_cube_ctrlpts

    out = []
    for p, ne, amp in specs:
        rl = rules(3, p, ne)
        co = precompute_coefficients(rl, unit_cube_ctrlpts(rl, amplitude=amp))
        out.append((rl, co["stiffness"], np.ones((1, 3, 2), dtype=bool)))
    return out


@pytest.fixture(scope="module")
def batch(cuda):
    from igaops_b200.batch import PatchBatch

    pats = _patches()
    return pats, PatchBatch(pats)


def _rhs(B, seed=0):
    rng = np.random.default_rng(seed)
    parts = []
    for p in B.patches:
        b = np.zeros(p.N)
        b[p.free] = rng.uniform(-1.0, 1.0, p.free.size)
        parts.append(b)
    return parts


def test_batch_matvec_equals_single(batch):
    _, B = batch
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.standard_normal(B.ntot)).cuda()
    for dt, tol in ((torch.float64, 1e-13), (torch.float32, 1e-6)):
        xd = x.to(dt)
        y = torch.empty_like(xd)
        B.matvec(xd, y)
        parts = B.split(y)
        xs = B.split(xd)
        for p, xp, yp in zip(B.patches, xs, parts):
            op = p.K64 if dt == torch.float64 else p.K32
            ref = op.apply(torch.from_numpy(np.ascontiguousarray(xp)).cuda()).cpu().numpy()
            ref[p.dirichlet] = 0.0
            assert rel_err(yp, ref) < tol
    B.check_status()


def test_batch_fd_tc_equals_single(batch):
    _, B = batch
    rng = np.random.default_rng(4)
    x = torch.from_numpy(rng.standard_normal(B.ntot)).float().cuda()
    y = torch.empty_like(x)
    B.precond(x, y)
    for p, xp, yp in zip(B.patches, B.split(x), B.split(y)):
        xs = torch.from_numpy(np.ascontiguousarray(xp)).cuda()
        ys = torch.empty_like(xs)
        p.fd.space_preconditioner.apply_device_tc(xs, ys)
        assert np.array_equal(ys.cpu().numpy(), yp)
    B.check_status()


def test_segmented_kernels_match_numpy(cuda):
    from igaops_b200.batch import _Seg

    sizes = [5000, 1, 4097, 2048, 9000]
    seg = _Seg(sizes, torch.device("cuda"))
    rng = np.random.default_rng(5)
    n = sum(sizes)
    m = 5
    A = rng.standard_normal((m, n))
    x = rng.standard_normal(n)
    o = seg.offs_host
    Ad = torch.from_numpy(A).cuda()
    xd = torch.from_numpy(x).cuda()
    out = torch.zeros((len(sizes), m), dtype=torch.float64, device="cuda")
    seg.gram(Ad, m, xd, out.data_ptr(), m)
    ref = np.stack([A[:, o[p]:o[p + 1]] @ x[o[p]:o[p + 1]] for p in range(len(sizes))])
    assert rel_err(out.cpu().numpy(), ref) < 1e-13
    coef = rng.standard_normal((len(sizes), m))
    y0 = rng.standard_normal(n)
    yd = torch.from_numpy(y0.copy()).cuda()
    cd = torch.from_numpy(coef).cuda()
    seg.combine(Ad, m, cd.data_ptr(), m, 2.0, -0.5, yd)
    refy = y0 * -0.5
    for p in range(len(sizes)):
        refy[o[p]:o[p + 1]] += 2.0 * coef[p] @ A[:, o[p]:o[p + 1]]
    assert rel_err(yd.cpu().numpy(), refy) < 1e-13
    s = np.abs(rng.standard_normal(len(sizes))) + 0.5
    sd = torch.from_numpy(s).cuda()
    zd = torch.from_numpy(x.copy()).cuda()
    seg.scale(zd, sd.data_ptr(), 1, 2)
    refz = x.copy()
    for p in range(len(sizes)):
        refz[o[p]:o[p + 1]] /= np.sqrt(s[p])
    assert rel_err(zd.cpu().numpy(), refz) < 1e-14


@pytest.mark.parametrize("inner,graphs", [(0, True), (2, True), (0, False)])
def test_batched_fgmres_reaches_tolerance(batch, inner, graphs):
    from igaops_b200.batch import BatchedFGMRES

    pats, B = batch
    parts = _rhs(B)
    solver = BatchedFGMRES(B, tolerance=1e-10, restart=12, inner_iters=inner, use_graphs=graphs)
    res = solver.solve(B.join(parts))
    B.check_status()
    assert res.success.all(), res.true_residual
    sols = B.split(res.solution)
    for (rl, C, _), p, x, b in zip(pats, B.patches, sols, parts):
        r = b - omf.mf_gradu_gradv(rl, C.cpu().numpy(), x)
        assert np.linalg.norm(r[p.free]) / np.linalg.norm(b[p.free]) < 1e-10
        assert np.all(x[p.dirichlet] == 0.0)


def test_batched_equals_sequential_fp64_and_alone(batch):
    """Each patch's solution is the same solved in the batch, solved alone
    in a batch of one, and solved by the plain FP64 path (within the
    tolerance the 1e-10 residual allows)."""
    from igaops_b200.batch import BatchedFGMRES, PatchBatch

    pats, B = batch
    parts = _rhs(B, seed=1)
    res = BatchedFGMRES(B, tolerance=1e-10).solve(B.join(parts))
    mix = B.split(res.solution)
    seq, _ = B.solve_fp64_sequential(B.join(parts))
    for i in (0, 3):
        alone_b = PatchBatch([pats[i]])
        r1 = BatchedFGMRES(alone_b, tolerance=1e-10).solve(alone_b.join([parts[i]]))
        alone = alone_b.split(r1.solution)[0]
        assert np.linalg.norm(alone - mix[i]) / np.linalg.norm(alone) < 1e-8
        s = seq[i].cpu().numpy() if isinstance(seq[i], torch.Tensor) else seq[i]
        assert np.linalg.norm(s - mix[i]) / np.linalg.norm(s) < 1e-8


def test_batched_fp64_arm_reaches_tolerance_and_matches_mixed(batch):
    """The FP64 arm of the batched engine (FP64 FD apply per patch, no
    low-precision work) converges to the same solutions."""
    from igaops_b200.batch import BatchedFGMRES

    pats, B = batch
    parts = _rhs(B, seed=2)
    r64 = BatchedFGMRES(B, tolerance=1e-10, precision="fp64").solve(B.join(parts))
    rmx = BatchedFGMRES(B, tolerance=1e-10).solve(B.join(parts))
    B.check_status()
    assert r64.success.all(), r64.true_residual
    assert rmx.success.all(), rmx.true_residual
    for (rl, C, _), p, x, b in zip(pats, B.patches, B.split(r64.solution), parts):
        r = b - omf.mf_gradu_gradv(rl, C.cpu().numpy(), x)
        assert np.linalg.norm(r[p.free]) / np.linalg.norm(b[p.free]) < 1e-10
    for a, b in zip(B.split(r64.solution), B.split(rmx.solution)):
        assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-8


def test_batched_matvec_skip_flags_follow_the_patch_not_the_group(batch):
    """Patches of different band widths run in separate launches; a
    patch's skip flag must reach that patch (regression: each launch read
    the flags of its group-local indices, so a converged patch 0 silenced
    the first patch of every other group)."""
    pats, B = batch
    rng = np.random.default_rng(9)
    x = torch.from_numpy(rng.standard_normal(B.ntot)).cuda()
    y_all = torch.empty_like(x)
    B.matvec(x, y_all)
    for k in range(B.np):
        skip = torch.full((B.np,), -1, dtype=torch.int32, device="cuda")
        skip[k] = 0
        y = torch.empty_like(x)
        B.matvec(x, y, skip)
        o = B.seg.offs_host
        for p in range(B.np):
            seg = y[o[p]:o[p + 1]]
            if p == k:
                assert bool((seg == 0).all())
            else:
                ref = y_all[o[p]:o[p + 1]]
                # atomics: summation order may differ between launches
                assert float((seg - ref).abs().max() / ref.abs().max()) < 1e-13, (k, p)


@pytest.mark.parametrize("restart", [12, 3])
def test_batched_arnoldi_stopping_rule(batch, restart):
    """residual="arnoldi": a cycle in which every patch met the tolerance by
    its Arnoldi estimate ends without b - A x; patches converge at
    different steps, and each reported estimate (held at its patch's
    convergence step) matches the oracle's residual of that patch's
    solution. With restart 3 the early cycles restart from the true
    residual."""
    from igaops_b200.batch import BatchedFGMRES

    pats, B = batch
    parts = _rhs(B, seed=3)
    res = BatchedFGMRES(B, tolerance=1e-10, restart=restart, max_cycles=12,
                        residual="arnoldi").solve(B.join(parts))
    B.check_status()
    assert res.residual_kind == "arnoldi"
    assert res.success.all(), res.true_residual
    for (rl, C, _), p, x, b, est in zip(pats, B.patches, B.split(res.solution), parts,
                                        res.true_residual):
        r = b - omf.mf_gradu_gradv(rl, C.cpu().numpy(), x)
        orc = np.linalg.norm(r[p.free]) / np.linalg.norm(b[p.free])
        assert orc < 1e-10
        assert abs(orc - est) < 1e-12
    if restart == 3:
        assert res.cycles > 1


def test_batched_first_graph_cycle_equals_eager(batch):
    """A fresh engine's first cycle with CUDA graphs (each step run eagerly
    once, then captured) takes the same steps, residual estimates and
    solutions as the eager engine: no step runs twice."""
    from igaops_b200.batch import BatchedFGMRES

    pats, B = batch
    parts = _rhs(B, seed=4)
    runs = [BatchedFGMRES(B, tolerance=1e-10, restart=12, residual="arnoldi",
                          use_graphs=g).solve(B.join(parts)) for g in (True, False)]
    B.check_status()
    rg, re_ = runs
    assert rg.cycles == re_.cycles
    assert rg.outer_steps == re_.outer_steps
    np.testing.assert_allclose(rg.true_residual, re_.true_residual, rtol=1e-6, atol=1e-14)
    for a, b in zip(B.split(rg.solution), B.split(re_.solution)):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
