"""The CPU legs of bench.py (cpu_baseline and --impl reference) run the
oracle on the reference's own 1D factors and never load the product package;
the slab split they use gives the oracle's whole-patch product."""
import subprocess
import sys
from pathlib import Path

import numpy as np

from oracle import mf as omf
from oracle.rules import bench_rule, slab_rule
from tests._golden import FixtureRule, load

ROOT = Path(__file__).resolve().parent.parent


def _rule64():
    d = load("quadrature")
    names = [str(n) for n in d["names"]]
    return FixtureRule(d, f"r{names.index('wq2:3:64:endpoint')}")


def test_slab_split_sums_to_whole_product():
    q = _rule64()
    nq, n = q.nbquadpts, q.nbctrlpts
    rng = np.random.default_rng(0)
    C = rng.standard_normal((3, 3, nq ** 3))
    C = 0.5 * (C + C.transpose(1, 0, 2))
    m = 1.0 + rng.random(nq ** 3)
    x = rng.standard_normal(n ** 3)
    ys = omf.mf_gradu_gradv([q, q, q], C, x)
    ym = omf.mf_u_v([q, q, q], m, x)
    acc_s, acc_m = np.zeros_like(ys), np.zeros_like(ym)
    cuts = np.linspace(0, nq, 6).astype(int)
    for a, b in zip(cuts[:-1], cuts[1:]):
        rl = [q, q, slab_rule(q, a, b)]
        sl = slice(a * nq * nq, b * nq * nq)
        acc_s += omf.mf_gradu_gradv(rl, C[:, :, sl], x)
        acc_m += omf.mf_u_v(rl, m[sl], x)
    assert np.max(np.abs(acc_s - ys)) / np.max(np.abs(ys)) < 1e-13
    assert np.max(np.abs(acc_m - ym)) / np.max(np.abs(ym)) < 1e-13


def test_bench_rule_fixture_is_the_benchmark_rule():
    q = bench_rule()
    assert q.degree == 3 and q.nbctrlpts == 131 and q.nbquadpts == 389
    assert len(q.basis) == 2 and len(q.weights) == 4


def test_cpu_legs_do_not_load_the_product_package():
    code = (
        "import sys, bench\n"
        "rl, C, m, x, (p0, p1), n = bench._cpu_slab(389, 200)\n"
        "ys, ym = bench._cpu_pair(rl, C, m, x)\n"
        "import numpy as np\n"
        "nz = np.flatnonzero(ys)\n"
        "assert nz.min() >= p0 * n * n and nz.max() < p1 * n * n\n"
        "bad = [k for k in sys.modules if k.startswith('igaops_b200')]\n"
        "assert not bad, bad\n"
        "print('ok')\n"
    )
    res = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0, res.stderr
    assert "ok" in res.stdout


def test_bench_refuses_bad_segment_counts():
    """--nseg takes 'auto' or two counts >= 1 (stiffness, mass); anything
    else is an argument error before any device work."""
    for bad in ("2", "0,1", "a,b", "1,2,3"):
        r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--nseg", bad],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 2, (bad, r.stderr[-300:])
        assert "--nseg" in r.stderr
