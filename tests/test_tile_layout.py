"""CPU checks of the tensor-core tile plan (igaops_b200/tile3d.py): the tile
geometry, the fragment tables (tensor-core operand order, the even / odd
point k-steps of direction 3) and the windows reproduce the oracle's
operators when the tile arithmetic is replayed in numpy (dense 8 x 8 blocks
decoded from the tables)."""
import numpy as np
import pytest

from igaops_b200 import _lib, tile3d
from oracle import mf as omf
from tests._problems import coefficients, rel_err, rules


@pytest.mark.parametrize("p,ne", [(3, 6), (2, 7), (4, 5), (3, [5, 9, 7]), (2, [17, 3, 9])])
@pytest.mark.parametrize("op", ["gradu_gradv", "u_v"])
def test_tile_replay_matches_oracle(p, ne, op):
    rl = rules(3, p, ne)
    rng = np.random.default_rng(7)
    N = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(N)
    c = coefficients(op, rl, rng)
    code = _lib.IGA_OP_STIFF if op == "gradu_gradv" else _lib.IGA_OP_MASS
    y = tile3d.emulate(rl, code, c, x)
    assert rel_err(y, omf.OPS[op](rl, c, x)) < 1e-13


@pytest.mark.parametrize("p", [2, 3, 4])
@pytest.mark.parametrize("ne", [1, 4, 16, 17, 96, 128])
def test_tile_windows_fit(p, ne):
    q = rules(1, p, ne)[0]
    for k in range(3):
        d = tile3d.DirTiles(q, k)
        assert d.ok
        g = d.geom
        assert np.all(g[:, tile3d.G_DX] <= tile3d.XP[k])
        assert np.all(g[:, tile3d.G_DY] <= tile3d.XP[k])
        assert np.all(g[:, tile3d.G_TW0:tile3d.G_TW1 + 1] + 8 <= tile3d.XP[k])
        assert np.all(g[:, tile3d.G_SW0:tile3d.G_SW1 + 1] + 8 <= tile3d.XP[k])
        assert int(g[:, tile3d.G_Q].sum()) == q.nbquadpts


def test_degree5_keeps_the_pencil_kernel():
    q = rules(1, 5, 16)[0]
    assert not tile3d.DirTiles(q, 0).ok


def test_shared_memory_fits():
    q = rules(1, 3, 128)[0]
    nt = [tile3d.DirTiles(q, k).ntile for k in range(3)]
    assert tile3d.smem_bytes(_lib.IGA_OP_STIFF, nt) <= tile3d.SMEM_LIMIT
    assert tile3d.smem_bytes(_lib.IGA_OP_MASS, nt) <= tile3d.SMEM_LIMIT
