"""Multi-rank replica path on CPU: two gloo ranks, each owning a disjoint
share of independent patches, no data-path collective, device-time maximum
and whole-job throughput as `bench.py --gpus N` computes them.  The per-patch
work here is the oracle's matrix-free product (the GPU path runs the fused
kernels instead); what is under test is the sharding and the reductions."""
import json
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from igaops_b200.replicas import job_throughput, max_over_ranks, rank_env, shard_units

N_PATCHES = 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _patch_product(i):
    from oracle import mf
    from tests import _problems as P

    rng = np.random.default_rng(100 + i)
    rl = P.rules(2, 2, 4 + i)
    c = P.coefficients("gradu_gradv", rl, rng)
    n = int(np.prod([q.nbctrlpts for q in rl]))
    x = rng.standard_normal(n)
    return mf.mf_gradu_gradv([q for q in rl], c, x)


def _rank_main(rank, world, port, out_path):
    import os

    import torch.distributed as dist

    from igaops_b200.replicas import finish, init_group

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    info = rank_env()
    assert (info.world, info.rank) == (world, rank)
    g = init_group(info, "gloo", timeout_s=60.0)
    assert g is dist and dist.get_world_size() == world
    mine = shard_units(N_PATCHES, world, rank)
    results = {i: _patch_product(i).tolist() for i in mine}
    # per-rank "device times": rank r reports 2.0 * (r + 1) ms and 7 - r ms
    ms = max_over_ranks([2.0 * (rank + 1), 7.0 - rank], g)
    gathered = [None] * world
    dist.all_gather_object(gathered, {"rank": rank, "patches": mine, "results": results,
                                      "ms": ms})
    if rank == 0:
        with open(out_path, "w") as f:
            json.dump(gathered, f)
    finish(g)


def test_shard_units_partitions():
    for n in range(0, 13):
        for world in range(1, 6):
            parts = [shard_units(n, world, r) for r in range(world)]
            flat = [i for p in parts for i in p]
            assert flat == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_units(3, 2, 2)


def test_single_rank_identity(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    info = rank_env()
    assert (info.world, info.rank, info.local) == (1, 0, 0)
    assert max_over_ranks([1.5, 2.5], None) == [1.5, 2.5]
    assert job_throughput(2_000_000, 1, 2.0) == pytest.approx(1.0)
    assert job_throughput(2_000_000, 4, 2.0) == pytest.approx(4.0)
    with pytest.raises(ValueError):
        job_throughput(1, 1, 0.0)
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "2")
    with pytest.raises(ValueError):
        rank_env()


def test_two_gloo_ranks(tmp_path):
    world = 2
    out = tmp_path / "gathered.json"
    mp.start_processes(_rank_main, args=(world, _free_port(), str(out)), nprocs=world,
                       join=True, start_method="spawn")
    gathered = json.loads(out.read_text())
    assert [g["rank"] for g in gathered] == [0, 1]
    # disjoint shares covering every patch once
    owned = [i for g in gathered for i in g["patches"]]
    assert sorted(owned) == list(range(N_PATCHES))
    assert len(set(owned)) == N_PATCHES
    # each rank's replica results equal a single-process run of the same patch
    for g in gathered:
        for i, r in g["results"].items():
            np.testing.assert_array_equal(np.asarray(r), _patch_product(int(i)))
    # every rank sees the element-wise maximum
    for g in gathered:
        assert g["ms"] == [4.0, 7.0]
    # weak scaling: whole-job throughput counts every rank's units
    assert job_throughput(1e9, world, 4.0) == pytest.approx(2 * 1e9 / 4e-3 / 1e9)
