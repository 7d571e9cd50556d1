"""Sharding of independent k-points / cells across ranks: LPT balance, the
Monkhorst-Pack mesh, and the two host-side reductions under gloo with
world size 2 (CPU, no GPU)."""
import os
import socket
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "chemrust-scf_b200"))
import sharding  # noqa: E402


def test_partition_balances_uneven_members():
    rng = np.random.default_rng(0)
    costs = list(rng.uniform(1.0, 20.0, 96))
    for n in (1, 2, 4, 8):
        parts, loads = sharding.partition(costs, n)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        # LPT makespan bound: max load <= 4/3 OPT <= 4/3 max(mean, max cost) + max cost / 3
        lb = max(sum(costs) / n, max(costs))
        assert max(loads) <= 4.0 / 3.0 * lb + 1e-9
        np.testing.assert_allclose(sum(loads), sum(costs))


def test_monkhorst_pack_mesh():
    ks, w = sharding.monkhorst_pack(4)
    assert len(ks) == 64 and abs(w.sum() - 1.0) < 1e-15
    coords = sorted({k[0] for k in ks})
    np.testing.assert_allclose(coords, [-0.375, -0.125, 0.125, 0.375])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [5.0, 3.0, 8.0, 1.0, 4.0, 6.0]
        parts, _ = sharding.partition(costs, world)
        mine = parts[rank]
        # each member contributes w_k * rho_k = (k + 1) on a tiny grid
        rho = sum(np.full(8, i + 1.0) for i in mine) if mine else np.zeros(8)
        total = sharding.reduce_kpoint_density(rho, dist)
        res = sharding.gather_results({i: float(i * i) for i in mine}, dist)
        q.put((rank, total.tolist(), sorted(res.items())))
    finally:
        dist.destroy_process_group()


def test_gloo_world_size_2_reductions():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = float(sum(i + 1 for i in range(6)))
    for rank, total, res in out:
        np.testing.assert_allclose(total, expect)
        assert res == [(i, float(i * i)) for i in range(6)]
