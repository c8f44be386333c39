"""Multi-rank sharding of independent graphs (host logic, CPU).

The batched diffusion shards whole graphs across ranks with no collective in
the data path. These tests check the longest-processing-time assignment and
run it as two gloo ranks on CPU: each rank diffuses its own graphs (with the
oracle standing in for the device kernel) and rank 0 collects every graph's
result exactly once."""
import os
import socket

import numpy as np
import pytest

from scl import sharding


def test_lpt_assignment_covers_every_graph_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(100_000), 64))
    costs = sizes * 15 * 1.67 * 16 * 8  # nnz * F * T
    for world in (1, 2, 3, 4, 8):
        a = sharding.lpt_assign(costs, world)
        flat = sorted(i for part in a for i in part)
        assert flat == list(range(64))
        loads = sharding.rank_loads(costs, a)
        # LPT bound: max load <= mean + largest single cost
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6
    assert sharding.lpt_assign([], 2) == [[], []]
    with pytest.raises(ValueError):
        sharding.lpt_assign([1.0], 0)


def test_single_rank_gather_is_identity():
    assert sharding.gather_results({3: 1, 5: 2}, 0, 1) == {3: 1, 5: 2}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_path):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "scl-core_b200")]
    import datetime

    import scipy.sparse as sp
    import torch.distributed as dist

    from oracle import port as oracle_port
    from scl import sharding as sh

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(42)
        sizes = rng.integers(30, 200, 9)
        graphs = []
        for b, n in enumerate(sizes):
            A = sp.random(int(n), int(n), density=0.05, random_state=int(b), format="csr")
            A = (A + A.T).tocsr()
            A.sort_indices()
            P = oracle_port.transition(A.indptr, A.indices, A.data.astype(np.float32), False, True)
            graphs.append((A.indptr, A.indices, P))
        costs = [g[1].size * 4 * 3 for g in graphs]
        mine = sh.shard_for_rank(costs, rank, world)
        local = {}
        for i in mine:
            ip, ind, P = graphs[i]
            X0 = np.random.default_rng(100 + i).standard_normal((ip.size - 1, 4)).astype(np.float32)
            local[i] = oracle_port.diffuse_matrix(ip, ind, P, X0, 3)
        merged = sh.gather_results(local, rank, world)
        if rank == 0:
            assert sorted(merged) == list(range(len(graphs)))
            for i, (ip, ind, P) in enumerate(graphs):
                X0 = np.random.default_rng(100 + i).standard_normal((ip.size - 1, 4)).astype(np.float32)
                np.testing.assert_array_equal(merged[i], oracle_port.diffuse_matrix(ip, ind, P, X0, 3))
            with open(out_path, "w") as f:
                f.write("ok")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_collect(tmp_path):
    import torch.multiprocessing as mp

    out = tmp_path / "result.txt"
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True, start_method="spawn")
    assert out.read_text() == "ok"
