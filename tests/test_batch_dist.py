"""Host side of the multi-GPU batch path, run as world_size-2 gloo ranks on the CPU.

The solver is replaced by a deterministic stand-in: what is tested here is the sharding
of realisations across ranks and the gather of the results to rank 0."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from specklesim_b200 import batch


def test_assign_is_a_partition_and_balanced():
    rng = np.random.default_rng(0)
    sizes = rng.integers(13000, 80000, 64) * 3 // 2  # C4-like uneven edge counts
    for world in (1, 2, 4, 8):
        plan = batch.assign_realisations(sizes, world)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(len(sizes)))
        assert batch.balance(plan, sizes) < 1.05
    # deterministic
    assert batch.assign_realisations(sizes, 4) == batch.assign_realisations(sizes, 4)


def test_assign_more_ranks_than_work():
    plan = batch.assign_realisations([5, 3], 4)
    assert sorted(i for p in plan for i in p) == [0, 1]
    assert sum(1 for p in plan if not p) == 2


def _fake_solve(r):
    # stands in for a GPU solve: intensities depend only on the realisation
    rng = np.random.default_rng(r["seed"])
    return {"seed": r["seed"], "intensity": rng.random(8), "iterations": int(r["n_edges"]) % 97}


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reals = [{"seed": 100 + i, "n_edges": 20000 + 997 * i} for i in range(9)]
        res = batch.run_batch(reals, _fake_solve, world=world, rank=rank)
        if rank == 0:
            np.save(out_path, np.stack([r["intensity"] for r in res]))
            assert [r["seed"] for r in res] == [100 + i for i in range(9)]
        else:
            assert res is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_run_batch_gloo_two_ranks(tmp_path):
    out = str(tmp_path / "gathered.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    want = np.stack([_fake_solve({"seed": 100 + i, "n_edges": 0})["intensity"] for i in range(9)])
    assert np.array_equal(got, want)
