"""The multi-rank logic of bench.py on CPU: two gloo ranks (torch.distributed), no GPU.

Each rank steps its own groom (weak scaling, no data-path collective); the job time is the slowest
rank's, and the reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 10.0 * (rank + 1)  # rank 1 is the slow one
        m = bench.max_over_ranks(local_ms, world, device="cpu")
        out[rank] = (m, bench.job_throughput(world, 640000, 20, 100, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_weak_scaling_throughput():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    assert out[0][0] == 20.0 and out[1][0] == 20.0
    # 2 ranks x 640,000 vertices x 20 iterations x 100 steps in 20 ms
    assert out[0][1] == pytest.approx(2 * 640000 * 20 * 100 / 0.020)


def _plan_main(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, r, local = bench.dist_setup()
        g = bench.rank_groom(r)
        mine = torch.tensor([float(local), float(g.positions[:64].sum()), float(g.num_vertices)], dtype=torch.float64)
        every = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(every, mine)
        out[rank] = [e.tolist() for e in every]
    finally:
        dist.destroy_process_group()


def test_each_rank_binds_its_own_device_and_groom():
    """bench.py's per-rank plan: rank r binds GPU LOCAL_RANK = r and steps a groom of its own (same
    size, different strands), so N ranks run N independent replicas."""
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_plan_main, args=(world, port, out), nprocs=world, join=True)
    plans = out[0]
    assert plans == out[1]
    assert [p[0] for p in plans] == [0.0, 1.0]  # distinct devices
    assert plans[0][1] != plans[1][1]  # distinct grooms
    assert plans[0][2] == plans[1][2] == 640000.0  # of the same size (weak scaling)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench

    class Args:
        steps, warmup, gpus = 3, 3, 2

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    bench.run_reference(Args())
    assert capsys.readouterr().out == ""
