"""bench.py --gpus N runs N independent replicas (the step has no data-path
collective): each rank steps its own lattice, the job's time is the max over
ranks and the job's MLUPS counts every rank's cells.  Checked with two gloo
ranks on the CPU (127.0.0.1 rendezvous)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    ms = [12.0, 15.5][rank]                      # rank 1 is the slow replica
    m = bench.max_over_ranks_of(ms, world, "cpu")
    dist.barrier()
    out.put((rank, m, bench.job_mlups(1_000_000, 100, world, m)))
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.5, 15.5]
    assert res[0][2] == pytest.approx(2 * 1_000_000 * 100 / 0.0155 / 1e6)


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.max_over_ranks_of(3.0, 1, "cpu") == 3.0
    assert bench.job_mlups(33_554_432, 1000, 1, 1430.0) == pytest.approx(23464.6, rel=1e-4)


def test_samples_are_split_by_cell_count():
    """Config 4's independent samples shard across GPUs by cell count: every
    sample in exactly one group, the groups' totals within the largest sample
    of each other, deterministic."""
    from fluidmaxxer_b200 import lattice, problems

    cells = [p.n_cells for p in problems.batch_samples(count=64)]
    for parts in (1, 2, 3, 8):
        groups = lattice.partition_samples(cells, parts)
        assert sorted(i for g in groups for i in g) == list(range(len(cells)))
        loads = [sum(cells[i] for i in g) for g in groups]
        assert max(loads) - min(loads) <= max(cells)
        assert groups == lattice.partition_samples(cells, parts)
