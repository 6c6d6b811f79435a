"""The N>1 path on the CPU: two gloo ranks split the shots, each propagates its own shots with the
C restatement (standing in for its GPU), the partial images are reduced onto rank 0 and must
equal a single-process run; per-rank timings reduce to the maximum."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from wavefd_b200.shots import partition_by_cost, partition_shots


def test_partition_shots_covers_all_once():
    for n in (1, 5, 64):
        for w in (1, 2, 3, 8):
            got = sorted(sum((partition_shots(n, w, r) for r in range(w)), []))
            assert got == list(range(n))


def test_partition_by_cost_balances():
    costs = [5, 1, 1, 1, 1, 1, 4, 3]
    parts = [partition_by_cost(costs, 2, r) for r in range(2)]
    assert sorted(parts[0] + parts[1]) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert abs(loads[0] - loads[1]) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _shot_image(seed, shape):
    """One 'shot': a few 3D Iso steps on the restatement, then an imaging accumulation."""
    from oracle.oracle import Oracle
    from tests.harness import OracleRunner, make_model
    o = Oracle()
    run = OracleRunner(o, "Prop3DAcoIsoDenQ_DEO2_FDTD", shape, fs=True)
    run.load(make_model(3, "iso", shape, seed=seed))
    for _ in range(3):
        run.step()
    img = np.zeros_like(run.arr("V"))
    o.image_iso(run.g, 0, run.arr("V"), run.arr("B"), None, run.arr("PSpace"), run.arr("POld"), img, None)
    return img


def _rank_main(rank, world, port, nshots, shape, out):
    import torch
    import torch.distributed as dist

    from wavefd_b200.shots import partition_shots, reduce_image, reduce_max
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    img = np.zeros((shape[2], shape[1], shape[0]), np.float32)
    for s in partition_shots(nshots, world, rank):
        img += _shot_image(100 + s, shape)
    t = torch.from_numpy(img)
    reduce_image(t, dst=0)
    tmax = reduce_max(1.0 + rank)
    if rank == 0:
        np.save(out, t.numpy())
        assert tmax == float(world)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_images(tmp_path):
    shape = (28, 22, 24)
    nshots = 3
    out = str(tmp_path / "img.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), nshots, shape, out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    want = sum(_shot_image(100 + s, shape) for s in range(nshots))
    assert np.allclose(got, want, rtol=1e-6, atol=1e-12)
