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


def _ledger_rank(rank, world, port, ledger_base, nshots, stop_after, out):
    import torch.distributed as dist

    from wavefd_b200.shots import ShotLedger, partition_shots
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    led = ShotLedger(ledger_base, rank)
    todo = led.pending(partition_shots(nshots, world, rank))
    ran = []
    for s in todo:
        if stop_after is not None and len(ran) == stop_after:
            break  # the job stops here (a restart picks up the rest)
        ran.append(s)
        led.done(s)
    with open(f"{out}.{rank}", "a") as f:
        f.write(" ".join(map(str, ran)) + "\n")
    dist.barrier()
    dist.destroy_process_group()


def test_shot_ledger_resume_two_ranks(tmp_path):
    """Two gloo ranks stop after one shot each; the restarted job runs only the remaining shots, and
    every shot is run exactly once over both runs. A half-written line (a crash mid-write) is ignored."""
    nshots = 7
    base = str(tmp_path / "ledger")
    out = str(tmp_path / "ran")
    mp.start_processes(_ledger_rank, args=(2, _free_port(), base, nshots, 1, out), nprocs=2, join=True,
                       start_method="spawn")
    with open(base + ".rank1", "a") as f:
        f.write("1 6")  # no newline: cut short
    mp.start_processes(_ledger_rank, args=(2, _free_port(), base, nshots, None, out), nprocs=2, join=True,
                       start_method="spawn")
    ran = []
    for r in range(2):
        with open(f"{out}.{r}") as f:
            for line in f:
                ran += [int(x) for x in line.split()]
    assert sorted(ran) == list(range(nshots))
    from wavefd_b200.shots import ShotLedger
    assert ShotLedger(base).finished() == set(range(nshots))
