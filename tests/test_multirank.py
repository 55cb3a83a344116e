"""Multi-rank host logic on CPU (gloo, world size 2): the irreducible q points are dealt
round-robin over ranks (src/cugw_utils.cu:115) and the partial Sigma are summed with an
all-reduce (src/gw_gpu_kernel.cpp:187); the sum must equal the single-rank build."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from green_gpu_b200 import synth
    from oracle import gw as ogw
    s = synth.make_system(mesh=(3, 2, 1), nao=4, NQ=10, ns=1, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=1,
                          symmetry="tr")
    # the library's own shard assignment (host-side, callable without a GPU)
    from green_gpu_b200 import native
    mine = native.q_shard_points(s.inq, rank, world)
    assert mine == list(range(rank, s.inq, world))
    part = ogw.gw_build(s, q_subset=mine)
    t = torch.from_numpy(part.view(np.float64).copy())
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy().view(np.complex128))
    dist.barrier()
    dist.destroy_process_group()


def test_q_sharded_sigma_sums_to_full(tmp_path):
    from green_gpu_b200 import synth
    from oracle import gw as ogw
    out = str(tmp_path / "sigma.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    s = synth.make_system(mesh=(3, 2, 1), nao=4, NQ=10, ns=1, beta=10.0, lam=100.0, nts=24, nw_b=21, seed=1,
                          symmetry="tr")
    full = ogw.gw_build(s)
    got = np.load(out)
    assert np.abs(got - full).max() < 1e-13 * np.abs(full).max()


def test_round_robin_partition_covers_every_q_once():
    from green_gpu_b200 import native
    for inq in (1, 4, 7, 64):
        for world in (1, 2, 3, 8):
            seen = sorted(q for r in range(world) for q in native.q_shard_points(inq, r, world))
            assert seen == list(range(inq))
    import pytest
    with pytest.raises(native.GreenError):
        native.q_shard_points(4, 2, 2)
