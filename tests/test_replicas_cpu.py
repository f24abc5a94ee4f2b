"""The N > 1 layout on the CPU: world size 2 over gloo (127.0.0.1).  The batched sweep's specimens are sharded
by rank with no data-path collective; the ranks' oracle assemblies reproduce the single-process result, and
the timing reduction takes the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ice_fem_2025a_b200 import replicas


def test_shard_blocks_cover_exactly():
    for n, w in [(5, 2), (256, 8), (3, 4), (0, 3)]:
        got = [list(replicas.shard(n, r, w)) for r in range(w)]
        assert sum(got, []) == list(range(n))
        assert max(map(len, got)) - min(map(len, got)) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from ice_fem_2025a_b200 import abi, config as cf
    from oracle import oracle as orc
    mesh, d, st = replicas.specimen_shard(0.02, 0, rank, world)
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o, st())
    o.assemble(0, dt=100.0)
    o.assemble(1, dt=100.0)
    r = np.array([np.sum(o.residual(0) ** 2), np.sum(o.residual(1) ** 2), o.stats(1).crack_length])
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), r)
    m = replicas.max_over_ranks(float(rank + 1), dist)
    np.save(os.path.join(out_dir, f"max{rank}.npy"), np.array([m]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_specimen_sharding(oracle_lib, tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    parts = sum(np.load(tmp_path / f"rank{r}.npy") for r in range(world))
    from ice_fem_2025a_b200 import config as cf
    from oracle import oracle as orc
    mesh, d, st = cf.config(4, scale=0.02)
    o = orc.context(mesh, cf.materials(d), cf.options_from_json(d))
    cf.apply_state(o, st())
    o.assemble(0, dt=100.0)
    o.assemble(1, dt=100.0)
    full = np.array([np.sum(o.residual(0) ** 2), np.sum(o.residual(1) ** 2), o.stats(1).crack_length])
    assert np.allclose(parts, full, rtol=1e-12, atol=0)
    assert all(float(np.load(tmp_path / f"max{r}.npy")[0]) == 2.0 for r in range(world))
