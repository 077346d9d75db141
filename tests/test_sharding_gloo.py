"""Instance sharding over 2 ranks (gloo, CPU).

The batched and served forms split independent models over GPUs with no
collective on the data path.  Here two CPU ranks split a batch of small
plates, solve their shares with the CPU restatement of the reference (the
oracle, standing in for the device batch) and exchange results once; every
rank must end with the serial results, in order.
"""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from solvix_b200 import workloads
from solvix_b200.sharding import shard_instances, solve_sharded


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _plates():
    rng = np.random.Generator(np.random.PCG64(21))
    return [workloads.plate(rng, nx=int(rng.integers(3, 9)), ny=int(rng.integers(2, 4)))
            for _ in range(10)]


def _oracle_solve(flats):
    from oracle import oracle
    return [oracle.solve_flat(f).u for f in flats]


def _rank_main(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        flats = _plates()
        seen = []

        def solve(shard):
            seen.extend(f.n_dof for f in shard)
            return _oracle_solve(shard)

        res = solve_sharded(flats, solve, rank, world)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.concatenate(res))
        np.save(os.path.join(out_dir, f"n{rank}.npy"), np.asarray(seen))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_and_gather(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    flats = _plates()
    serial = np.concatenate(_oracle_solve(flats))
    shards = shard_instances([f.n_dof for f in flats], world)
    for r in range(world):
        np.testing.assert_array_equal(np.load(tmp_path / f"r{r}.npy"), serial)
        # each rank solved exactly its own shard
        assert sorted(np.load(tmp_path / f"n{r}.npy").tolist()) == \
            sorted(flats[k].n_dof for k in shards[r])
