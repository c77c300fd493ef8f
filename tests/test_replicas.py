"""Replica plumbing of the multi-GPU benchmark on CPU: two gloo ranks.

The physics stage does not partition a world; bench.py --gpus N runs one
independent replica per GPU.  What crosses ranks is the measurement: the
slowest rank's timed region (max) and the work of all ranks (sum), with
barriers around the timed region, and each rank steps distinct worlds
(its own seed).  Here two processes check exactly that with the gloo
backend, together with the split of one set of worlds across ranks by
cell count (the batched benchmark's ``--partition global``).
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world_size), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from alien_b200.replicas import Replicas

    reps = Replicas(backend="gloo", timeout_s=60)
    reps.barrier()
    ms = 10.0 + 5.0 * rank          # rank 1 is the slowest
    cells = 1000 * (rank + 1)
    sizes = [5, 90, 17, 33, 33, 1, 64, 20]
    mine = reps.share(sizes)
    out[rank] = (reps.max(ms), reps.sum(cells), reps.seed(7), mine, reps.sum(sum(sizes[i] for i in mine)))
    reps.barrier()
    reps.close()


def test_two_gloo_replicas_reduce_timing_and_work():
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0][0] == out[1][0] == 15.0      # max over ranks
    assert out[0][1] == out[1][1] == 3000.0    # sum over ranks
    assert out[0][2] != out[1][2]              # distinct worlds per rank
    assert sorted(out[0][3] + out[1][3]) == list(range(8))   # every world on exactly one rank
    assert out[0][4] == out[1][4] == 263.0


def test_partition_balances_cells():
    import numpy as np

    from alien_b200 import worldgen
    from alien_b200.replicas import partition_worlds

    sizes = worldgen.batched_sizes(seed=0, count=256)
    for n in (1, 2, 3, 4, 8):
        parts = partition_worlds(sizes, n)
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        loads = [int(np.sum(np.asarray(sizes)[p])) for p in parts]
        # greedy placement: no rank exceeds the mean by more than one world
        assert max(loads) <= sum(loads) / n + max(sizes)
        assert partition_worlds(sizes, n) == parts     # same split on every call
    assert partition_worlds([3, 3, 2, 2, 2], 2) == [[0, 2, 4], [1, 3]]
    assert partition_worlds([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        partition_worlds([1], 0)


def test_single_process_is_identity():
    from alien_b200.replicas import Replicas

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    reps = Replicas(backend="gloo")
    assert reps.world_size == 1 and reps.max(3.5) == 3.5 and reps.sum(2) == 2.0
    reps.close()
