"""Replica plumbing of the multi-GPU benchmark on CPU: two gloo ranks.

The physics stage does not partition a world; bench.py --gpus N runs one
independent replica per GPU.  What crosses ranks is the measurement: the
slowest rank's timed region (max) and the work of all ranks (sum), with
barriers around the timed region, and each rank steps distinct worlds
(its own seed).  Here two processes check exactly that with the gloo
backend.
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
    out[rank] = (reps.max(ms), reps.sum(cells), reps.seed(7))
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


def test_single_process_is_identity():
    from alien_b200.replicas import Replicas

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    reps = Replicas(backend="gloo")
    assert reps.world_size == 1 and reps.max(3.5) == 3.5 and reps.sum(2) == 2.0
    reps.close()
