"""Replica plumbing on CPU: two gloo ranks split a batch, bootstrap their
shares with the CPU statement of the path and agree on the job time and
count; the union of the shares equals the single-process result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tfhe_b200.replicas import shard


def test_shard_covers_batch_exactly_once():
    for batch in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in shard(batch, r, world)]
            assert got == list(range(batch))
            sizes = [len(shard(batch, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (root, here, os.path.join(root, "blind-spiking-lstm_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    from oracle import tfhe_oracle as O
    from tfhe_b200.replicas import max_over_ranks, shard as shard_fn, total_over_ranks
    from pbs_cases import PARAMS, inputs, keys, ks_params, step_body

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    name = "tiny_c3"
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = inputs(name, 10)
    mine = shard_fn(10, rank, world)
    ca, cb = O.key_switch_LWE(k.ksk, (a[mine.start:mine.stop], b[mine.start:mine.stop]), ks_params(name))
    body = step_body(name)
    n = len(mine)
    oa, ob = O.cuboot_merge((ca, cb), [np.zeros((n, p["N"])), np.broadcast_to(body, (n, p["N"]))],
                            k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"], p["collapse"], k.all_rot, 1)
    np.save(os.path.join(out_dir, f"rank{rank}_a.npy"), oa)
    np.save(os.path.join(out_dir, f"rank{rank}_b.npy"), ob)
    t_max = max_over_ranks(1.0 + rank, dist)
    total = total_over_ranks(n, dist)
    np.save(os.path.join(out_dir, f"rank{rank}_stats.npy"), np.array([t_max, total]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_single_process(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    from oracle import tfhe_oracle as O
    from pbs_cases import PARAMS, inputs, keys, ks_params, step_body
    name = "tiny_c3"
    p = PARAMS[name]
    k = keys(name)
    msgs, a, b = inputs(name, 10)
    ca, cb = O.key_switch_LWE(k.ksk, (a, b), ks_params(name))
    body = step_body(name)
    wa, wb = O.cuboot_merge((ca, cb), [np.zeros((10, p["N"])), np.broadcast_to(body, (10, p["N"]))],
                            k.bsk_ordered, p["q"], p["beta_bs"], p["l_bs"], p["N"], p["collapse"], k.all_rot, 1)
    got_a = np.concatenate([np.load(tmp_path / f"rank{r}_a.npy") for r in range(world)])
    got_b = np.concatenate([np.load(tmp_path / f"rank{r}_b.npy") for r in range(world)])
    assert np.array_equal(got_a, wa) and np.array_equal(got_b, wb)
    for r in range(world):
        t_max, total = np.load(tmp_path / f"rank{r}_stats.npy")
        assert t_max == 2.0 and total == 10
