"""The N > 1 host path on CPU: world_size 2 with the gloo backend. Each rank
tallies its own shard of photons (here with the CPU oracle: no GPU needed);
the integer reduction must equal the single-process tally of all photons, and
the timing reduction must return the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, mode):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from gpu_optical_photons_b200 import params as P
    from gpu_optical_photons_b200.distributed import (max_over_ranks, reduce_tallies,
                                                      shard_events, shard_first_id)
    from gpu_optical_photons_b200.wavefront import batched_events
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = P.TallyConfig(100, 50.0, 10)
        if mode == "photons":
            p = P.config2()[0]
            n = 20_000
            t = O.tally(p, c, n, shard_first_id(rank, n), threads=1)
        else:
            events, counts = batched_events(n_events=24, seed=3, median=800, n_min=10, n_max=5000)
            (lo, hi), off = shard_events(counts, rank, world)
            offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
            arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
            per_event = O.batch_tally(arr, offs, c, threads=1)
            t = np.zeros((len(events), c.length), np.uint64)
            t[lo:hi] = per_event[lo:hi]
            assert int(offs[lo]) == off
        total = reduce_tallies(t, dist)
        m = max_over_ranks(10.0 + rank, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, f"{mode}.npy"), total)
            with open(os.path.join(out_dir, f"{mode}_max.txt"), "w") as f:
                f.write(str(m))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["photons", "events"])
def test_two_rank_shards_reduce_exactly(tmp_path, oracle, mode):
    from gpu_optical_photons_b200 import params as P
    from gpu_optical_photons_b200.wavefront import batched_events
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), mode), nprocs=world,
                       start_method="spawn", join=True)
    got = np.load(tmp_path / f"{mode}.npy")
    c = P.TallyConfig(100, 50.0, 10)
    if mode == "photons":
        want = oracle.tally(P.config2()[0], c, 40_000, 0, threads=2)
    else:
        events, counts = batched_events(n_events=24, seed=3, median=800, n_min=10, n_max=5000)
        offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
        arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
        want = oracle.batch_tally(arr, offs, c, threads=2)
    assert np.array_equal(got, want)
    assert float((tmp_path / f"{mode}_max.txt").read_text()) == 11.0


def test_shard_events_covers_all():
    from gpu_optical_photons_b200.distributed import shard_events
    counts = np.array([5, 0, 100, 7, 7, 300, 1, 1, 50], np.uint64)
    for world in (1, 2, 3, 4):
        ranges = [shard_events(counts, r, world)[0] for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == len(counts)
        for a, b in zip(ranges, ranges[1:]):
            assert a[1] == b[0]
