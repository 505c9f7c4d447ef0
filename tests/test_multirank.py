"""Run sharding over ranks (the bench's weak-scaling path), on CPU with the
gloo backend and world size 2: each rank simulates its own run ranges with
the CPU oracle (standing in for its GPU), the counters are summed and the
times maxed across ranks, and the combined result equals one process
simulating the union of the ranges."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from cusmc_b200 import api, netgen, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, blob, qargs, out_dir):
    import torch.distributed as dist

    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    q = api.variable_query(*qargs[:2], threshold=qargs[2], is_max=True)
    hits = steps = 0
    ms = 0.0
    for s in range(3):
        r, _, wall = oracle.run(blob, q, 5, 64, shard.first_run(s, rank, world, 64), threads=1)
        hits += r.hits
        steps += r.steps
        ms += wall
    (hits, steps), (ms,) = shard.combine([hits, steps], [ms])
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array([hits, steps, ms]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_cover_disjoint_ranges_and_combine_exactly():
    import oracle
    w = netgen.epidemic(n_agents=20)
    with tempfile.TemporaryDirectory() as d:
        blob = api.compile_model(w.write(os.path.join(d, "e.xml")))
        qargs = (w.var_id, 40, 9)
        mp.start_processes(_worker, args=(2, _free_port(), blob, qargs, d), nprocs=2, start_method="spawn")
        got = [np.load(os.path.join(d, f"rank{r}.npy")) for r in range(2)]
    assert np.array_equal(got[0][:2], got[1][:2])  # every rank holds the combined counters
    q = api.variable_query(qargs[0], qargs[1], threshold=qargs[2], is_max=True)
    r, _, _ = oracle.run(blob, q, 5, 6 * 64, 0, threads=0)  # steps 0..2 x ranks 0..1 = runs 0..383
    assert int(got[0][0]) == r.hits and int(got[0][1]) == r.steps


def test_ranges_are_disjoint_and_contiguous():
    seen = []
    for s in range(4):
        for rank in range(3):
            a = shard.first_run(s, rank, 3, 10)
            seen.extend(range(a, a + 10))
    assert sorted(seen) == list(range(120))
