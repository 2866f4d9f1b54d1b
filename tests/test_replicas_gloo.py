"""The multi-GPU path of bench.py on CPU: two gloo ranks, each a replica on
its own seeded snapshot (the path has no exchange step), timed as the max
over ranks.  The hot path of each replica runs on the oracle backend here
(no GPU); the rank logic is the bench's own."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    import bench
    from asohf_b200 import driver, synth
    from oracle import oracle as O
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        cfg = bench.replica_config(synth.CONFIGS["tiny"], rank)
        r = driver.run(synth.generate(cfg), O.OracleBackend(nthreads=1), with_subs=False)
        ms_local = 10.0 * (rank + 1)  # unequal per-rank times: the job is as slow as its slowest rank
        ms = bench.max_over_ranks(ms_local, WORLD, dist, "cpu")
        dist.barrier()
        n = r.cat.nclus
        out[rank] = (cfg.seed, ms, r.cat.realclus[:n].copy(), r.u1.copy())
    finally:
        dist.destroy_process_group()


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, port, out)) for r in range(WORLD)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    (s0, ms0, rc0, u0), (s1, ms1, rc1, u1) = res[0], res[1]
    assert s1 == s0 + 1                      # one snapshot per rank
    assert ms0 == ms1 == 20.0                # max over ranks, the same on every rank
    assert not np.array_equal(u0, u1)        # independent replicas
    # a replica's result does not depend on the other rank (no exchange)
    import bench
    from asohf_b200 import driver, synth
    from oracle import oracle as O
    r = driver.run(synth.generate(bench.replica_config(synth.CONFIGS["tiny"], 1)), O.OracleBackend(nthreads=1),
                   with_subs=False)
    assert np.array_equal(r.u1, u1)
    assert np.array_equal(r.cat.realclus[:r.cat.nclus], rc1)
