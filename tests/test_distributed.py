"""Multi-rank host logic on CPU: world_size 2, gloo, a fake per-rank compute
(the device call is replaced; no GPU is used)."""
import os

import numpy as np
import torch.multiprocessing as mp


def _fake_compute(ms, params, T, n, precision, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(params["N"]) * n, float(n), {"seed": seed}


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from hawaiihybrid_b200.distributed import correlation_iteration_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        crln, ntraj, st = correlation_iteration_sharded(None, {"N": 16}, 300.0, 100, 0, 7,
                                                        compute=_fake_compute)
        out[rank] = (crln.tolist(), ntraj, st["seed"])
    finally:
        dist.destroy_process_group()


def test_sharded_allreduce_gloo():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    expected = sum(_fake_compute(None, {"N": 16}, 300.0, 100, 0, 7 + 1000 * r)[0] for r in range(2))
    for r in range(2):
        crln, ntraj, seed = out[r]
        assert seed == 7 + 1000 * r
        assert ntraj == 200.0
        np.testing.assert_allclose(crln, expected, rtol=1e-14)


def test_rank_seed_table():
    from hawaiihybrid_b200.distributed import rank_seed
    seeds = [rank_seed(42, r) for r in range(8)]
    assert seeds[0] == 42 and len(set(seeds)) == 8 and all(s > 0 for s in seeds)
