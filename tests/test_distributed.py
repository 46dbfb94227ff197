"""Multi-rank host logic on CPU: world_size 2, gloo.  The device calls are
replaced by CPU stand-ins (a seeded fake for C(t); the oracle's M0/M2 integrand
sums over a Philox counter range for the moments); no GPU is used."""
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


def _oracle_moment(ms, params, T, n, offset, seed, moment, precision):
    from oracle import oracle as O
    from tests.helpers import oracle_params, oracle_system
    fn = O.m0 if moment == 0 else O.m2
    return fn(oracle_system("co2ar"), oracle_params("co2ar", 64, 100.0), T, n, seed, offset=offset, nthreads=1)


def _moment_worker(rank, world, port, out, moment):
    import torch.distributed as dist
    from hawaiihybrid_b200 import hawaii as H
    from hawaiihybrid_b200.distributed import moment_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = H.CalcParams(sampler_Rmin=4.0, sampler_Rmax=40.0)
        m, e = moment_sharded(None, p, [150.0, 300.0, 400.0], 20000, 99, moment=moment,
                              compute=_oracle_moment)
        out[rank] = (m.tolist(), e.tolist())
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_moment_sharded_equals_single_rank_gloo():
    """Two ranks over disjoint Philox counter ranges, all-reduced, give the moments of
    one rank drawing all the samples (mpi_calculate_M0 / M2 partitioning)."""
    import pytest
    from oracle import oracle as O
    from tests.helpers import oracle_params, oracle_system
    from hawaiihybrid_b200 import hawaii as H
    if not O.lib():
        pytest.skip("oracle not built")
    T = np.array([150.0, 300.0, 400.0])
    p = H.CalcParams(sampler_Rmin=4.0, sampler_Rmax=40.0)
    for moment, fn in ((0, O.m0), (2, O.m2)):
        mgr = mp.Manager()
        out = mgr.dict()
        mp.spawn(_moment_worker, args=(2, _free_port(), out, moment), nprocs=2, join=True)
        sw, sw2 = fn(oracle_system("co2ar"), oracle_params("co2ar", 64, 100.0), T, 40000, 99, nthreads=1)
        m_ref, e_ref = H.moment_from_sums(sw, sw2, 40000, H.moment_scale(p, moment))
        for r in range(2):
            m, e = out[r]
            np.testing.assert_allclose(m, m_ref, rtol=1e-12)
            np.testing.assert_allclose(e, e_ref, rtol=1e-9)
        assert np.all(np.asarray(out[0][0]) > 0)
