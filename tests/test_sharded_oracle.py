"""State-sharded runs on CPU: two gloo ranks, each holding a block of the states, with the density
exchange (sum over ranks after every density reduction) reproduce the single-process run.

This checks the sharding rule (getnwfip, hpc-engine/pca_utils.c:660-664), the exchange points
(initial measurement and both half steps, pca.c:948, 1433, 1505) and the per-rank bookkeeping
on the oracle, whose hook has the same contract as the library's wtd_set_density_exchange.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from wslda_b200.sharding import gather_rows, shard_range, shard_rows, shard_vector

NSTEPS = 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_partition():
    for nwf in (1, 2, 7, 13, 64, 1000):
        for world in (1, 2, 3, 4, 8):
            if world > nwf:
                continue
            rs = [shard_range(nwf, world, r) for r in range(world)]
            assert rs[0][0] == 0
            assert sum(c for _, c in rs) == nwf
            for (o0, c0), (o1, _) in zip(rs, rs[1:]):
                assert o1 == o0 + c0
            assert max(c for _, c in rs) - min(c for _, c in rs) <= 1
            # the reference's rule: nwf // np, plus one for the first nwf % np ranks
            assert [c for _, c in rs] == [nwf // world + (1 if r < nwf % world else 0) for r in range(world)]
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_shard_gather_roundtrip():
    rng = np.random.default_rng(3)
    nwf, n = 11, 7
    y = rng.standard_normal(2 * nwf * n) + 1j * rng.standard_normal(2 * nwf * n)
    parts = [shard_rows(y, nwf, n, 3, r) for r in range(3)]
    assert np.array_equal(gather_rows(parts, n), y)
    occ = np.arange(nwf, dtype=float)
    assert np.array_equal(np.concatenate([shard_vector(occ, nwf, 3, r) for r in range(3)]), occ)


def _rank_main(rank, world, port, project, nwf, outdir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from oracle_lib import Oracle
        from parity_util import inputs
        proj, d = inputs(project, nwf)
        o = Oracle(project, threads=2)
        o.setup(shard_rows(d["states"], nwf, proj.numel, world, rank), d["pots"],
                shard_vector(d["occ"], nwf, world, rank), d["params"], d["extra"])
        calls = [0]

        def hook(dens):
            t = torch.from_numpy(dens)  # shares the oracle's buffer
            dist.all_reduce(t)
            calls[0] += 1

        o.set_density_exchange(hook)
        o.initial_measurement()
        o.steps(NSTEPS)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), states=o.states(), dens=o.densities(), pots=o.potentials(),
                 energy=o.energy(), qpe=o.qpe(), calls=calls[0])
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("project,nwf", [("t2d_slda", 13), ("c4_bdg2d", 10), ("t1d_aslda", 9)])
def test_sharded_oracle_matches_single(project, nwf):
    import torch.multiprocessing as mp
    from oracle_lib import build
    from parity_util import inputs, rel, run_oracle
    build(project)  # once, before the ranks load it
    world = 2
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_rank_main, args=(world, _free_port(), project, nwf, td), nprocs=world, join=True,
                           start_method="spawn")
        rs = [dict(np.load(os.path.join(td, f"r{r}.npz"))) for r in range(world)]
    proj, d = inputs(project, nwf)
    full = run_oracle(project, nwf, NSTEPS, inp=d, threads=2)
    for r in rs:
        # initial measurement + two half steps per step
        assert int(r["calls"]) == 1 + 2 * NSTEPS
        assert rel(r["dens"], full["densities"]) < 1e-12
        assert rel(r["pots"], full["potentials"]) < 1e-12
        assert np.allclose(r["energy"], full["energy"], rtol=1e-11, atol=1e-12)
    y = gather_rows([r["states"] for r in rs], proj.numel)
    assert rel(y, full["states"]) < 1e-12
    assert rel(np.concatenate([r["qpe"] for r in rs]), full["qpe"]) < 1e-11
