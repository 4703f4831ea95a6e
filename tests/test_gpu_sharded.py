"""State-sharded runs through the library on one GPU.

Two contexts, each with a block of the states, run in two host threads; their density exchange
is a host hook that waits for the context stream, sums the two partial density arrays and
writes the sum back (no kernel waits on another: the meeting point is a host barrier after
each stream has drained).  The result must equal one context holding all states — forward
step, energies and the adjoint gradient.  NCCL is checked as a one-rank communicator (the
in-place all-reduce on the context stream), since this machine gives one GPU per run.
"""
import threading

import numpy as np
import pytest

from parity_util import inputs, rel
from wslda_b200.sharding import gather_rows, shard_rows, shard_vector

NSTEPS = 4


class _DevArray:
    """zero-copy view of device doubles for torch.as_tensor"""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class PairExchange:
    """density exchange of two contexts driven by two host threads"""

    def __init__(self, world=2):
        self.world = world
        self.bar = threading.Barrier(world, timeout=120)
        self.bufs = [None] * world
        self.calls = [0] * world

    def hook(self, rank):
        def fn(ptr, count, stream):
            import torch
            torch.cuda.ExternalStream(int(stream)).synchronize()
            t = torch.as_tensor(_DevArray(ptr, count), device="cuda")
            self.bufs[rank] = t.cpu().numpy().copy()
            self.bar.wait()
            total = self.bufs[0].copy()
            for b in self.bufs[1:]:
                total += b
            t.copy_(torch.from_numpy(total).cuda())
            torch.cuda.synchronize()
            self.calls[rank] += 1
            self.bar.wait()
        return fn


def _run_threads(fns):
    out, errs = [None] * len(fns), []

    def wrap(i):
        try:
            out[i] = fns[i]()
        except Exception as e:  # surfaced in the test
            errs.append(e)

    ths = [threading.Thread(target=wrap, args=(i,)) for i in range(len(fns))]
    for t in ths:
        t.start()
    for t in ths:
        t.join(timeout=600)
    assert not errs, errs
    return out


def _sharded_runs(project, nwf, world):
    from wslda_b200 import TDRun
    proj, d = inputs(project, nwf)
    ex = PairExchange(world)
    runs = []
    for r in range(world):
        run = TDRun(project, len(shard_vector(d["occ"], nwf, world, r)))
        run.setup(shard_rows(d["states"], nwf, proj.numel, world, r), d["pots"], shard_vector(d["occ"], nwf, world, r),
                  d["params"], d["extra"])
        run.set_density_exchange(ex.hook(r))
        runs.append(run)
    return proj, d, ex, runs


@pytest.mark.gpu
@pytest.mark.parametrize("project,nwf", [("t2d_slda", 37), ("c4_bdg2d", 24)])
def test_sharded_step_matches_single(has_gpu, project, nwf):
    import torch
    torch.cuda.init()
    from parity_util import run_gpu
    world = 2
    proj, d, ex, runs = _sharded_runs(project, nwf, world)

    def job(run):
        def f():
            run.initial_measurement()
            run.steps(NSTEPS)
            return dict(states=run.states(), dens=run.densities(), pots=run.potentials(), energy=run.energy())
        return f

    res = _run_threads([job(r) for r in runs])
    for r in runs:
        r.close()
    full = run_gpu(project, nwf, NSTEPS, inp=d)
    assert ex.calls == [1 + 2 * NSTEPS] * world
    for r in res:
        assert rel(r["dens"], full["densities"]) < 1e-12
        assert rel(r["pots"], full["potentials"]) < 1e-12
        assert np.allclose(r["energy"], full["energy"], rtol=1e-11, atol=1e-12)
    assert rel(gather_rows([r["states"] for r in res], proj.numel), full["states"]) < 1e-12


@pytest.mark.gpu
def test_sharded_adjoint_matches_single(has_gpu):
    import torch
    torch.cuda.init()
    from wslda_b200 import TDRun
    project, nwf, world = "c4_bdg2d", 24, 2
    proj, d, ex, runs = _sharded_runs(project, nwf, world)
    out = _run_threads([lambda r=r: r.adjoint(5, nparam=14, checkpoint_every=2) for r in runs])
    for r in runs:
        r.close()
    one = TDRun(project, nwf)
    one.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    loss, g = one.adjoint(5, nparam=14, checkpoint_every=2)
    one.close()
    for l_r, g_r in out:
        assert abs(l_r - loss) <= 1e-12 * abs(loss)
        assert rel(g_r, g) < 1e-10


@pytest.mark.gpu
def test_nccl_single_rank_exchange(has_gpu):
    """a one-rank NCCL communicator: the in-place all-reduce runs on the context stream and
    leaves the run unchanged"""
    import torch
    torch.cuda.init()
    from parity_util import run_gpu
    from wslda_b200 import TDRun
    project, nwf = "t2d_slda", 16
    proj, d = inputs(project, nwf)
    run = TDRun(project, nwf)
    run.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    run.attach_nccl(run.nccl_unique_id(), 1, 0)
    run.initial_measurement()
    run.steps(NSTEPS)
    dens, y = run.densities(), run.states()
    run.close()
    full = run_gpu(project, nwf, NSTEPS, inp=d)
    assert np.array_equal(dens, full["densities"])
    assert np.array_equal(y, full["states"])
