"""Checkpoints in the reference's file layout (wtd_checkpoint_save / _load) against the reference's
own writer and reader (hpc-engine/tdwslda_checkpoint.c compiled where it lies with a
single-process MPI shim, oracle/ck_ref.c, oracle/_ref/<p>/libckref.so).

A run of 3 ranks in IO groups of 2 (two files) is emulated by one context per rank on one GPU,
each with its share of the states (getnwfip) advanced a few steps so that the ABM history is
not zero:
- every file the library writes equals, byte for byte, the one the reference writes from the
  same arrays;
- the library reads the reference's files back exactly (states, history, potentials, header,
  energies, transverse momenta);
- a run that stops, writes a checkpoint and restarts from it continues the uninterrupted run.
"""
import ctypes
import os

import numpy as np
import pytest

from parity_util import inputs

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = ["t2d_slda", "t1d_aslda", "t3d_slda"]
NRANKS, HOWMANY = 3, 2
_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _nwfip(rank, nranks, nwf):
    return nwf // nranks + (1 if rank < nwf % nranks else 0)


def _ckref(name):
    so = os.path.join(REPO, "oracle", "_ref", name, "libckref.so")
    if not os.path.exists(so):
        pytest.skip("the reference's checkpoint code is built in the build container (make -C oracle ckref)")
    lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    lib.ckref_save.restype = lib.ckref_load.restype = ctypes.c_int
    return lib


def _shards(name, nwf):
    """per rank: (states, occupations, k_perp) of its share, in rank order"""
    proj, d = inputs(name, nwf)
    N, st = proj.numel, d["states"].reshape(2, nwf, -1)
    out, first = [], 0
    for r in range(NRANKS):
        n = _nwfip(r, NRANKS, nwf)
        s = np.ascontiguousarray(st[:, first:first + n].reshape(-1))
        out.append((s, d["occ"][first:first + n], first, n))
        first += n
    return proj, d, out


def _meta(proj, it):
    c = proj.constants()
    return dict(t0=c["t0"] + it * c["dt"], mu_a=c["mu_a"], mu_b=c["mu_b"], ec=c["ec"], kF=c["kF"],
                eF=0.5 * c["kF"] ** 2, Effg=12.5, beta=20.0, nwf=0)


def _kperp(proj, first, n):
    k = 0.1 * (np.arange(first, first + n) % 5 - 2)
    if proj.codedim == 2:
        return k
    if proj.codedim == 1:
        return np.concatenate([k, -0.5 * k])
    return None


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_checkpoint_files_match_reference(has_gpu, tmp_path, name):
    from wslda_b200 import TDRun
    lib = _ckref(name)
    nwf = 23
    proj, d, shards = _shards(name, nwf)
    nh = proj.nhist
    scheme = {3: 34, 4: 45, 5: 55}[nh]
    lib_dir, ref_dir = tmp_path / "lib", tmp_path / "ref"
    lib_dir.mkdir(); ref_dir.mkdir()
    runs = []
    for r, (s, occ, first, n) in enumerate(shards):
        run = TDRun(name, n)
        run.setup(s, d["pots"], occ, d["params"], d["extra"])
        run.initial_measurement()
        run.steps(3)
        info = _meta(proj, 3)
        info["nwf"] = nwf
        En = np.linspace(-1.0, 1.0, nwf)[first:first + n].copy()
        kp = _kperp(proj, first, n)
        run.checkpoint_save(str(lib_dir), info, En, kp, rank=r, nranks=NRANKS, howmany=HOWMANY)
        # the reference writes the same arrays
        y = run.states()
        hist = [run.history(h) for h in range(nh)] + [None] * (5 - nh)
        pots = run.potentials()
        meta = np.array([info[k] for k in ("t0", "mu_a", "mu_b", "ec", "kF", "eF", "Effg", "beta")])
        kpr = np.zeros(2 * n) if kp is None else np.ascontiguousarray(kp)
        rc = lib.ckref_save(os.fsencode(str(ref_dir)), r, NRANKS, HOWMANY, scheme, nwf, _p(y.view(np.float64)),
                            *[_p(None if h is None else h.view(np.float64)) for h in hist], _p(pots), _p(meta),
                            _p(En), _p(kpr))
        assert rc == 0
        runs.append((run, y, hist[:nh], pots, En, kp, info))
    groups = sorted(os.listdir(lib_dir))
    assert groups == sorted(os.listdir(ref_dir)) == ["checkpoint_0", "checkpoint_1"]
    for g in groups:
        a = (lib_dir / g).read_bytes()
        b = (ref_dir / g).read_bytes()
        assert len(a) == len(b), (g, len(a), len(b))
        assert a == b, g
    # the library reads the reference's files back
    for r, (run, y, hist, pots, En, kp, info) in enumerate(runs):
        s, occ, first, n = shards[r]
        fresh = TDRun(name, n)
        c = proj.constants()
        fresh.setup(s * 0.5, d["pots"] * 0, occ * 0, d["params"], d["extra"])
        got_info, got_en, got_kp = fresh.checkpoint_load(str(ref_dir), rank=r, nranks=NRANKS, howmany=HOWMANY)
        assert got_info["nwf"] == nwf and got_info["beta"] == info["beta"] and got_info["t0"] == info["t0"]
        assert np.array_equal(got_en, En)
        if kp is not None:
            assert np.array_equal(got_kp[: kp.size], kp)
        for h in range(nh):
            assert np.array_equal(fresh.history(h), hist[h]), (r, h)
        # the load renormalises the (already normalised) states, as the restart measurement does
        assert np.abs(fresh.states() - y).max() < 1e-14
        first_rank = r - r % HOWMANY
        assert np.array_equal(fresh.potentials(), runs[first_rank][3])
        fresh.close()
        run.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_restart_continues_run(has_gpu, tmp_path, name):
    """write a checkpoint after 4 steps and restart from it: 3 more steps give the
    uninterrupted run's states and densities"""
    from wslda_b200 import TDRun
    nwf = 24
    proj, d = inputs(name, nwf)
    c = proj.constants()
    a = TDRun(name, nwf)
    a.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    a.initial_measurement()
    a.steps(3)
    a.steps(1)
    info = _meta(proj, 4)
    info["nwf"] = nwf
    # energies whose fbeta at beta = 20 gives back the run's occupations (1, then 0) exactly
    En = np.where(d["occ"] > 0.5, -10.0, 10.0)
    kp = None if proj.codedim == 3 else np.zeros(nwf * (2 if proj.codedim == 1 else 1))
    a.checkpoint_save(str(tmp_path), info, En, kp, rank=0, nranks=1, howmany=24)
    a.steps(3)
    want_states, want_dens = a.states(), a.densities()
    a.close()
    b = TDRun(name, nwf)
    const = dict(c)
    const["t0"] = info["t0"]
    b.setup(d["states"] * 0.5, d["pots"] * 0, d["occ"] * 0, d["params"], d["extra"], const=const)
    got_info, got_en, _ = b.checkpoint_load(str(tmp_path))
    assert got_info["nwf"] == nwf and np.array_equal(got_en, En)
    b.steps(3)
    assert np.abs(b.states() - want_states).max() < 1e-12
    assert np.abs(b.densities() - want_dens).max() < 1e-12 * max(1.0, np.abs(want_dens).max())
    b.close()
