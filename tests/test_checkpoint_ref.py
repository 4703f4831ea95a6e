"""The reference's checkpoint writer and reader (oracle/ck_ref.c over oracle/mpi_shim) on the CPU:
what a 3-rank run in IO groups of 2 writes, it reads back rank by rank, so the shim's emulation
of the ranks and IO groups is the one the reference's code assumes."""
import ctypes
import os

import numpy as np
import pytest

from wslda_b200 import projects as P

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


@pytest.mark.parametrize("name", ["t2d_slda", "t1d_aslda", "t3d_slda"])
def test_reference_checkpoint_roundtrip(tmp_path, name):
    so = os.path.join(REPO, "oracle", "_ref", name, "libckref.so")
    if not os.path.exists(so):
        pytest.skip("the reference's checkpoint code is built in the build container (make -C oracle ckref)")
    lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    lib.ckref_load.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 4 + [_dp] * 8 + [ctypes.POINTER(ctypes.c_int), _dp, _dp]
    proj = P.Project(name)
    N, nh = proj.numel, proj.nhist
    scheme = {3: 34, 4: 45, 5: 55}[nh]
    nwf, nranks, howmany = 23, 3, 2
    rng = np.random.default_rng(5)
    data = []
    for r in range(nranks):
        n = nwf // nranks + (1 if r < nwf % nranks else 0)
        arrs = [rng.standard_normal(2 * n * N) + 1j * rng.standard_normal(2 * n * N) for _ in range(1 + nh)]
        arrs += [None] * (5 - nh)
        pots = rng.standard_normal(12 * N)
        meta = np.array([0.25, 0.5, 0.4, 12.0, 1.0, 0.5, 30.0, 20.0])
        En, kp = rng.standard_normal(n), rng.standard_normal(2 * n)
        rc = lib.ckref_save(os.fsencode(str(tmp_path)), r, nranks, howmany, scheme, nwf,
                            *[_p(None if a is None else a.view(np.float64)) for a in arrs], _p(pots), _p(meta),
                            _p(En), _p(kp))
        assert rc == 0
        data.append((n, arrs, pots, meta, En, kp))
    assert sorted(os.listdir(tmp_path)) == ["checkpoint_0", "checkpoint_1"]
    for r, (n, arrs, pots, meta, En, kp) in enumerate(data):
        got = [np.zeros(2 * n * N, dtype=np.complex128) for _ in range(1 + nh)] + [None] * (5 - nh)
        gp, gm, gn, ge, gk = np.zeros(12 * N), np.zeros(8), ctypes.c_int(0), np.zeros(n), np.zeros(2 * n)
        rc = lib.ckref_load(os.fsencode(str(tmp_path)), r, nranks, howmany, scheme,
                            *[_p(None if a is None else a.view(np.float64)) for a in got], _p(gp), _p(gm),
                            ctypes.byref(gn), _p(ge), _p(gk))
        assert rc == 0 and gn.value == nwf
        for a, b in zip(arrs[:1 + nh], got[:1 + nh]):
            assert np.array_equal(a, b)
        assert np.array_equal(gm, meta) and np.array_equal(ge, En)
        if proj.codedim == 2:
            assert np.array_equal(gk[:n], kp[:n])
        elif proj.codedim == 1:
            assert np.array_equal(gk, kp)
        # the potentials come from the first rank of the group
        assert np.array_equal(gp, data[r - r % howmany][2])
