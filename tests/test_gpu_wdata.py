"""W-data output (wtd_wdata_begin / _write) against the reference's own writer
(hpc-engine/wslda_writevars.c over lib/wdata, compiled where they lie with the single-process MPI
shim: oracle/wd_ref.c, oracle/_ref/<p>/libwdref.so) fed the same densities, potentials and
external fields.  Every variable tag of the input's writevar list, over three cycles with steps
between them: the .wdat files are byte-identical and the .wtxt metadata equal line by line
(after the generator's comment line)."""
import ctypes
import os

import numpy as np
import pytest

from parity_util import inputs

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ALL = "rho j tau V V_ext velocity_ext delta delta_ext nu alpha A"
_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


@pytest.mark.gpu
@pytest.mark.parametrize("name,fprec", [("t2d_vext", 0), ("t3d_aslda", 0), ("t1d_bdg_sym", 0), ("t2d_vext", 1)])
def test_wdata_matches_reference_writer(has_gpu, tmp_path, name, fprec):
    from wslda_b200 import TDRun
    so = os.path.join(REPO, "oracle", "_ref", name, "libwdref.so")
    if not os.path.exists(so):
        pytest.skip("the reference's W-data writer is built in the build container (make -C oracle wdref)")
    ref = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    ref.wdref_begin.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    ref.wdref_write.argtypes = [ctypes.c_int] + [_dp] * 7
    ref.wdref_meta.argtypes = [ctypes.c_char_p]
    nwf = 24
    proj, d = inputs(name, nwf)
    N, dim = proj.numel, proj.codedim
    c = proj.constants()
    sym = 1 if "_sym" in name else 0
    run = TDRun(name, nwf)
    run.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    run.initial_measurement()
    lib_prefix, ref_prefix = str(tmp_path / "lib" / "td"), str(tmp_path / "ref" / "td")
    os.makedirs(os.path.dirname(lib_prefix)); os.makedirs(os.path.dirname(ref_prefix))
    t0, dtc = c["t0"], 2 * c["dt"]
    run.wdata_begin(lib_prefix, ALL, t0, dtc, float_prec=bool(fprec))
    assert ref.wdref_begin(os.fsencode(ref_prefix), ALL.encode(), t0, dtc, sym, c["kF"], 0.5 * c["kF"] ** 2,
                           c["mu_a"], c["mu_b"], fprec) == 0
    lib = run.lib
    lib.get_v_ext.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
    lib.get_velocity_ext.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
    lib.get_delta_ext.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, _dp]
    for cycle in range(3):
        run.wdata_write()
        it = run.time_index()
        dens, pots = run.densities(), run.potentials()
        vext = [np.zeros(N), np.zeros(N)]
        velext = [np.zeros(3 * N), np.zeros(3 * N)]
        for s in range(2):
            assert lib.get_v_ext(dim, s, it, _p(vext[s])) == 0
            assert lib.get_velocity_ext(dim, s, it, _p(velext[s])) == 0
        dext = np.zeros(2 * N)
        states, dptr, pptr = ctypes.c_void_p(), ctypes.POINTER(ctypes.c_double)(), ctypes.POINTER(ctypes.c_double)()
        run._check(lib.wtd_device_pointers(run.h, ctypes.byref(states), ctypes.byref(dptr), ctypes.byref(pptr)))
        delta_dev = ctypes.cast(pptr, ctypes.c_void_p).value + 2 * N * 8
        assert lib.get_delta_ext(dim, it, ctypes.c_void_p(delta_dev), _p(dext)) == 0
        assert ref.wdref_write(it, _p(dens), _p(pots), _p(vext[0]), _p(vext[1]), _p(velext[0]), _p(velext[1]),
                               _p(dext)) == 0
        run.steps(2)
    run.close()
    names = sorted(f for f in os.listdir(tmp_path / "ref") if f.endswith(".wdat"))
    assert names and names == sorted(f for f in os.listdir(tmp_path / "lib") if f.endswith(".wdat"))
    for f in names:
        a, b = (tmp_path / "lib" / f).read_bytes(), (tmp_path / "ref" / f).read_bytes()
        assert len(a) == len(b) and a == b, f
    # the reference's metadata of the set after its three cycles
    wd = ref.wdref_meta
    meta_ref = str(tmp_path / "ref.wtxt")
    assert wd(os.fsencode(meta_ref)) == 0
    mine = open(lib_prefix + ".wtxt").read().splitlines()
    theirs = open(meta_ref).read().splitlines()
    assert mine[0].startswith("# Generated by") and mine[1] == ""
    # the reference counts cycles in the same call that writes them (wdata_add_cycle); the prefix
    # differs only by directory
    mine = [l.replace(lib_prefix, ref_prefix) for l in mine[2:]]
    theirs = [l for l in theirs]
    assert mine == theirs
