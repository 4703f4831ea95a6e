"""The reference-named per-kernel ABI (include/wslda_td_compat.h) driven exactly as the
reference's host loop drives it (hpc-engine/pca.c:939-958 and 1401-1571, restated below over
ctypes with device buffers from gpu_malloc), checked against the golden outputs of the
reference's own kernels (tests/golden) and against the CPU oracle."""
import ctypes
import os
import sys

import numpy as np
import pytest

from parity_util import density_errors, inputs, rel, run_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from golden.make_golden import CASES  # noqa: E402

TOL = 1e-10
VP = ctypes.c_void_p
AB = {3: 34, 4: 45, 5: 55}


class Dev:
    """device buffer owned by the caller, as in the reference driver (pca.c:749-765)"""

    def __init__(self, lib, nbytes):
        self.lib = lib
        self.p = VP()
        assert lib.gpu_malloc(ctypes.c_size_t(nbytes), ctypes.byref(self.p)) == 0
        self.nbytes = nbytes

    def put(self, a):
        a = np.ascontiguousarray(a)
        assert self.lib.memcopy_host2gpu(a.ctypes.data_as(VP), self.p, ctypes.c_size_t(a.nbytes)) == 0

    def get(self, dtype, count):
        a = np.zeros(count, dtype=dtype)
        assert self.lib.memcopy_gpu2host(self.p, a.ctypes.data_as(VP), ctypes.c_size_t(a.nbytes)) == 0
        return a

    def zero(self):
        self.put(np.zeros(self.nbytes, dtype=np.uint8))

    def free(self):
        self.lib.gpu_free(self.p)


def run_compat(name, nwf, nsteps, nmeas):
    from wslda_b200 import load_library
    proj, d = inputs(name, nwf)
    lib = load_library(name)
    for fn in ("gpu_malloc", "gpu_free", "memcopy_host2gpu", "memcopy_gpu2host", "create_cufftPlans"):
        getattr(lib, fn).restype = ctypes.c_int
    lib.memcopy_const.argtypes = [ctypes.c_double] * 6
    lib.memcopy_const_sclgth.argtypes = [ctypes.c_double]
    N, S, nh, cd = proj.numel, nwf, proj.nhist, proj.codedim
    M = 2 * S * N
    c = proj.constants()
    assert lib.memcopy_const(c["mu_a"], c["mu_b"], c["ec"], c["t0"], c["dt"], c["kF"]) == 0
    params = np.ascontiguousarray(d["params"])
    assert lib.memcopy_const_params(params.ctypes.data_as(VP)) == 0
    assert lib.memcopy_const_sclgth(c["sclgth"]) == 0
    extra = None
    if d["extra"].size:
        extra = Dev(lib, d["extra"].nbytes)
        extra.put(d["extra"])
        assert lib.memcopy_extra_data(ctypes.c_size_t(d["extra"].nbytes), extra.p) == 0
    else:
        assert lib.memcopy_extra_data(ctypes.c_size_t(0), None) == 0
    wf = Dev(lib, M * 16)
    wf.put(d["states"])
    f = [Dev(lib, M * 16) for _ in range(nh)]
    for x in f:
        x.zero()
    dx, dy, dz, lap = (Dev(lib, M * 16) for _ in range(4))
    alap = Dev(lib, M * 16)
    dens = Dev(lib, 16 * N * 8)
    dens.zero()
    pots = Dev(lib, 12 * N * 8)
    pots.put(d["pots"])
    fb = Dev(lib, S * 8)
    fb.put(d["occ"])
    kk = Dev(lib, 2 * S * 8)
    kk.zero()
    cnt = Dev(lib, S * 4)
    cnt.put(np.ones(S, dtype=np.int32))
    ws = ctypes.c_size_t()
    assert lib.create_cufftPlans(2 * S, S, ctypes.byref(ws)) == 0
    work = Dev(lib, max(ws.value, 11 * N * 8 + 64))
    assert lib.set_workspace_for_cufftPlan(work.p) == 0
    const_mass = proj.const_mass
    scheme = AB[nh]

    def dens_call(g):
        if cd == 3:
            r = lib.calculate_densities(S, wf.p, dx.p, dy.p, dz.p, lap.p, fb.p, None, dens.p, g, 512)
        elif cd == 2:
            r = lib.calculate_densities(S, wf.p, dx.p, dy.p, lap.p, kk.p, fb.p, None, dens.p, g, 512)
        else:
            r = lib.calculate_densities(S, wf.p, dx.p, lap.p, kk.p, fb.p, None, cnt.p, dens.p, g, 512)
        assert r == 0, r

    def h_call(it, out):
        qf = ctypes.c_double(0.0)
        if cd == 3:
            r = lib.apply_hamiltonian(it, S, wf.p, out.p, dx.p, dy.p, dz.p, lap.p, alap.p, dens.p, pots.p, qf, None, qf, 512)
        elif cd == 2:
            r = lib.apply_hamiltonian(it, S, wf.p, out.p, dx.p, dy.p, kk.p, lap.p, alap.p, dens.p, pots.p, qf, None, qf, 512)
        else:
            r = lib.apply_hamiltonian(it, S, wf.p, out.p, dx.p, kk.p, lap.p, alap.p, dens.p, pots.p, qf, None, qf, 512)
        assert r == 0, r

    def derivs(g):
        if g:
            assert lib.compute_derivatives(2 * S, wf.p, dx.p, dy.p, dz.p, lap.p, 512) == 0
        else:
            assert lib.compute_laplace(2 * S, wf.p, lap.p, 512) == 0

    def half(it1, g):
        derivs(g)
        dens_call(g)
        if g:
            assert lib.density_caculate_tau(dens.p, 512) == 0
        assert lib.compute_potentials(it1, dens.p, pots.p, ctypes.c_double(1.0), 512) == 0
        if not const_mass:
            assert lib.multiply_wf_by_alpha(S, wf.p, alap.p, pots.p, 512) == 0
            assert lib.compute_laplace(2 * S, alap.p, alap.p, 512) == 0

    # initial measurement (pca.c:939-958)
    assert lib.normalize_wf(S, wf.p, 512) == 0
    derivs(1)
    dens_call(1)
    assert lib.density_caculate_tau(dens.p, 512) == 0
    it = 0
    for _ in range(nmeas):
        for s in range(nsteps):
            fp = [x.p for x in f] + [None] * (5 - nh)
            assert lib.abm_step1(S, wf.p, *fp, scheme, 512) == 0
            assert lib.normalize_wf(S, wf.p, 512) == 0
            half(it + 1, 0 if const_mass else 1)
            h_call(it + 1, lap)
            assert lib.abm_step4(S, lap.p, wf.p, f[nh - 1].p, scheme, 512) == 0
            assert lib.normalize_wf(S, wf.p, 512) == 0
            half(it + 1, 1 if (not const_mass or s == nsteps - 1) else 0)
            f = [f[nh - 1]] + f[: nh - 1]
            h_call(it + 1, f[0])
            it += 1
    qpe = work.get(np.float64, S)
    assert lib.compute_energy(it, dens.p, pots.p, work.p, 512) == 0
    out = dict(states=wf.get(np.complex128, M), densities=dens.get(np.float64, 12 * N),
               potentials=pots.get(np.float64, 12 * N), energy=work.get(np.float64, 11), qpe=qpe,
               history0=f[0].get(np.complex128, M))
    for x in [wf, dx, dy, dz, lap, alap, dens, pots, fb, kk, cnt, work] + f + ([extra] if extra else []):
        x.free()
    return out


SMALL = ["t1d_custom", "t1d_aslda", "t2d_slda", "t2d_bdg", "t3d_slda", "t3d_aslda", "c1_bdg1d", "c4_bdg2d",
         "c2_slda2d", "c3_aslda3d", "c5_slda3d", "t2d_vext", "t1d_bdg_vext", "t2d_big", "t2d_sldae", "t3d_sldae",
         "t1d_sldae_a1", "t2d_aslda_sym", "t3d_sldae_a1_sym", "t1d_bdg_sym"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", SMALL)
def test_compat_abi_matches_reference_golden(has_gpu, name):
    g = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    nwf, nsteps, nmeas = int(g["nwf"]), int(g["nsteps"]), int(g["nmeas"])
    o = run_compat(name, nwf, nsteps, nmeas)
    dens, pots = o["densities"], o["potentials"]
    if "points" in g.files:
        dens = dens.reshape(12, -1)[:, g["points"]].reshape(-1)
        pots = pots.reshape(12, -1)[:, g["points"]].reshape(-1)
    for k, v in density_errors(dens, g["densities"], dens.size // 12).items():
        assert v < TOL, f"{name}: density {k} rel err {v:.3e}"
    assert rel(pots, g["potentials"]) < TOL
    for k in range(11):
        if abs(g["energy"][k]) > 1e-12:
            assert abs(o["energy"][k] - g["energy"][k]) / abs(g["energy"][k]) < TOL, (k, o["energy"][k], g["energy"][k])
    assert rel(o["qpe"], g["qpe"]) < TOL
    if "states" in g.files:
        assert rel(o["states"], g["states"]) < TOL
        assert rel(o["history0"], g["history0"]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["t1d_aslda", "t2d_slda", "t3d_aslda", "c3_aslda3d"])
def test_compat_high_k_filters(has_gpu, name):
    """high_frequency_filter_{d,massive_d,c} (pca_derivative.cu:829-963) against the oracle's
    filter, in place and out of place, on the fused-size and the plane/pencil (32^3) lattices"""
    from oracle_lib import Oracle
    from wslda_b200 import load_library
    from wslda_b200.projects import Project
    proj = Project(name)
    N = proj.numel
    lib = load_library(name)
    for fn in ("gpu_malloc", "gpu_free", "memcopy_host2gpu", "memcopy_gpu2host"):
        getattr(lib, fn).restype = ctypes.c_int
    lib.high_frequency_filter_massive_d.argtypes = [ctypes.c_int, VP, VP, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.high_frequency_filter_d.argtypes = [VP, VP, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.high_frequency_filter_c.argtypes = [VP, VP, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    emax = 0.5 * np.pi ** 2 / proj.dx ** 2
    mu, T = 0.35 * emax, 0.04 * emax
    o = Oracle(name)
    o.set_high_k_filter(1, mu, T)
    rng = np.random.default_rng(11)
    f = rng.standard_normal((3, N))
    want = np.stack([o.filter_field(f[k]) for k in range(3)])
    src, dst = Dev(lib, f.nbytes), Dev(lib, f.nbytes)
    src.put(f)
    assert lib.high_frequency_filter_massive_d(3, src.p, dst.p, mu, T, 512) == 0
    got = dst.get(np.float64, 3 * N).reshape(3, N)
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(f))
    assert np.array_equal(src.get(np.float64, 3 * N).reshape(3, N), f)  # input untouched
    assert lib.high_frequency_filter_d(src.p, src.p, mu, T, 512) == 0  # in place, first field
    assert np.max(np.abs(src.get(np.float64, N) - want[0])) < 1e-12 * np.max(np.abs(f))
    # complex field: the filter is real and even in k, so it acts on Re and Im separately
    z = f[1] + 1j * f[2]
    zs, zd = Dev(lib, z.nbytes), Dev(lib, z.nbytes)
    zs.put(z)
    assert lib.high_frequency_filter_c(zs.p, zd.p, mu, T, 512) == 0
    zg = zd.get(np.complex128, N)
    assert np.max(np.abs(zg - (want[1] + 1j * want[2]))) < 1e-12 * np.max(np.abs(f))
    o.set_high_k_filter(0, 0.0, 1.0)
    for x in (src, dst, zs, zd):
        x.free()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["t1d_aslda", "t2d_slda", "t3d_aslda", "c4_bdg2d", "t2d_aslda_sym", "t1d_bdg_sym"])
def test_compat_quantum_friction_densities(has_gpu, name):
    """calculate_quantum_friction_densities (pca_dens.cu:431 and the 2D/1D forms) against the
    oracle on the normalised initial states"""
    from oracle_lib import Oracle
    from wslda_b200 import load_library
    proj, d = inputs(name, 16)
    N, S = proj.numel, 16
    o = Oracle(name)
    o.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    o.initial_measurement()
    want = o.qf_densities()
    y = o.states()
    lib = load_library(name)
    for fn in ("gpu_malloc", "gpu_free", "memcopy_host2gpu", "memcopy_gpu2host", "create_cufftPlans"):
        getattr(lib, fn).restype = ctypes.c_int
    wf, lap, fb, qf = Dev(lib, y.nbytes), Dev(lib, y.nbytes), Dev(lib, S * 8), Dev(lib, 4 * N * 8)
    wf.put(y)
    fb.put(np.ascontiguousarray(d["occ"], dtype=np.float64))
    assert lib.compute_laplace(2 * S, wf.p, lap.p, 512) == 0
    if proj.codedim == 3:
        rc = lib.calculate_quantum_friction_densities(S, wf.p, lap.p, fb.p, None, qf.p, 512)
    elif proj.codedim == 2:
        kk = Dev(lib, S * 8)
        kk.put(np.zeros(S))
        rc = lib.calculate_quantum_friction_densities(S, wf.p, lap.p, kk.p, fb.p, None, qf.p, 512)
    else:
        kk, cnt = Dev(lib, 2 * S * 8), Dev(lib, S * 4)
        kk.put(np.zeros(2 * S))
        cnt.put(np.ones(S, dtype=np.int32))
        rc = lib.calculate_quantum_friction_densities(S, wf.p, lap.p, kk.p, fb.p, None, cnt.p, qf.p, 512)
    assert rc == 0
    got = qf.get(np.float64, 4 * N)
    assert rel(got, want) < 1e-12, rel(got, want)
