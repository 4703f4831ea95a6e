"""The CPU oracle's own arithmetic: FFT against numpy, spectral derivatives against analytic
Gaussians (the known-answer tests of lib/wderiv/c/test-wderiv.c:91-111), conservation of the
state norm and the ABM/normalisation structure of a step."""
import numpy as np
import pytest

from oracle_lib import Oracle
from parity_util import inputs

SMALL = ["t1d_custom", "t1d_aslda", "t2d_slda", "t2d_bdg", "t3d_slda", "t3d_aslda", "t2d_sldae", "t1d_sldae_a1",
         "t2d_aslda_sym", "t1d_bdg_sym"]


@pytest.mark.parametrize("name", SMALL + ["c1_bdg1d", "c2_slda2d", "c4_bdg2d"])
def test_fft_matches_numpy(name):
    o = Oracle(name)
    p = o.proj
    rng = np.random.default_rng(1)
    f = rng.standard_normal(p.numel) + 1j * rng.standard_normal(p.numel)
    shape = p.dims[: p.codedim]
    fw = o.fft_field(f, -1)
    ref = np.fft.fftn(f.reshape(shape)).reshape(-1)
    assert np.abs(fw - ref).max() / np.abs(ref).max() < 1e-14
    bw = o.fft_field(fw, +1)
    assert np.abs(bw / p.numel - f).max() < 1e-14


@pytest.mark.parametrize("name", ["c1_bdg1d", "c2_slda2d", "c4_bdg2d"])
def test_spectral_derivatives_of_gaussian(name):
    """d/dx_d and laplacian of a periodic-enough Gaussian against the analytic result."""
    o = Oracle(name)
    p = o.proj
    axes = [(np.arange(n) - n // 2) * d for n, d in zip(p.dims, (p.dx, p.dy, p.dz))][: p.codedim]
    grids = np.meshgrid(*axes, indexing="ij")
    width = min(p.dims[: p.codedim]) / 16.0 * max(p.dx, 1.0)
    r2 = sum(g * g for g in grids)
    f = np.exp(-r2 / (2 * width ** 2)) * (1 + 0.5j)
    dx, dy, dz, lap = o.derivatives_field(f.reshape(-1))
    ex_dx = (-grids[0] / width ** 2 * f).reshape(-1)
    ex_lap = ((r2 / width ** 4 - p.codedim / width ** 2) * f).reshape(-1)
    assert np.abs(dx - ex_dx).max() < 5e-6 * np.abs(ex_dx).max() + 1e-9
    assert np.abs(lap - ex_lap).max() < 5e-5 * np.abs(ex_lap).max() + 1e-9


@pytest.mark.parametrize("name", SMALL)
def test_step_keeps_states_normalised(name):
    proj, d = inputs(name, 16)
    o = Oracle(name)
    o.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    o.initial_measurement()
    o.steps(3)
    y = o.states().reshape(2, 16, proj.numel)
    norms = (np.abs(y[0]) ** 2 + np.abs(y[1]) ** 2).sum(1) * proj.dv
    assert np.allclose(norms, 1.0, atol=1e-13)
    e = o.energy()
    assert np.all(np.isfinite(e))
    dens = o.densities()
    n = proj.numel
    # particle number: sum of rho over the lattice, times dV, equals the energy slots 7, 8
    assert abs(dens[2 * n:3 * n].sum() * {1: proj.dx, 2: proj.dx * proj.dy, 3: proj.dv}[proj.codedim] - e[7]) < 1e-10 * max(1, abs(e[7]))
    assert o.lib.orc_get_it() == 3


@pytest.mark.parametrize("project", ["t1d_aslda", "t2d_slda", "t3d_aslda"])
def test_oracle_high_k_filter_matches_numpy(project):
    """the oracle's Fermi-Dirac filter (high_frequency_filter_d) against numpy's FFT"""
    from oracle_lib import Oracle
    from wslda_b200.projects import Project
    proj = Project(project)
    o = Oracle(project)
    dims = proj.dims[:proj.codedim]
    spacing = [proj.dx, proj.dy, proj.dz][:proj.codedim]
    rng = np.random.default_rng(7)
    f = rng.standard_normal(proj.numel)
    emax = 0.5 * np.pi ** 2 / proj.dx ** 2
    mu, T = 0.35 * emax, 0.04 * emax
    o.set_high_k_filter(1, mu, T)
    got = o.filter_field(f)
    o.set_high_k_filter(0, 0.0, 1.0)
    ks = [2 * np.pi * np.fft.fftfreq(n, d=h) for n, h in zip(dims, spacing)]
    # the reference counts the Nyquist mode as -pi/dx; k^2 is the same either way
    grids = np.meshgrid(*ks, indexing="ij")
    ek = 0.5 * sum(k ** 2 for k in grids)
    w = 1.0 / (np.exp((ek - mu) / T) + 1.0)
    want = np.fft.ifftn(np.fft.fftn(f.reshape(dims)) * w).real.reshape(-1)
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(f))
    # a very high cut-off keeps the field, a constant keeps FD(0) of itself
    o.set_high_k_filter(1, 1e6 * emax, 1e-3 * emax)
    assert np.allclose(o.filter_field(f), f, rtol=0, atol=1e-12)
    o.set_high_k_filter(1, mu, T)
    c = o.filter_field(np.full(proj.numel, 2.0))
    assert np.allclose(c, 2.0 / (np.exp(-mu / T) + 1.0), rtol=1e-13)
    o.set_high_k_filter(0, 0.0, 1.0)


@pytest.mark.parametrize("name", ["c2_slda2d", "t1d_aslda", "t3d_aslda", "c4_bdg2d"])
def test_wderiv_baseline_matches_oracle(name):
    """the host-core baseline (the reference's lib/wderiv derivatives over the in-repo FFTW-API
    shim, with the oracle's local update) reproduces the oracle's step: densities, energies and
    states after a few steps at 1e-12"""
    from oracle_lib import Oracle, wderiv_library
    from parity_util import density_errors, inputs, rel
    if wderiv_library(name) is None:
        pytest.skip("wderiv baseline not built (reference tree absent)")
    proj, d = inputs(name, 12)
    out = []
    for variant in (None, "wderiv"):
        o = Oracle(name, threads=2, variant=variant)
        o.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
        o.initial_measurement()
        o.steps(3)
        out.append((o.densities(), o.energy(), o.states()))
    (d0, e0, s0), (d1, e1, s1) = out
    for k, v in density_errors(d1, d0, proj.numel).items():
        assert v < 1e-12, (k, v)
    assert rel(e1[:9], e0[:9]) < 1e-12
    assert rel(s1, s0) < 1e-12
