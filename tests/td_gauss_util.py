"""Replay of the reference testsuite's td-gauss runs (testsuite/td-gauss-*/) through the library.

A td-gauss run starts from the reference's uniform solution (inittype 0: pca.c:257-330,
cpca.c:258-325, ccpca.c): plane-wave quasiparticle states with BCS amplitudes u_k, v_k and
occupations f = fbeta(E_k, beta), uniform potentials V_a, V_b, Delta.  It then evolves
`measurements` blocks of `timesteps` steps under a time-dependent Gaussian stirrer and logs N_a,
N_b and the energy terms after every block (the .wlog file; the final values in the .cmp file).

The fixtures under tests/golden/td_gauss/ (made by tests/golden/make_td_gauss.py) hold the
uniform solution that the reference's own solver gives for the case, each state's plane wave
and amplitudes, and the reference's logged trajectory.  This module rebuilds the initial
states exactly as the reference's create_uniform_wf / _2d / _1d do (pca_uniform.h:636-851,
2044-2296, 2321-2572) and runs the trajectory through the library's C ABI with the reference
driver's order of operations (pca.c:882-1000, 1397-1600).
"""
import os

import numpy as np

from wslda_b200 import projects as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "td_gauss")
# wlog columns (pca.c:1590): time*eF, Na, Nb, Na+Nb, Etot/Effg, EKIN..EVELEXT / Effg
WLOG_COLUMNS = ("time_eF", "Na", "Nb", "N", "Etot", "EKIN", "EPOT", "EPAIR", "ECURRENT", "EPOTEXT",
                "EPAIREXT", "EVELEXT")


def fixtures():
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load(case):
    return dict(np.load(os.path.join(GOLDEN, f"{case}.npz")))


def lattice_k(n, L):
    """k values of one axis in the reference's order (pca_uniform.h:652-676): 2 pi / L * j,
    j = 0..n/2-1 then -n/2..-1"""
    j = np.concatenate([np.arange(0, n // 2), np.arange(-(n // 2), 0)]).astype(np.float64)
    return 2. * np.pi / L * j


def fbeta(E, beta):
    """occupation 1/(exp(beta E) + 1) with the reference's cut-offs at |beta E| > 50
    (pca_uniform.h:70-76)"""
    bE = beta * np.asarray(E, dtype=np.float64)
    with np.errstate(over="ignore"):
        f = 1.0 / (np.exp(np.clip(bE, -60, 60)) + 1.0)
    return np.where(bE > 50., 0.0, np.where(bE < -50., 1.0, f))


def initial_states(proj, fx):
    """[u_0..u_{S-1}, v_0..v_{S-1}] of the uniform solution: u_n(r) = u_k e^{i k.r} / sqrt(V),
    v_n(r) = v_k e^{i k.r} / sqrt(V) with k the plane wave of state n over the engine's own
    axes (x, y, z in 3D; x, y in 2D; x in 1D) and V the engine's volume (LXYZ, LXY, LX)"""
    d = int(fx["codedim"])
    nx, ny, nz = proj.nx, proj.ny, proj.nz
    dx, dy, dz = proj.dx, proj.dy, proj.dz
    kx, ky, kz = lattice_k(nx, dx * nx), lattice_k(ny, dy * ny), lattice_k(nz, dz * nz)
    ix = np.arange(nx, dtype=np.float64)[:, None, None]
    iy = np.arange(ny, dtype=np.float64)[None, :, None]
    iz = np.arange(nz, dtype=np.float64)[None, None, :]
    kidx = fx["kidx"].astype(np.int64)
    S = kidx.shape[0]
    if d == 3:
        vol = (dx * nx) * (dy * ny) * (dz * nz)
        shape = (nx, ny, nz)
    elif d == 2:
        vol = (dx * nx) * (dy * ny)
        shape = (nx, ny, 1)
    else:
        vol = dx * nx
        shape = (nx, 1, 1)
    sq = np.sqrt(vol)
    out = np.zeros((2, S) + shape, dtype=np.complex128)
    for n in range(S):
        a, b, c = kidx[n]
        arg = ix * dx * kx[a]
        if d >= 2:
            arg = arg + iy * dy * ky[b]
        if d == 3:
            arg = arg + iz * dz * kz[c]
        ph = np.exp(1j * np.broadcast_to(arg, np.broadcast_shapes(arg.shape, shape)))
        ph = ph.reshape(shape)
        out[0, n] = ph * fx["uk"][n] / sq
        out[1, n] = ph * fx["vk"][n] / sq
    return out.reshape(-1)


def case_inputs(proj, fx):
    """states, potentials, occupations, transverse momenta and constants of the run's start"""
    n0 = float(fx["meta"][0] + fx["meta"][1])
    meta = fx["meta"]
    S = int(fx["nwf"])
    N = proj.numel
    pots = np.zeros(12 * N)
    pots[0:N] = meta[4]                 # V_a
    pots[N:2 * N] = meta[5]             # V_b
    pots[2 * N:4 * N:2] = meta[9]       # Re Delta
    pots[4 * N:6 * N] = 1.0             # alpha_a, alpha_b (reset_potentials, wslda_potdens.c:76-98)
    kF = (3.0 * np.pi * np.pi * n0) ** (1.0 / 3.0)
    eF = (3.0 * np.pi * np.pi * n0) ** (2.0 / 3.0) / 2.0
    lxyz = (proj.dx * proj.nx) * (proj.dy * proj.ny) * (proj.dz * proj.nz)
    effg = 0.6 * n0 * eF * lxyz
    kky = kkz = cnt = None
    d = int(fx["codedim"])
    if d == 2:
        kkz = fx["kperp"][:S]
    elif d == 1:
        kky, kkz = fx["kperp"][:S], fx["kperp"][S:2 * S]
        cnt = fx["cnt"]
    return dict(states=initial_states(proj, fx), pots=pots, occ=fbeta(fx["En"], float(meta[10])),
                kky=kky, kkz=kkz, cnt=cnt, kF=kF, eF=eF, effg=effg, mu_a=float(meta[2]), mu_b=float(meta[3]),
                ec=float(meta[8]), sclgth=float(meta[11]))


def prepare(fx, hook):
    """the run's start (case_inputs) plus params and constants after the user's process_params
    hook(params, kF[1], mu[2]) and the driver's eF = kF^2/2, dt = dt_input / eF (pca.c:903-906)"""
    proj = P.Project(str(fx["project"]))
    ci = case_inputs(proj, fx)
    params = np.zeros(32)
    params[:fx["params"].size] = fx["params"]
    kF = np.array([ci["kF"]])
    mu = np.array([ci["mu_a"], ci["mu_b"]])
    hook(params, kF, mu)
    eF = 0.5 * kF[0] * kF[0]
    dt = float(fx["dt_eF"]) / eF
    const = dict(mu_a=mu[0], mu_b=mu[1], ec=ci["ec"], t0=0.0, dt=dt, kF=kF[0], sclgth=ci["sclgth"])
    return proj, ci, params, const, eF


def energy_row(e, t_eF, effg):
    """one log row from the 11 energy items: [time*eF, Na, Nb, Na+Nb, Etot/Effg, EKIN/Effg, ...,
    EVELEXT/Effg] (pca.c:1590)"""
    na, nb = e[P_NPARTA], e[P_NPARTB]
    return [t_eF, na, nb, na + nb, e[:7].sum() / effg, *(e[:7] / effg)]


def replay(case, measurements=None, fx=None, backend="gpu", steps_per_block=None):
    """run the case; returns (rows, reference rows) of energy_row.  backend "gpu" is the
    library (TDRun over the C ABI), "oracle" the CPU restatement; steps_per_block overrides
    the block length."""
    fx = load(case) if fx is None else fx
    name = str(fx["project"])
    S = int(fx["nwf"])
    nmeas = int(fx["measurements"]) if measurements is None else int(measurements)
    block = int(fx["timesteps"]) if steps_per_block is None else int(steps_per_block)
    if backend == "gpu":
        from wslda_b200 import TDRun
        r = TDRun(name, S)
        hook = lambda pr, k, m: r._check(r.lib.wtd_process_params(r.h, pr.ctypes.data_as(_dp()),  # noqa: E731
                                                                  k.ctypes.data_as(_dp()), m.ctypes.data_as(_dp())))
    else:
        from oracle_lib import Oracle
        r = Oracle(name)
        hook = r.process_params
    proj, ci, params, const, eF = prepare(fx, hook)
    r.setup(ci["states"], ci["pots"], ci["occ"], params, const=const, kky=ci["kky"], kkz=ci["kkz"], cnt=ci["cnt"])
    if backend == "gpu":
        r.initial_measurement(0)
    else:
        r.initial_measurement()
    rows = [energy_row(r.energy(), 0.0, ci["effg"])]
    it = 0
    for _ in range(nmeas):
        r.steps(block)
        it += block
        rows.append(energy_row(r.energy(), it * const["dt"] * eF, ci["effg"]))
    if backend == "gpu":
        r.close()
    ref = fx["wlog"][: nmeas + 1, 1:13]
    return np.array(rows), ref


P_NPARTA, P_NPARTB = 7, 8


def _dp():
    import ctypes
    return ctypes.POINTER(ctypes.c_double)
