"""Shared helpers of the parity tests: seeded inputs, oracle and CUDA runs, error measures."""
import numpy as np

from wslda_b200 import projects as P

DENS_BLOCKS = ["nu", "rho_a", "tau_a", "j_a_x", "j_a_y", "j_a_z", "rho_b", "tau_b", "j_b_x", "j_b_y", "j_b_z"]


def inputs(name, nwf, seed_salt=0):
    proj = P.Project(name)
    seed = P.config_seed(name, seed_salt)
    y0 = P.make_states(proj, nwf, seed)
    occ = P.make_occupations(nwf)
    pots = P.make_potentials(proj)
    params = P.stirrer_params(proj, seed) if proj.cfg.get("stirrer_params") else proj.params
    extra = P.make_extra(proj, seed)
    return proj, dict(states=y0, pots=pots, occ=occ, params=params, extra=extra)


def run_oracle(name, nwf, nsteps, nmeas=1, inp=None, threads=None, hkf=None, selfstart=False, qf=None):
    from oracle_lib import Oracle
    proj, d = inputs(name, nwf) if inp is None else (P.Project(name), inp)
    o = Oracle(name, threads=threads)
    if hkf is not None:
        o.set_high_k_filter(*hkf)
    if qf is not None:
        o.set_quantum_friction(*qf)
    o.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    o.initial_measurement()
    if selfstart:
        o.selfstart()
    for _ in range(nmeas):
        o.steps(nsteps)
    return dict(states=o.states(), densities=o.densities(), potentials=o.potentials(), energy=o.energy(),
                qpe=o.qpe(), history=[o.history(s) for s in range(proj.nhist)])


def run_gpu(name, nwf, nsteps, nmeas=1, precision=0, inp=None, hkf=None, selfstart=False, qf=None):
    from wslda_b200 import TDRun
    proj, d = inputs(name, nwf) if inp is None else (P.Project(name), inp)
    r = TDRun(name, nwf, precision=precision)
    if hkf is not None:
        r.set_high_k_filter(*hkf)
    if qf is not None:
        r.set_quantum_friction(*qf)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    r.initial_measurement()
    if selfstart:
        r.selfstart()
    for _ in range(nmeas):
        r.steps(nsteps)
    out = dict(states=r.states(), densities=r.densities(), potentials=r.potentials(), energy=r.energy(),
               qpe=r.qpe(), history0=r.history(0), launches=r.launches())
    r.close()
    return out


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def density_errors(d, ref, n):
    """relative L2 error per density block (nu is complex: 2n words)"""
    out = {}
    offs = [(0, 2 * n)] + [((2 + k) * n, (3 + k) * n) for k in range(10)]
    for name, (a, b) in zip(DENS_BLOCKS, offs):
        if np.linalg.norm(ref[a:b]) > 0:
            out[name] = rel(d[a:b], ref[a:b])
    return out
