"""Generate golden vectors from the REFERENCE's own CUDA kernels (run on a B200).

Loads oracle/_ref/<project>/libref.so (hpc-engine/*.cu compiled unmodified for sm_100a plus
oracle/ref_harness.cu, built in the build container by `make -C oracle ref PROJECT=<p>`),
regenerates the seeded inputs of wslda_b200.projects, runs the reference's time loop and
saves the outputs as tests/golden/<project>.npz.  The fixtures pin the CPU oracle
(tests/test_oracle_golden.py) and the CUDA library (tests/test_gpu_parity.py).

    python tests/golden/make_golden.py --out <folder> [project ...]
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from wslda_b200 import projects as P  # noqa: E402

# (project, nwf, steps per measurement, measurements, store full states?)
CASES = {
    "t1d_custom": (24, 3, 2, True),
    "t1d_aslda": (24, 3, 2, True),
    "t2d_slda": (24, 3, 2, True),
    "t2d_bdg": (24, 3, 2, True),
    "t3d_slda": (24, 3, 2, True),
    "t3d_aslda": (24, 3, 2, True),
    "c1_bdg1d": (256, 100, 1, False),
    "c2_slda2d": (16, 4, 1, False),
    "c3_aslda3d": (8, 2, 1, False),
    "c4_bdg2d": (16, 4, 1, False),
    "c5_slda3d": (4, 2, 1, False),
    "t2d_vext": (24, 3, 2, True),
    "t1d_bdg_vext": (24, 3, 2, True),
    "t2d_big": (8, 3, 1, False),
    "t2d_sldae": (24, 3, 2, True),
    "t3d_sldae": (24, 3, 2, True),
    "t1d_sldae_a1": (24, 3, 2, True),
    "t2d_aslda_sym": (24, 3, 2, True),
    "t3d_sldae_a1_sym": (24, 3, 2, True),
    "t1d_bdg_sym": (24, 3, 2, True),
}

# effective-mass filter cases (pca.c:1448-1453, hkf_mode 1): the same runs with alpha_a,
# alpha_b filtered by FD(k^2/2; mu, T) after every functional evaluation; mu and T as fractions
# of E_max = pi^2 / (2 dx^2), as the reference's input gives them (pca.c:183-185)
HKF_CASES = {
    "t1d_aslda": (24, 3, 2, True),
    "t3d_aslda": (24, 3, 2, True),
    "c3_aslda3d": (8, 2, 1, False),
}
HKF_FRACTIONS = (0.35, 0.04)
# hkf_mode 2 also filters the pairing field (apply_hamiltonian, pca_kernels.cu:758-762)
HKF2_CASES = {
    "t2d_slda": (24, 3, 2, True),
    "t3d_aslda": (24, 3, 2, True),
}


# Taylor self-start of the history (pca.c:1086-1330, selfstart 1) before the steps
SS_CASES = {
    "t2d_slda": (24, 3, 2, True),
    "t1d_aslda": (24, 3, 2, True),
    "c4_bdg2d": (16, 4, 1, False),
    "c3_aslda3d": (8, 2, 1, False),
}


# quantum friction (pca.c:1405-1430, 1458) switched on over the run: input qfalpha, qfbeta,
# qfgamma, qfNreq and qfstart, qfstop, qfswitch (in 1/eF)
QF_CASES = {
    "t2d_slda": (24, 3, 2, True),
    "t1d_aslda": (24, 3, 2, True),
    "c4_bdg2d": (16, 4, 1, False),
    "t3d_aslda": (24, 3, 2, True),
    "t2d_aslda_sym": (24, 3, 2, True),
    "t1d_bdg_sym": (24, 3, 2, True),
    "c3_aslda3d": (8, 2, 1, False),
    "t2d_big": (8, 3, 1, False),
}
QF_PARAMS = (0.5, 0.3, 0.2, 10.0, 0.0, 100.0, 0.02)


def hkf_params(proj, mode=1):
    emax = 0.5 * np.pi ** 2 / proj.dx ** 2
    return mode, HKF_FRACTIONS[0] * emax, HKF_FRACTIONS[1] * emax




def fixture_suffix(hkf):
    return {0: "", 1: "_hkf", 2: "_hkf2"}[hkf]


_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def case_inputs(name, nwf):
    proj = P.Project(name)
    seed = P.config_seed(name)
    y0 = P.make_states(proj, nwf, seed)
    occ = P.make_occupations(nwf)
    pots = P.make_potentials(proj)
    params = P.stirrer_params(proj, seed) if proj.cfg.get("stirrer_params") else proj.params
    extra = P.make_extra(proj, seed)
    return proj, y0, occ, pots, params, extra


def state_moments(y, nwf, n):
    """Per-state checksums: norm of u, norm of v, sum of u weighted by a fixed ramp."""
    a = y.reshape(2, nwf, n)
    ramp = np.linspace(-1.0, 1.0, n)
    return np.stack([np.sum(np.abs(a[0]) ** 2, 1), np.sum(np.abs(a[1]) ** 2, 1),
                     (a[0] @ ramp).real, (a[0] @ ramp).imag, (a[1] @ ramp).real, (a[1] @ ramp).imag], 1)


MAX_POINTS = 2048


def point_sample(n):
    """Lattice points kept for fields of large lattices (fixed, seeded, sorted)."""
    if n <= MAX_POINTS:
        return np.arange(n)
    return np.sort(np.random.Generator(np.random.PCG64(12345)).choice(n, MAX_POINTS, replace=False))


def slim(rec, n):
    """Keep the 12 density and 12 potential blocks only at point_sample(n) for large lattices."""
    idx = point_sample(n)
    if idx.size == n:
        return rec
    for key in ("densities", "potentials"):
        blocks = rec[key].reshape(12, n)
        rec[key] = np.ascontiguousarray(blocks[:, idx]).reshape(-1)
    rec["points"] = idx
    return rec


def run_case(name, out_dir, hkf=0, selfstart=False, qf=False):
    table = QF_CASES if qf else SS_CASES if selfstart else {0: CASES, 1: HKF_CASES, 2: HKF2_CASES}[hkf]
    nwf, nsteps, nmeas, full = table[name]
    proj, y0, occ, pots, params, extra = case_inputs(name, nwf)
    so = os.path.join(REPO, "oracle", "_ref", name, "libref.so")
    lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    lib.refh_set_hkf.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
    mode, mu, T = hkf_params(proj, hkf) if hkf else (0, 0.0, 1.0)
    lib.refh_set_hkf(mode, mu, T)
    lib.refh_set_selfstart.argtypes = [ctypes.c_int]
    lib.refh_set_selfstart(1 if selfstart else 0)
    lib.refh_set_quantum_friction.argtypes = [ctypes.c_double] * 7
    lib.refh_set_quantum_friction(*(QF_PARAMS if qf else (0.0,) * 7))
    lib.refh_numel.restype = ctypes.c_int
    lib.refh_nhist.restype = ctypes.c_int
    n = lib.refh_numel()
    nh = lib.refh_nhist()
    assert n == proj.numel
    c = proj.constants()
    lib.refh_run.argtypes = ([ctypes.c_int] + [_dp] * 5 + [ctypes.POINTER(ctypes.c_int)] + [ctypes.c_double] * 7 +
                             [_dp, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_dp] * 7)
    M = 2 * nwf * n
    y = np.zeros(M, dtype=np.complex128)
    dens = np.zeros(12 * n)
    potso = np.zeros(12 * n)
    en = np.zeros(11)
    qpe = np.zeros(nwf)
    hist = np.zeros(nh * M, dtype=np.complex128)
    ms = np.zeros(1)
    ex = np.ascontiguousarray(extra)
    rc = lib.refh_run(nwf, _p(y0.view(np.float64)), _p(pots), _p(occ), None, None, None,
                      c["mu_a"], c["mu_b"], c["ec"], c["t0"], c["dt"], c["kF"], c["sclgth"],
                      _p(np.ascontiguousarray(params)), ex.ctypes.data if ex.size else None, ex.nbytes,
                      nsteps, nmeas, 0, _p(y.view(np.float64)), _p(dens), _p(potso), _p(en), _p(qpe),
                      _p(hist.view(np.float64)), _p(ms))
    if rc != 0:
        raise RuntimeError(f"{name}: refh_run returned {rc}")
    rec = dict(nwf=nwf, nsteps=nsteps, nmeas=nmeas, densities=dens, potentials=potso, energy=en, qpe=qpe,
               input_moments=state_moments(y0, nwf, n), moments=state_moments(y, nwf, n), ms_per_step=ms[0])
    if full:
        rec["states"] = y
        rec["history0"] = hist[:M]
    if hkf:
        rec["hkf"] = np.array([mode, mu, T])
    rec = slim(rec, n)
    path = os.path.join(out_dir, f"{name}{'_qf' if qf else '_ss' if selfstart else fixture_suffix(hkf)}.npz")
    np.savez_compressed(path, **rec)
    print(f"{name}: nwf={nwf} steps={nsteps}x{nmeas} E={en[:7].sum():.12g} N={en[7]:.12g},{en[8]:.12g} "
          f"ms/step={ms[0]:.3f} -> {path}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--slim-existing", action="store_true", help="apply slim() to fixtures in --out")
    ap.add_argument("--hkf", type=int, default=0, choices=[0, 1, 2],
                    help="1: the effective-mass filter cases (HKF_CASES); 2: masses and pairing field (HKF2_CASES)")
    ap.add_argument("--selfstart", action="store_true", help="the Taylor self-start cases (SS_CASES)")
    ap.add_argument("--qf", action="store_true", help="the quantum-friction cases (QF_CASES)")
    ap.add_argument("projects", nargs="*")
    a = ap.parse_args()
    if a.slim_existing:
        for name in (a.projects or list(CASES)):
            path = os.path.join(a.out, f"{name}.npz")
            if os.path.exists(path):
                rec = dict(np.load(path))
                n = P.Project(name).numel
                if "points" not in rec:
                    np.savez_compressed(path, **slim(rec, n))
        return
    os.makedirs(a.out, exist_ok=True)
    table = QF_CASES if a.qf else SS_CASES if a.selfstart else {0: CASES, 1: HKF_CASES, 2: HKF2_CASES}[a.hkf]
    for name in (a.projects or list(table)):
        run_case(name, a.out, hkf=a.hkf, selfstart=a.selfstart, qf=a.qf)


if __name__ == "__main__":
    main()
