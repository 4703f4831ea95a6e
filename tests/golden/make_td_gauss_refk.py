"""Trajectories of the td-gauss replay cases under the reference's current kernels (run on a B200).

Loads oracle/_ref/<project>/libref.so (hpc-engine/*.cu compiled unmodified for sm_100a plus
oracle/ref_harness.cu, built in the build container by `make -C oracle ref PROJECT=<p>`),
starts it from the uniform-solution state of tests/golden/td_gauss/<case>.npz exactly as
tests/td_gauss_util starts the library, and records the 11 energy items after the initial
measurement and after every measurement block (refh_set_energy_log).

The reference's published logs (testsuite/td-gauss-*/ref/*.wlog.ref) come from its 2021.11.06
version.  Its changelog records two later fixes to the current terms of the variable-mass
(A != 1) functionals, ASLDA and SLDAE (2026.08.20: "current corrections to the evolution
Hamiltonian"; 2026.09.25: "current-dependent mean fields").  These fixtures give the current
reference's own trajectory for every case, so the library is pinned to it where the 2021 log
no longer applies.

    python tests/golden/make_td_gauss_refk.py --out <folder> [--measurements M] [case ...]

The 1D and 2D fixtures hold all 100 blocks; the 3D ones the first 20 (5,720 steps, 11,440 for
SLDAE), which covers the ramp-up of the stirrer, to bound the reference's run time.
"""
import argparse
import ctypes
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))
from td_gauss_util import energy_row, fixtures, load, prepare  # noqa: E402

_dp = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def run_reference(case, measurements=None):
    from oracle_lib import Oracle
    fx = load(case)
    name = str(fx["project"])
    proj, ci, params, const, eF = prepare(fx, Oracle(name).process_params)
    so = os.path.join(REPO, "oracle", "_ref", name, "libref.so")
    if not os.path.exists(so):
        import subprocess
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"PROJECT={name}"], check=True)
    lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    for fn in ("refh_set_hkf", "refh_set_selfstart", "refh_set_quantum_friction", "refh_set_energy_log"):
        getattr(lib, fn).restype = ctypes.c_int
    lib.refh_set_hkf.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
    lib.refh_set_hkf(0, 0.0, 1.0)
    lib.refh_set_selfstart.argtypes = [ctypes.c_int]
    lib.refh_set_selfstart(0)
    lib.refh_set_quantum_friction.argtypes = [ctypes.c_double] * 7
    lib.refh_set_quantum_friction(*(0.0,) * 7)
    S, nmeas, block = int(fx["nwf"]), int(fx["measurements"]), int(fx["timesteps"])
    if measurements:
        nmeas = min(nmeas, int(measurements))
    elog = np.zeros(11 * (nmeas + 1))
    lib.refh_set_energy_log.argtypes = [_dp]
    lib.refh_set_energy_log(_p(elog))
    lib.refh_run.argtypes = ([ctypes.c_int] + [_dp] * 5 + [ctypes.POINTER(ctypes.c_int)] + [ctypes.c_double] * 7 +
                             [_dp, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_dp] * 7)
    y0 = np.ascontiguousarray(ci["states"])
    cnt = None if ci["cnt"] is None else np.ascontiguousarray(ci["cnt"], dtype=np.int32)
    kky = None if ci["kky"] is None else np.ascontiguousarray(ci["kky"])
    kkz = None if ci["kkz"] is None else np.ascontiguousarray(ci["kkz"])
    ms = np.zeros(1)
    t = time.time()
    rc = lib.refh_run(S, _p(y0.view(np.float64)), _p(ci["pots"]), _p(np.ascontiguousarray(ci["occ"])), _p(kky), _p(kkz),
                      None if cnt is None else cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                      const["mu_a"], const["mu_b"], const["ec"], const["t0"], const["dt"], const["kF"], const["sclgth"],
                      _p(params), None, 0, block, nmeas, 0, None, None, None, None, None, None, _p(ms))
    lib.refh_set_energy_log(None)
    if rc != 0:
        raise RuntimeError(f"{case}: refh_run returned {rc}")
    e = elog.reshape(nmeas + 1, 11)
    rows = np.array([energy_row(e[m], m * block * const["dt"] * eF, ci["effg"]) for m in range(nmeas + 1)])
    return rows, ms[0], time.time() - t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "td_gauss_refk"))
    ap.add_argument("--measurements", type=int, default=0, help="first blocks only (the 3D runs)")
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for case in a.cases or fixtures():
        rows, ms, wall = run_reference(case, a.measurements)
        ref = load(case)["wlog"][: rows.shape[0], 1:13]
        dev = np.abs(rows - ref)[:, 1:].max()
        np.savez_compressed(os.path.join(a.out, f"{case}.npz"), rows=rows, ms_per_step=np.float64(ms))
        print(f"{case}: {ms:.3f} ms/step, {wall:.1f} s, max |current reference - 2021 log| = {dev:.3e}", flush=True)


if __name__ == "__main__":
    main()
