"""Pin the CPU oracle to the reference: outputs of hpc-engine's own CUDA kernels (tests/golden,
made by tests/golden/make_golden.py on a B200) against the oracle on the same seeded inputs."""
import os

import sys
import numpy as np
import pytest

from parity_util import density_errors, inputs, rel, run_oracle
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from golden.make_golden import CASES, HKF2_CASES, HKF_CASES, QF_CASES, QF_PARAMS, SS_CASES, state_moments  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-10


def _cases():
    plain = [n for n in CASES if os.path.exists(os.path.join(GOLDEN, f"{n}.npz"))]
    hkf = [f"{n}_hkf" for n in HKF_CASES if os.path.exists(os.path.join(GOLDEN, f"{n}_hkf.npz"))]
    hkf2 = [f"{n}_hkf2" for n in HKF2_CASES if os.path.exists(os.path.join(GOLDEN, f"{n}_hkf2.npz"))]
    ss = [f"{n}_ss" for n in SS_CASES if os.path.exists(os.path.join(GOLDEN, f"{n}_ss.npz"))]
    qf = [f"{n}_qf" for n in QF_CASES if os.path.exists(os.path.join(GOLDEN, f"{n}_qf.npz"))]
    return plain + hkf + hkf2 + ss + qf


@pytest.mark.parametrize("name", _cases())
def test_oracle_matches_reference_golden(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    hkf = tuple(g["hkf"]) if "hkf" in g.files else None
    selfstart = name.endswith("_ss")
    qf = QF_PARAMS if name.endswith("_qf") else None
    name = name[:-3] if (selfstart or qf) else name.rsplit("_hkf", 1)[0]
    nwf, nsteps, nmeas = int(g["nwf"]), int(g["nsteps"]), int(g["nmeas"])
    proj, d = inputs(name, nwf)
    # the regenerated inputs are the ones the fixture was made from
    assert rel(state_moments(d["states"], nwf, proj.numel), g["input_moments"]) < 1e-12
    o = run_oracle(name, nwf, nsteps, nmeas, inp=d, hkf=None if hkf is None else (int(hkf[0]), hkf[1], hkf[2]),
                   selfstart=selfstart, qf=qf)
    if "points" in g.files:  # large lattice: fixture keeps a fixed sample of points
        idx = g["points"]
        o["densities"] = o["densities"].reshape(12, -1)[:, idx].reshape(-1)
        o["potentials"] = o["potentials"].reshape(12, -1)[:, idx].reshape(-1)
    npts = o["densities"].size // 12
    errs = density_errors(o["densities"], g["densities"], npts)
    for k, v in errs.items():
        assert v < TOL, f"{name}: density {k} rel err {v:.3e}"
    assert rel(o["potentials"], g["potentials"]) < TOL
    for k in range(11):
        if abs(g["energy"][k]) > 1e-12:
            assert abs(o["energy"][k] - g["energy"][k]) / abs(g["energy"][k]) < TOL, (name, k, o["energy"][k], g["energy"][k])
    assert rel(o["qpe"], g["qpe"]) < TOL
    assert rel(state_moments(o["states"], nwf, proj.numel), g["moments"]) < TOL
    if "states" in g.files:
        assert rel(o["states"], g["states"]) < TOL
        assert rel(o["history"][0], g["history0"]) < TOL
