"""The td-gauss replay fixtures and the CPU oracle against the reference testsuite's logs.

- Each fixture's uniform solution (the reference's own solver, compiled where it lies) agrees
  with the run it replays: the log header's state count, k_F and E_FFG.
- The oracle's initial measurement, from the rebuilt uniform-solution states, reproduces the
  first log row (N_a, N_b, every energy term) within the testsuite's tolerance, for all 24 runs.
- On the 1D engine the oracle runs the first 10 measurement blocks (2,860 steps; 5,720 for
  SLDAE) and follows the reference's current kernels (tests/golden/td_gauss_refk) to 1e-9 in
  the particle numbers and 1e-10 Effg in the energies.
"""
import os

import numpy as np
import pytest

from td_gauss_util import GOLDEN, case_inputs, fixtures, load, replay
from wslda_b200 import projects as P

REFK = os.path.join(os.path.dirname(GOLDEN), "td_gauss_refk")
TESTSUITE = 1e-4


@pytest.mark.parametrize("case", fixtures())
def test_fixture_matches_log_header(case):
    fx = load(case)
    proj = P.Project(str(fx["project"]))
    ci = case_inputs(proj, fx)
    assert int(fx["nwf"]) == int(fx["ref_nwf"])
    # the header prints 6 significant digits
    assert abs(ci["kF"] / float(fx["ref_kF"]) - 1) < 5e-6
    assert abs(ci["effg"] / float(fx["ref_Effg"]) - 1) < 5e-6
    assert np.abs(ci["states"]).max() > 0 and np.all(np.isfinite(ci["states"]))


@pytest.mark.parametrize("case", fixtures())
def test_oracle_initial_measurement_matches_log(case):
    rows, log = replay(case, measurements=0, backend="oracle")
    effg = float(load(case)["ref_Effg"])
    d = np.abs(rows[0] - log[0])
    assert d[1:3].max() <= TESTSUITE, (case, d[1:3])
    assert (d[5:] * effg).max() <= TESTSUITE, (case, d[5:] * effg)


@pytest.mark.parametrize("case", [c for c in fixtures() if c.endswith("_1d")])
def test_oracle_follows_reference_kernels_1d(case):
    path = os.path.join(REFK, f"{case}.npz")
    if not os.path.exists(path):
        pytest.skip("no trajectory of the reference's kernels for this case")
    rows, _ = replay(case, measurements=10, backend="oracle")
    rk = np.load(path)["rows"][: rows.shape[0]]
    d = np.abs(rows - rk)
    assert d[:, 1:4].max() < 1e-9, (case, d[:, 1:4].max())
    assert d[:, 4:].max() < 1e-10, (case, d[:, 4:].max())
