"""Adjoint of the TD-BdG step (C4: 2D contact BdG with a 14-parameter moving Gaussian stirrer).

The gradient dL/dtheta of L = sum_r |Delta(r, T)|^2 dV with respect to the stirrer parameters,
from wtd_adjoint's reverse sweep, is checked against Richardson-extrapolated central finite
differences of the loss (steps h and h/2, error O(h^4); h = 1e-3 max(1, |theta|) keeps the
loss's rounding noise, ~1e-16 L / h, far below the gradient):
  - of the CUDA forward itself (the same library, loss-only calls),
  - of the CPU oracle's forward (an independent implementation of the step),
to a relative tolerance of 1e-6, with several checkpoint intervals (segments of 1, 3 and all
steps, a partial last segment included).  The same gradient is also taken through the
torch.autograd.Function of tests/adjoint_autograd.py, alone and inside a composite loss.
"""
import numpy as np
import pytest

from parity_util import inputs, rel

PROJ = "c4_bdg2d"
NWF = 32
NSTEPS = 7
# the oracle check runs a longer horizon: the gradient grows with it, while the two forwards'
# rounding differences (which the finite differences divide by h) do not
NSTEPS_ORACLE = 20
NPARAM = 14
TOL = 1e-6


def _fd_step(theta):
    return 1e-3 * max(1.0, abs(theta))


def _richardson_fd(loss_at, th, j):
    """(4 D(h/2) - D(h)) / 3 with D the central difference of loss_at in parameter j"""
    def central(h):
        vals = []
        for sgn in (+1, -1):
            tp = th.copy()
            tp[j] += sgn * h
            vals.append(loss_at(tp))
        return (vals[0] - vals[1]) / (2 * h)
    h = _fd_step(th[j])
    return (4.0 * central(h / 2) - central(h)) / 3.0


def _loss_from_pots(pots, n, dv, mask=None):
    d = pots[2 * n: 4 * n].reshape(n, 2)
    a2 = d[:, 0] ** 2 + d[:, 1] ** 2
    if mask is not None:
        a2 = a2 * mask
    return float(a2.sum() * dv)


def _mask(proj):
    """a smooth weight on the lattice (a centred disc), so the loss is not the plain norm"""
    n0, n1 = proj.dims[0], proj.dims[1]
    x = np.arange(n0) - n0 / 2
    y = np.arange(n1) - n1 / 2
    r2 = x[:, None] ** 2 + y[None, :] ** 2
    return np.exp(-r2 / (2 * (n0 / 5.0) ** 2)).reshape(-1)


@pytest.fixture(scope="module")
def setup_run(has_gpu):
    from wslda_b200 import TDRun
    proj, d = inputs(PROJ, NWF)
    run = TDRun(PROJ, NWF)

    def fresh(params):
        run.setup(d["states"], d["pots"], d["occ"], params, d["extra"])

    yield proj, d, run, fresh
    run.close()


@pytest.mark.gpu
def test_adjoint_loss_is_forward_loss(setup_run):
    """the loss the adjoint reports is |Delta|^2 of the plain forward's final potentials"""
    proj, d, run, fresh = setup_run
    m = _mask(proj)
    fresh(d["params"])
    run.initial_measurement()
    run.steps(NSTEPS)
    ref = _loss_from_pots(run.potentials(), proj.numel, proj.dv, m)
    fresh(d["params"])
    loss, _ = run.adjoint(NSTEPS, mask=m)
    assert abs(loss - ref) <= 1e-13 * abs(ref)
    assert ref > 0


@pytest.mark.gpu
@pytest.mark.parametrize("K", [1, 3, NSTEPS, 0])
def test_adjoint_gradient_vs_cuda_fd(setup_run, K):
    proj, d, run, fresh = setup_run
    m = _mask(proj)
    th = np.array(d["params"], dtype=np.float64)
    fresh(th)
    loss, g = run.adjoint(NSTEPS, nparam=NPARAM, mask=m, checkpoint_every=K)

    def loss_at(tp):
        fresh(tp)
        return run.adjoint(NSTEPS, mask=m)[0]

    fd = np.array([_richardson_fd(loss_at, th, j) for j in range(NPARAM)])
    err = rel(g, fd)
    print(f"K={K} loss={loss:.12e} |g|={np.linalg.norm(g):.6e} rel err vs CUDA FD {err:.3e}")
    assert err < TOL, (g, fd)
    # per component: 1e-5 relative, above the finite differences' own noise floor (the loss's
    # rounding, ~1e-16 L / h, here ~1e-7 of the largest component)
    assert np.all(np.abs(g - fd) <= 10 * TOL * np.abs(fd) + TOL * np.abs(fd).max())


@pytest.mark.gpu
def test_adjoint_checkpoint_interval_invariant(setup_run):
    """recompute is deterministic: the gradient does not depend on the checkpoint interval"""
    proj, d, run, fresh = setup_run
    m = _mask(proj)
    out = []
    for K in (1, 2, NSTEPS, 0):
        fresh(d["params"])
        out.append(run.adjoint(NSTEPS, nparam=NPARAM, mask=m, checkpoint_every=K)[1])
    assert all(np.array_equal(out[0], o) for o in out[1:])


@pytest.mark.gpu
def test_adjoint_leaves_forward_state(setup_run):
    """after the adjoint the run is where the forward left it: the next steps match"""
    proj, d, run, fresh = setup_run
    fresh(d["params"])
    run.initial_measurement()
    run.steps(NSTEPS)
    y_ref = run.states()
    it_ref = run.time_index()
    fresh(d["params"])
    run.adjoint(NSTEPS, nparam=NPARAM, checkpoint_every=3)
    assert run.time_index() == it_ref
    assert np.array_equal(run.states(), y_ref)
    # the call's device time, split at the loss: both parts ran
    ms_fwd, ms_rev = run.adjoint_times()
    assert ms_fwd > 0 and ms_rev > 0


@pytest.mark.gpu
def test_adjoint_gradient_vs_oracle_fd(setup_run):
    """against finite differences of the independent CPU step (the oracle)"""
    from oracle_lib import Oracle
    proj, d, run, fresh = setup_run
    m = _mask(proj)
    th = np.array(d["params"], dtype=np.float64)
    fresh(th)
    _, g = run.adjoint(NSTEPS_ORACLE, nparam=NPARAM, mask=m, checkpoint_every=6)
    o = Oracle(PROJ)

    def loss_at(tp):
        o.setup(d["states"], d["pots"], d["occ"], tp, d["extra"])
        o.initial_measurement()
        o.steps(NSTEPS_ORACLE)
        return _loss_from_pots(o.potentials(), proj.numel, proj.dv, m)

    fd = np.array([_richardson_fd(loss_at, th, j) for j in range(NPARAM)])
    err = rel(g, fd)
    print(f"rel err vs oracle FD {err:.3e}")
    assert err < TOL, (g, fd)


@pytest.mark.gpu
def test_adjoint_unsupported_elsewhere(has_gpu):
    """projects without the contact-BdG adjoint, and mixed precision, refuse cleanly"""
    from wslda_b200 import TDRun, WtdError
    proj, d = inputs("t2d_slda", 8)
    r = TDRun("t2d_slda", 8)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    with pytest.raises(WtdError, match="not supported"):
        r.adjoint(2, nparam=1)
    r.close()
    proj, d = inputs(PROJ, 8)
    r = TDRun(PROJ, 8, precision=2)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    with pytest.raises(WtdError, match="not supported"):
        r.adjoint(2, nparam=1)
    r.close()


@pytest.mark.gpu
def test_adjoint_through_torch_autograd(setup_run):
    """the torch.autograd.Function wrapper: backward() gives the adjoint gradient, which matches
    finite differences of the wrapper's own forward, and the chain rule through a composite loss
    (log(1 + L^2)) holds"""
    import torch
    from adjoint_autograd import StirrerLoss
    proj, d, run, fresh = setup_run
    m = _mask(proj)
    th0 = np.array(d["params"][:NPARAM], dtype=np.float64)
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    loss = StirrerLoss.apply(theta, run, d, NSTEPS, m, 3)
    loss.backward()
    g = theta.grad.numpy().copy()

    def loss_at(tp):
        with torch.no_grad():
            return float(StirrerLoss.apply(torch.tensor(tp), run, d, NSTEPS, m, 3))

    fd = np.array([_richardson_fd(loss_at, th0, j) for j in range(NPARAM)])
    assert rel(g, fd) < TOL, (g, fd)
    # composite: d/dtheta log(1 + L^2) = 2 L / (1 + L^2) dL/dtheta
    theta2 = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    L = StirrerLoss.apply(theta2, run, d, NSTEPS, m, 0)
    torch.log1p(L * L).backward()
    lv = float(L.detach())
    assert rel(theta2.grad.numpy(), 2 * lv / (1 + lv * lv) * g) < 1e-12


@pytest.mark.gpu
def test_adjoint_split_forward_backward(setup_run):
    """wtd_adjoint_forward + wtd_adjoint_backward give the one-call gradient bit for bit; the
    backward refuses a second time and after the run changed"""
    from wslda_b200 import WtdError
    proj, d, run, fresh = setup_run
    m = _mask(proj)
    fresh(d["params"])
    loss1, g1 = run.adjoint(NSTEPS, nparam=NPARAM, mask=m, checkpoint_every=3)
    fresh(d["params"])
    loss2 = run.adjoint_forward(NSTEPS, mask=m, checkpoint_every=3)
    g2 = run.adjoint_backward(NPARAM)
    assert loss1 == loss2 and np.array_equal(g1, g2)
    ms_fwd, ms_rev = run.adjoint_times()
    assert ms_fwd > 0 and ms_rev > 0
    with pytest.raises(WtdError):
        run.adjoint_backward(NPARAM)
    fresh(d["params"])
    run.adjoint_forward(NSTEPS, mask=m, checkpoint_every=3)
    run.steps(1)
    with pytest.raises(WtdError):
        run.adjoint_backward(NPARAM)
    fresh(d["params"])
    run.adjoint_forward(NSTEPS, mask=m, checkpoint_every=3)
    run.upload_states(d["states"])
    with pytest.raises(WtdError):
        run.adjoint_backward(NPARAM)
