"""calculate_densities_noalloc: the density sums for callers that cannot call cudaMalloc.

Some hosts cannot let a library allocate device memory — a driver whose device memory is all
reserved by a pool at start-up, or an embedding runtime that forbids allocation on its behalf.
calculate_densities_noalloc serves them: same inputs and outputs as calculate_densities, but
its scratch is a fixed array inside the library instead of a caller-provided work area.  This
test calls it through the C ABI twice in a row and checks each result against
calculate_densities on the same states (tolerance 1e-10 relative, as the other parity tests),
and checks that a lattice too large for the fixed scratch is refused.  It is collected last on
purpose and also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from parity_util import density_errors, inputs

TOL = 1e-10
VP = ctypes.c_void_p


def _dev(lib, a):
    p = VP()
    a = np.ascontiguousarray(a)
    assert lib.gpu_malloc(ctypes.c_size_t(max(a.nbytes, 16)), ctypes.byref(p)) == 0
    if a.nbytes:
        assert lib.memcopy_host2gpu(a.ctypes.data_as(VP), p, ctypes.c_size_t(a.nbytes)) == 0
    return p


def _get(lib, p, n):
    a = np.zeros(n)
    assert lib.memcopy_gpu2host(p, a.ctypes.data_as(VP), ctypes.c_size_t(a.nbytes)) == 0
    return a


def _plane_waves(proj, S, planewave):
    """per-state plane-wave data of the 1D/2D engines: all zero, or (planewave) a mix of zero and
    nonzero k_z (2D weight 1 or 2) and, in 1D, nonzero k_y, k_z with degeneracies cnt > 1"""
    if not planewave:
        return np.zeros(2 * S), np.ones(S, dtype=np.int32)
    rng = np.random.Generator(np.random.PCG64(7))
    k = rng.uniform(-0.8, 0.8, 2 * S)
    k[::3] = 0.0                      # some states in the k_perp = 0 plane (weight 1)
    if proj.codedim == 2:
        k[S:] = 0.0                   # the 2D engine reads only k_z (first S entries)
        k[1] = -np.pi / proj.dz       # the edge of the Brillouin zone (weight 1 with a cubic cut-off)
    cnt = rng.integers(1, 7, S).astype(np.int32)
    return k, cnt


def _densities(name, nwf, grads, weighted, planewave=False):
    from wslda_b200 import load_library
    proj, d = inputs(name, nwf)
    lib = load_library(name)
    N, S, cd = proj.numel, nwf, proj.codedim
    M = 2 * S * N
    wf = _dev(lib, d["states"])
    dx, dy, dz, lap = (_dev(lib, np.zeros(M, dtype=np.complex128)) for _ in range(4))
    fb = _dev(lib, d["occ"])
    w = _dev(lib, np.linspace(0.5, 1.5, S)) if weighted else None
    kk_h, cnt_h = _plane_waves(proj, S, planewave)
    kk = _dev(lib, kk_h)
    cnt = _dev(lib, cnt_h)
    outs = [_dev(lib, np.zeros(12 * N)) for _ in range(3)]
    assert lib.compute_derivatives(2 * S, wf, dx, dy, dz, lap, 512) == 0
    # the entry point that uses a caller-provided work area
    ws = ctypes.c_size_t()
    assert lib.create_cufftPlans(2 * S, S, ctypes.byref(ws)) == 0
    work = _dev(lib, np.zeros(ws.value // 8 + 1))
    assert lib.set_workspace_for_cufftPlan(work) == 0

    def call(fn, out):
        if cd == 3:
            return fn(S, wf, dx, dy, dz, lap, fb, w, out, grads, 512)
        if cd == 2:
            return fn(S, wf, dx, dy, lap, kk, fb, w, out, grads, 512)
        return fn(S, wf, dx, lap, kk, fb, w, cnt, out, grads, 512)

    assert call(lib.calculate_densities, outs[0]) == 0
    # two calls in a row of the no-allocation variant
    assert call(lib.calculate_densities_noalloc, outs[1]) == 0
    assert call(lib.calculate_densities_noalloc, outs[2]) == 0
    res = [_get(lib, o, 12 * N) for o in outs]
    for p in [wf, dx, dy, dz, lap, fb, kk, cnt, work] + outs + ([w] if w else []):
        lib.gpu_free(p)
    return N, res


@pytest.mark.gpu
@pytest.mark.parametrize("name,grads,weighted,planewave", [
    ("t2d_slda", 1, False, False), ("t2d_slda", 0, True, False), ("t1d_custom", 1, True, False),
    ("t3d_slda", 1, False, False), ("c2_slda2d", 0, False, False),
    # the plane-wave weights the kernel forms itself: 2D k_z != 0 counts twice, 1D states carry
    # their degeneracy cnt and |k_perp|^2 enters tau
    ("t2d_slda", 1, True, True), ("t2d_bdg", 1, False, True), ("t1d_custom", 1, False, True),
    ("t1d_aslda", 1, True, True), ("t1d_sldae_a1", 1, False, True)])
def test_noalloc_densities_match_workspace_densities(has_gpu, name, grads, weighted, planewave):
    N, (ref, first, second) = _densities(name, 24, grads, weighted, planewave)
    assert np.linalg.norm(ref) > 0
    for got in (first, second):
        for k, v in density_errors(got, ref, N).items():
            assert v < TOL, f"{name}: {k} rel err {v:.3e}"


@pytest.mark.gpu
def test_noalloc_rejects_lattice_beyond_fixed_scratch(has_gpu):
    """48^3: 12*N doubles exceed the 8 MiB array; the call returns -6 before any GPU work."""
    from wslda_b200 import load_library
    lib = load_library("c5_slda3d")
    rc = lib.calculate_densities_noalloc(4, None, None, None, None, None, None, None, None, 1, 512)
    assert rc == -6
    assert "too large" in lib.wtd_error_string(-6).decode()
