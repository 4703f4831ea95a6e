"""B200-native TD-(A)SLDA/BdG step for W-SLDA projects.

The product is the per-project CUDA library ``libwtd.so`` (C ABI in ``include/wtd.h``).  This
package builds it (``wslda_b200.build``) and mirrors the reference's host driver calls in
Python for tests and benchmarks (:class:`TDRun`).  There is no CPU fallback: a context can
only be created where the CUDA library loads and a GPU is present.
"""
import ctypes
import os

import numpy as np

from . import build as _build
from .projects import Project

__all__ = ["Project", "TDRun", "load_library", "FP64", "MIXED_H64", "MIXED_H32"]

FP64, MIXED_H64, MIXED_H32 = 0, 1, 2
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_LIBS = {}

# every symbol include/wtd.h declares, with its ctypes signature
SIGNATURES = {
    "wtd_info": (ctypes.c_int, [_ip, _ip, _ip, _ip, _ip, _ip]),
    "wtd_device_bytes": (ctypes.c_size_t, [ctypes.c_int, ctypes.c_int]),
    "wtd_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "wtd_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "wtd_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "wtd_set_constants": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_double] * 6),
    "wtd_set_params": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_set_sclgth": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "wtd_set_extra_data": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "wtd_process_params": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp]),
    "wtd_upload_states": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_upload_potentials": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_upload_occupations": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _ip]),
    "wtd_upload_history": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "wtd_download_history": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "wtd_initial_measurement": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "wtd_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "wtd_selfstart": (ctypes.c_int, [ctypes.c_void_p]),
    "wtd_subset_densities": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    "wtd_wdata_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_int]),
    "wtd_wdata_write": (ctypes.c_int, [ctypes.c_void_p]),
    "wtd_checkpoint_info_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "wtd_checkpoint_save": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p, _dp, _dp]),
    "wtd_checkpoint_load": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           _ip, ctypes.c_void_p, _dp, _dp]),
    "wtd_energy": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "wtd_time_index": (ctypes.c_int, [ctypes.c_void_p]),
    "wtd_download_states": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_download_densities": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_download_potentials": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_download_qpe": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "wtd_device_pointers": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(_dp), ctypes.POINTER(_dp)]),
    "wtd_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "wtd_launch_count": (ctypes.c_longlong, [ctypes.c_void_p]),
    "wtd_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "wtd_pass_times": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _ip, _ip]),
    "wtd_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp]),
    "wtd_adjoint_release": (ctypes.c_int, [ctypes.c_void_p]),
    "wtd_adjoint_times": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    "wtd_adjoint_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]),
    "wtd_adjoint_backward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "wtd_set_high_k_filter": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    "wtd_set_quantum_friction": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_double] * 7),
    "wtd_nccl_unique_id": (ctypes.c_int, [ctypes.c_void_p]),
    "wtd_nccl_attach": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "wtd_set_density_exchange": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
}

# host hook of a state-sharded run: int fn(void *user, double *dens, size_t count, void *stream)
class CheckpointInfo(ctypes.Structure):
    """wtd_checkpoint_info (include/wtd.h): the checkpoint file header"""
    _fields_ = [("t0", ctypes.c_double), ("mu_a", ctypes.c_double), ("mu_b", ctypes.c_double),
                ("ec", ctypes.c_double), ("kF", ctypes.c_double), ("eF", ctypes.c_double),
                ("Effg", ctypes.c_double), ("beta", ctypes.c_double), ("nwf", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)


def load_library(project, build=True):
    """Load (building if needed) the CUDA library of a project."""
    if project in _LIBS:
        return _LIBS[project]
    path = _build.lib_path(project)
    if build:
        path = _build.build(project)
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library for {project} not built ({path}); run python -m wslda_b200.build {project}")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIBS[project] = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


class WtdError(RuntimeError):
    pass


def checkpoint_info(project, directory, rank=0, howmany=24):
    """the header of a checkpoint in the reference's layout (t0, mu, ec, kF, eF, Effg, beta,
    nwf) as a dict"""
    name = project.name if isinstance(project, Project) else project
    lib = load_library(name)
    ci = CheckpointInfo()
    rc = lib.wtd_checkpoint_info_read(os.fsencode(directory), int(rank), int(howmany), ctypes.byref(ci))
    if rc != 0:
        raise WtdError(f"{name}: {lib.wtd_error_string(rc).decode()} ({rc})")
    return ci.as_dict()


class TDRun:
    """One TD run on one GPU: the reference driver's sequence (pca.c:749-1571) over the C ABI."""

    def __init__(self, project, nwf, precision=FP64, device=0, build=True):
        self.proj = project if isinstance(project, Project) else Project(project)
        self.lib = load_library(self.proj.name, build=build)
        self.nwf = int(nwf)
        self.N = self.proj.numel
        h = ctypes.c_void_p()
        self._check(self.lib.wtd_create(ctypes.byref(h), self.nwf, int(precision), int(device)))
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise WtdError(f"{self.proj.name}: {self.lib.wtd_error_string(rc).decode()} ({rc})")

    def close(self):
        if getattr(self, "h", None):
            self.lib.wtd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self, states, pots, occ, params, extra=None, const=None, it0=0, kky=None, kkz=None, cnt=None):
        self.upload_states(states)
        self.setup_fields(pots, occ, params, extra, const, it0, kky, kkz, cnt)

    def setup_fields(self, pots, occ, params, extra=None, const=None, it0=0, kky=None, kkz=None, cnt=None):
        """everything of setup() but the states (for states written on the device directly)"""
        c = const or self.proj.constants()
        self._check(self.lib.wtd_set_constants(self.h, c["mu_a"], c["mu_b"], c["ec"], c["t0"], c["dt"], c["kF"]))
        self._check(self.lib.wtd_set_sclgth(self.h, c["sclgth"]))
        self._params = np.ascontiguousarray(params, dtype=np.float64)
        self._check(self.lib.wtd_set_params(self.h, _p(self._params)))
        ex = np.ascontiguousarray(extra if extra is not None else np.zeros(0), dtype=np.float64)
        self._check(self.lib.wtd_set_extra_data(self.h, ex.ctypes.data if ex.size else None, ex.nbytes))
        self._check(self.lib.wtd_upload_potentials(self.h, _p(np.ascontiguousarray(pots, dtype=np.float64))))
        cnt_p = None if cnt is None else np.ascontiguousarray(cnt, dtype=np.int32).ctypes.data_as(_ip)
        kky = None if kky is None else np.ascontiguousarray(kky, dtype=np.float64)
        kkz = None if kkz is None else np.ascontiguousarray(kkz, dtype=np.float64)
        self._check(self.lib.wtd_upload_occupations(self.h, _p(np.ascontiguousarray(occ, dtype=np.float64)),
                                                     _p(kky), _p(kkz), cnt_p))
        self.it0 = it0

    def upload_states(self, states):
        st = np.ascontiguousarray(states, dtype=np.complex128)
        self._check(self.lib.wtd_upload_states(self.h, _p(st.view(np.float64))))

    def initial_measurement(self, it0=None):
        self._check(self.lib.wtd_initial_measurement(self.h, int(self.it0 if it0 is None else it0)))

    def subset_densities(self, weights):
        """densities (12 N) of the states weighted by weights (subset tracking)"""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        out = np.zeros(12 * self.N)
        self._check(self.lib.wtd_subset_densities(self.h, _p(w), _p(out)))
        return out

    def selfstart(self):
        """Taylor self-start of the ABM history (after initial_measurement)"""
        self._check(self.lib.wtd_selfstart(self.h))

    def steps(self, n):
        self._check(self.lib.wtd_steps(self.h, int(n)))

    def sync(self):
        self._check(self.lib.wtd_sync(self.h))

    def energy(self):
        e = np.zeros(11)
        self._check(self.lib.wtd_energy(self.h, _p(e)))
        return e

    def states(self, out=None):
        a = out if out is not None else np.zeros(2 * self.nwf * self.N, dtype=np.complex128)
        self._check(self.lib.wtd_download_states(self.h, _p(a.view(np.float64))))
        return a

    def densities(self, out=None):
        a = out if out is not None else np.zeros(12 * self.N)
        self._check(self.lib.wtd_download_densities(self.h, _p(a)))
        return a

    def potentials(self):
        a = np.zeros(12 * self.N)
        self._check(self.lib.wtd_download_potentials(self.h, _p(a)))
        return a

    def qpe(self):
        a = np.zeros(self.nwf)
        self._check(self.lib.wtd_download_qpe(self.h, _p(a)))
        return a

    def history(self, slot):
        a = np.zeros(2 * self.nwf * self.N, dtype=np.complex128)
        self._check(self.lib.wtd_download_history(self.h, int(slot), _p(a.view(np.float64))))
        return a

    def time_index(self):
        return self.lib.wtd_time_index(self.h)

    def launches(self):
        return self.lib.wtd_launch_count(self.h)

    def stream(self):
        return self.lib.wtd_stream(self.h)

    def set_timing(self, on=True):
        self._check(self.lib.wtd_set_timing(self.h, 1 if on else 0))

    def pass_times(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        na, nb = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.wtd_pass_times(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(na), ctypes.byref(nb)))
        return a.value, b.value, na.value, nb.value

    def nccl_unique_id(self):
        """128-byte NCCL unique id (made on one rank, sent to all)"""
        buf = ctypes.create_string_buffer(128)
        self._check(self.lib.wtd_nccl_unique_id(buf))
        return buf.raw

    def attach_nccl(self, uid, nranks, rank):
        """sum the density partials over nranks contexts with NCCL on this context's stream"""
        buf = ctypes.create_string_buffer(bytes(uid), 128)
        self._check(self.lib.wtd_nccl_attach(self.h, buf, int(nranks), int(rank)))

    def set_density_exchange(self, fn):
        """host hook fn(dens_ptr, count, stream_ptr) -> None, called after every density
        reduction; it must leave the sum over ranks in place (None removes the hook)"""
        if fn is None:
            self._xfn = None
            self._check(self.lib.wtd_set_density_exchange(self.h, None, None))
            return

        def tramp(_user, ptr, count, stream):
            try:
                fn(ptr, count, stream)
                return 0
            except Exception:  # reported to the library as a failed exchange
                import traceback
                traceback.print_exc()
                return 1

        self._xfn = EXCHANGE_FN(tramp)
        self._check(self.lib.wtd_set_density_exchange(self.h, ctypes.cast(self._xfn, ctypes.c_void_p), None))

    def set_high_k_filter(self, mode, mu, T):
        """Fermi-Dirac filter of alpha_a, alpha_b after each functional evaluation (variable
        mass); mu, T are energies"""
        self._check(self.lib.wtd_set_high_k_filter(self.h, int(mode), float(mu), float(T)))

    def set_quantum_friction(self, alpha, beta, gamma, nreq, start, stop, ramp):
        """quantum friction as the reference's input qfalpha, qfbeta, qfgamma, qfNreq, qfstart,
        qfstop, qfswitch (times in 1/eF); all coefficients 0 turns it off"""
        self._check(self.lib.wtd_set_quantum_friction(self.h, *[float(x) for x in (alpha, beta, gamma, nreq, start,
                                                                                   stop, ramp)]))

    def adjoint_forward(self, nsteps, mask=None, checkpoint_every=0, it0=None):
        """the forward of adjoint() with its checkpoints and records, for a later
        adjoint_backward(); returns L.  The run must not change before the backward."""
        loss = np.zeros(1)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        self._check(self.lib.wtd_adjoint_forward(self.h, int(self.it0 if it0 is None else it0), int(nsteps),
                                                 int(checkpoint_every), _p(m), _p(loss)))
        return float(loss[0])

    def adjoint_backward(self, nparam):
        """the reverse sweep after adjoint_forward(): dL/dparams[:nparam]"""
        grad = np.zeros(nparam)
        self._check(self.lib.wtd_adjoint_backward(self.h, int(nparam), _p(grad)))
        return grad

    def adjoint_times(self):
        """(ms of the last adjoint forward, ms of the reverse sweep after it), device-timed"""
        a, b = np.zeros(1), np.zeros(1)
        self._check(self.lib.wtd_adjoint_times(self.h, _p(a), _p(b)))
        return float(a[0]), float(b[0])

    def adjoint_release(self):
        """free the adjoint's device workspace (kept between gradient calls)"""
        self._check(self.lib.wtd_adjoint_release(self.h))

    def checkpoint_save(self, directory, info, En, kperp=None, rank=0, nranks=1, howmany=24):
        """write this rank's part of <directory>/checkpoint_<rank // howmany> in the reference's
        layout; info: dict of CheckpointInfo fields (nwf = states of all ranks)"""
        ci = CheckpointInfo(**info)
        en = np.ascontiguousarray(En, dtype=np.float64)
        kp = None if kperp is None else np.ascontiguousarray(kperp, dtype=np.float64)
        self._check(self.lib.wtd_checkpoint_save(self.h, os.fsencode(directory), int(rank), int(nranks), int(howmany),
                                                 ctypes.byref(ci), _p(en), _p(kp)))

    def checkpoint_load(self, directory, rank=0, nranks=1, howmany=24, cnt=None):
        """read this rank's part back and measure; returns (info dict, E_n, k_perp)"""
        ci = CheckpointInfo()
        en = np.zeros(self.nwf)
        kp = np.zeros(2 * self.nwf)
        c = None if cnt is None else np.ascontiguousarray(cnt, dtype=np.int32)
        self._check(self.lib.wtd_checkpoint_load(self.h, os.fsencode(directory), int(rank), int(nranks), int(howmany),
                                                 None if c is None else c.ctypes.data_as(_ip), ctypes.byref(ci),
                                                 _p(en), _p(kp)))
        return ci.as_dict(), en, kp

    def wdata_begin(self, prefix, vars=None, t0=0.0, dt_cycle=1.0, float_prec=False):
        """start a W-data set <prefix>.wtxt / <prefix>_<var>.wdat (the reference's output format)"""
        v = None if vars is None else (vars if isinstance(vars, str) else " ".join(vars)).encode()
        self._check(self.lib.wtd_wdata_begin(self.h, os.fsencode(prefix), v, float(t0), float(dt_cycle),
                                             1 if float_prec else 0))

    def wdata_write(self):
        """append one cycle of the current densities and potentials"""
        self._check(self.lib.wtd_wdata_write(self.h))

    def set_params(self, params):
        self._params = np.ascontiguousarray(params, dtype=np.float64)
        self._check(self.lib.wtd_set_params(self.h, _p(self._params)))

    def adjoint(self, nsteps, nparam=0, mask=None, checkpoint_every=0, it0=None):
        """Loss L = sum_r |Delta(r,T)|^2 mask dV after initial_measurement(it0) + nsteps steps
        from the uploaded states, and (nparam > 0) dL/dparams[:nparam] by the adjoint sweep
        (checkpoint_every 0: the largest interval that fits in device memory).
        Returns (L, grad or None); the run is left at the end of the forward."""
        loss = np.zeros(1)
        grad = np.zeros(max(nparam, 1))
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        self._check(self.lib.wtd_adjoint(self.h, int(self.it0 if it0 is None else it0), int(nsteps),
                                         int(checkpoint_every), _p(m), int(nparam), _p(loss),
                                         _p(grad) if nparam > 0 else None))
        return float(loss[0]), (grad[:nparam].copy() if nparam > 0 else None)
