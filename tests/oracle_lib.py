"""ctypes loader for the CPU oracle (test infrastructure; see oracle/wtd_oracle.cpp)."""
import ctypes
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def build(project):
    so = os.path.join(ORACLE_DIR, "_build", project, "liboracle.so")
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, f"PROJECT={project}"], check=True)
    return so


def _stale(so):
    if not os.path.exists(so):
        return True
    t = os.path.getmtime(so)
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("wtd_oracle.cpp", "oracle_surface.h", "oracle_edf.h")]
    return any(os.path.exists(f) and os.path.getmtime(f) > t for f in srcs)


def wderiv_library(project):
    """the wderiv baseline library of a project, built when the reference tree is present;
    None when it is neither built nor buildable"""
    so = os.path.join(ORACLE_DIR, "_ref", project, "liboracle_wderiv.so")
    ref = os.environ.get("WSLDA_REFERENCE", os.path.join(REPO, os.pardir, "reference"))
    if os.path.isdir(os.path.join(ref, "lib", "wderiv")):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "wderiv", f"PROJECT={project}"], check=True)
    return so if os.path.exists(so) else None


class Oracle:
    """One oracle instance per project (a separate process-level library, as it keeps state)."""

    def __init__(self, project, threads=None, variant=None):
        """variant "wderiv": the host-core baseline build, whose state derivatives come from the
        reference's lib/wderiv (oracle/_ref/<project>/liboracle_wderiv.so, made by
        `make -C oracle wderiv PROJECT=<project>` where the reference tree is present)"""
        from wslda_b200.projects import Project
        self.proj = Project(project)
        if variant == "wderiv":
            so = wderiv_library(project)
            if so is None:
                raise FileNotFoundError(f"no wderiv build of {project}")
        else:
            so = os.path.join(ORACLE_DIR, "_build", project, "liboracle.so")
            if _stale(so):
                build(project)
        self.lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
        L = self.lib
        for fn in ("orc_numel", "orc_codedim", "orc_nhist", "orc_functional", "orc_const_mass", "orc_get_it",
                   "orc_initial_measurement"):
            getattr(L, fn).restype = ctypes.c_int
        L.orc_set_constants.argtypes = [ctypes.c_double] * 7
        L.orc_set_params.argtypes = [_dp]
        L.orc_set_extra_data.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        L.orc_setup.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _ip, ctypes.c_int]
        L.orc_steps.argtypes = [ctypes.c_int]
        L.orc_energy.argtypes = [_dp]
        for fn in ("orc_get_states", "orc_get_densities", "orc_get_potentials", "orc_get_qpe"):
            getattr(L, fn).argtypes = [_dp]
        L.orc_get_history.argtypes = [ctypes.c_int, _dp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_fft_field.argtypes = [_dp, ctypes.c_int]
        L.orc_derivatives_field.argtypes = [_dp] * 5
        L.orc_set_density_exchange.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_set_high_k_filter.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.orc_selfstart.restype = ctypes.c_int
        L.orc_set_quantum_friction.argtypes = [ctypes.c_double] * 7
        L.orc_qf_densities.argtypes = [_dp]
        L.orc_subset_densities.argtypes = [_dp, _dp]
        L.orc_filter_field.argtypes = [_dp]
        L.orc_process_params.argtypes = [_dp, _dp, _dp]
        self._xfn = None
        # the library is shared by every instance in the process: start from a plain run
        L.orc_set_high_k_filter(0, 0.0, 1.0)
        L.orc_set_quantum_friction(0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
        L.orc_set_density_exchange(None, None)
        if threads:
            L.orc_set_threads(int(threads))
        self.N = L.orc_numel()
        self.S = 0

    def setup(self, states, pots, occ, params, extra=None, const=None, it0=0, kky=None, kkz=None, cnt=None):
        c = const or self.proj.constants()
        self.lib.orc_set_constants(c["mu_a"], c["mu_b"], c["ec"], c["t0"], c["dt"], c["kF"], c["sclgth"])
        self.params = np.ascontiguousarray(params, dtype=np.float64)
        self.lib.orc_set_params(_p(self.params))
        self.extra = np.ascontiguousarray(extra if extra is not None else np.zeros(0), dtype=np.float64)
        self.lib.orc_set_extra_data(self.extra.ctypes.data if self.extra.size else None, self.extra.nbytes)
        self.S = occ.size
        st = np.ascontiguousarray(states, dtype=np.complex128).view(np.float64)
        kky = None if kky is None else np.ascontiguousarray(kky, dtype=np.float64)
        kkz = None if kkz is None else np.ascontiguousarray(kkz, dtype=np.float64)
        cnt_p = None if cnt is None else np.ascontiguousarray(cnt, dtype=np.int32).ctypes.data_as(_ip)
        self.lib.orc_setup(self.S, _p(st), _p(np.ascontiguousarray(pots, dtype=np.float64)),
                           _p(np.ascontiguousarray(occ, dtype=np.float64)), _p(kky), _p(kkz), cnt_p, it0)

    def process_params(self, params, kF, mu):
        """the project's process_params hook on (params, kF[1], mu[2]) in place"""
        self.lib.orc_process_params(_p(params), _p(kF), _p(mu))

    def initial_measurement(self):
        return self.lib.orc_initial_measurement()

    def selfstart(self):
        return self.lib.orc_selfstart()

    def subset_densities(self, weights):
        w = np.ascontiguousarray(weights, dtype=np.float64)
        a = np.zeros(12 * self.N)
        self.lib.orc_subset_densities(_p(w), _p(a))
        return a

    def qf_densities(self):
        a = np.zeros(4 * self.N)
        self.lib.orc_qf_densities(_p(a))
        return a

    def set_quantum_friction(self, alpha, beta, gamma, nreq, start, stop, ramp):
        """friction coefficients and the switch times (units of 1/eF), as the reference's input
        qfalpha, qfbeta, qfgamma, qfNreq, qfstart, qfstop, qfswitch"""
        self.lib.orc_set_quantum_friction(alpha, beta, gamma, nreq, start, stop, ramp)

    def set_high_k_filter(self, mode, mu, T):
        self.lib.orc_set_high_k_filter(int(mode), float(mu), float(T))

    def filter_field(self, f):
        a = np.ascontiguousarray(f, dtype=np.float64).copy()
        self.lib.orc_filter_field(_p(a))
        return a

    def set_density_exchange(self, fn):
        """fn(dens) with dens a numpy view of the 12N partial densities, summed in place over
        ranks (None removes the hook)"""
        if fn is None:
            self._xfn = None
            self.lib.orc_set_density_exchange(None, None)
            return
        proto = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t)

        def tramp(_user, ptr, count):
            fn(np.ctypeslib.as_array(ptr, shape=(count,)))
            return 0

        self._xfn = proto(tramp)
        self.lib.orc_set_density_exchange(ctypes.cast(self._xfn, ctypes.c_void_p), None)

    def steps(self, n):
        return self.lib.orc_steps(int(n))

    def energy(self):
        e = np.zeros(11)
        self.lib.orc_energy(_p(e))
        return e

    def states(self):
        a = np.zeros(2 * self.S * self.N, dtype=np.complex128)
        self.lib.orc_get_states(_p(a.view(np.float64)))
        return a

    def densities(self):
        a = np.zeros(12 * self.N)
        self.lib.orc_get_densities(_p(a))
        return a

    def potentials(self):
        a = np.zeros(12 * self.N)
        self.lib.orc_get_potentials(_p(a))
        return a

    def qpe(self):
        a = np.zeros(self.S)
        self.lib.orc_get_qpe(_p(a))
        return a

    def history(self, slot):
        a = np.zeros(2 * self.S * self.N, dtype=np.complex128)
        self.lib.orc_get_history(slot, _p(a.view(np.float64)))
        return a

    def fft_field(self, f, sign):
        a = np.ascontiguousarray(f, dtype=np.complex128).copy()
        self.lib.orc_fft_field(_p(a.view(np.float64)), sign)
        return a

    def derivatives_field(self, f):
        f = np.ascontiguousarray(f, dtype=np.complex128)
        outs = [np.zeros(self.N, dtype=np.complex128) for _ in range(4)]
        self.lib.orc_derivatives_field(*[_p(x.view(np.float64)) for x in [f] + outs])
        return outs
