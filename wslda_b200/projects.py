"""Project registry and seeded synthetic inputs.

A *project* is a W-SLDA user project (predefines.h + problem-definition.h, compiled into one
library per project exactly as the reference compiles one td-wslda-{1d,2d,3d} binary per
project) plus ``project.json`` holding the run-time inputs the reference reads from input.txt.

Synthetic inputs follow one recipe for every workload: numpy PCG64 seeded with
``20261203 + config id``, complex Gaussian (u, v) states QR-orthonormalised and scaled so that
sum_x (|u|^2 + |v|^2) dV = 1, occupations f_n = 1 for n < S/2 else 0, initial potentials
V = 0, Delta = 0, alpha = 1, A = 0 (the reference's reset_potentials, wslda_potdens.c:76-98).
"""
import json
import os

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PROJECTS_DIR = os.path.join(ROOT, "projects")
SEED_BASE = 20261203
CONFIG_IDS = {"c1_bdg1d": 1, "c2_slda2d": 2, "c3_aslda3d": 3, "c4_bdg2d": 4, "c5_slda3d": 5}


def project_dir(name):
    d = os.path.join(PROJECTS_DIR, name)
    if not os.path.isdir(d):
        raise ValueError(f"unknown project {name!r}")
    return d


def _parse_predefines(name):
    vals = {}
    with open(os.path.join(project_dir(name), "predefines.h")) as fh:
        for line in fh:
            parts = line.split()
            if len(parts) >= 3 and parts[0] == "#define":
                vals[parts[1]] = " ".join(parts[2:]).strip("()")
            elif len(parts) == 2 and parts[0] == "#define":
                vals[parts[1]] = True
    return vals


class Project:
    """Compile-time lattice and run-time inputs of one project."""

    def __init__(self, name):
        self.name = name
        with open(os.path.join(project_dir(name), "project.json")) as fh:
            self.cfg = json.load(fh)
        pre = _parse_predefines(name)
        self.codedim = int(self.cfg["codedim"])
        self.nx, self.ny, self.nz = int(pre["NX"]), int(pre["NY"]), int(pre["NZ"])
        self.dx, self.dy, self.dz = float(pre["DX"]), float(pre["DY"]), float(pre["DZ"])
        self.functional = pre["FUNCTIONAL"]
        self.scheme = pre.get("INTEGRATION_SCHEME", "AB4AM5")
        self.nhist = {"AB3AM4": 3, "AB4AM5": 4, "AB5AM5": 5}[self.scheme]
        # an external velocity field forces the variable-mass (current-correction) path
        self.const_mass = bool((self.functional in ("SLDA", "BDG") or "SLDA_FORCE_A1" in pre
                                or "SLDAE_FORCE_A1" in pre)
                               and "ENABLE_VELOCITY_EXT" not in pre)
        self.dims = [self.nx, self.ny if self.codedim >= 2 else 1, self.nz if self.codedim >= 3 else 1]
        self.numel = int(np.prod(self.dims))
        self.dv = {1: self.dx, 2: self.dx * self.dy, 3: self.dx * self.dy * self.dz}[self.codedim]

    @property
    def params(self):
        p = np.zeros(32)
        for k, v in self.cfg.get("params", {}).items():
            p[int(k)] = v
        return p

    def constants(self):
        c = self.cfg
        return dict(mu_a=c["mu_a"], mu_b=c["mu_b"], ec=c["ec"], t0=0.0, dt=c["dt"], kF=c["kF"],
                    sclgth=c.get("sclgth", 0.0))


def config_seed(name, salt=0):
    return SEED_BASE + CONFIG_IDS.get(name, 100 + sum(map(ord, name)) % 100) + salt


def make_states(proj, nwf, seed, orthonormal=True):
    """(2*nwf*N) complex128 array laid out [u_0..u_{S-1}, v_0..v_{S-1}], each of length N."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n2 = 2 * proj.numel
    a = rng.standard_normal((n2, nwf)) + 1j * rng.standard_normal((n2, nwf))
    if orthonormal and nwf <= n2:
        a, _ = np.linalg.qr(a)
    else:
        a /= np.linalg.norm(a, axis=0, keepdims=True)
    a = a / np.sqrt(proj.dv)
    u = a[: proj.numel, :].T
    v = a[proj.numel:, :].T
    return np.ascontiguousarray(np.concatenate([u, v], axis=0).reshape(-1))


def make_occupations(nwf):
    f = np.zeros(nwf)
    f[: nwf // 2] = 1.0
    return f


def make_potentials(proj):
    p = np.zeros(12 * proj.numel)
    n = proj.numel
    p[4 * n:6 * n] = 1.0  # alpha_a, alpha_b
    return p


def make_extra(proj, seed):
    """Seeded extra_data for projects whose hooks read a field from it (delta_noise)."""
    ex = proj.cfg.get("extra")
    if not ex:
        return np.zeros(0)
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    if ex["kind"] == "delta_noise":
        mag = ex["mean"] + ex["sigma"] * rng.standard_normal(proj.numel)
        d = mag * np.exp(1j * ex.get("phase", 0.0))
        return np.ascontiguousarray(d.astype(np.complex128)).view(np.float64)
    raise ValueError(ex["kind"])


def stirrer_params(proj, seed):
    """C4's 14 stirrer parameters, seeded U[0.1, 1] (path coefficients, A, w)."""
    rng = np.random.Generator(np.random.PCG64(seed + 11))
    p = proj.params.copy()
    p[: proj.cfg.get("stirrer_params", 0)] = rng.uniform(0.1, 1.0, proj.cfg.get("stirrer_params", 0))
    return p
