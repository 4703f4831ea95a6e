"""Make the td-gauss replay fixtures (tests/golden/td_gauss/<case>.npz) in the build container.

For each td-gauss test of the reference's testsuite (testsuite/td-gauss-*/test.desc) this:

1. writes the run's input file as test.desc does (input.txt.<dim>, plus `params7 1` for the
   spin-imbalanced "ss0" runs);
2. builds and runs oracle/_ref/<project>/uniform_init, the reference's own uniform-solution
   generator (hpc-engine/pca_uniform.h) compiled where it lies by `make -C oracle uniform`;
3. reduces each generated state to its plane wave (the k index per axis) and its amplitudes
   u_k, v_k, and checks that tests/td_gauss_util.initial_states rebuilds every state from them;
4. reads the reference's logged trajectory (ref/<stem>.wlog.ref: time*eF, N_a, N_b, energies
   / Effg after each of the 100 measurement blocks) and final values (ref/<stem>.cmp.ref).

    python tests/golden/make_td_gauss.py [case ...]

The reference's td-gauss-sldae log was written with dt*eF = 0.00175 (its header), not the
0.0035 of the input file now in the tree; the fixture takes dt*eF from the log's header and
the block length from its time column, for every case.
"""
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.dirname(HERE))
from wslda_b200 import projects as P  # noqa: E402
from td_gauss_util import GOLDEN, initial_states  # noqa: E402

# the reference tree: WSLDA_REFERENCE, by default a "reference" folder beside the repository
REFERENCE = os.environ.get("WSLDA_REFERENCE", os.path.join(REPO, os.pardir, "reference"))
TESTSUITE = os.path.join(REFERENCE, "testsuite")


def cases():
    out = {}
    for fam in ("bdg", "slda", "aslda"):
        for d in (1, 2, 3):
            out[f"{fam}_ss0_{d}d"] = (f"td-gauss-{fam}", f"test.ss0-{d}d", f"gauss_{fam}_{d}d", d, ["params7       1"])
            out[f"{fam}_ss1_{d}d"] = (f"td-gauss-{fam}", f"test.ss1-{d}d", f"gauss_{fam}_{d}d_sym", d, [])
    for fam, ref in (("sldae", "td-gauss-sldae"), ("sldae_a1", "td-gauss-sldae-a1")):
        for d in (1, 2, 3):
            out[f"{fam}_ss1_{d}d"] = (ref, f"test.ss1-{d}d", f"gauss_{fam}_{d}d_sym", d, [])
    return out


def read_params(text):
    """paramsN values of an input file, the last line of a tag winning (pca_utils.c:162-560)"""
    p = np.zeros(8)
    for line in text.splitlines():
        m = re.match(r"\s*params\[?\s*(\d+)\s*\]?\s+([-+0-9.eE]+)", line)
        if m and int(m.group(1)) < 8:
            p[int(m.group(1))] = float(m.group(2))
    return p


def read_wlog(path):
    head, rows = {}, []
    for line in open(path):
        if line.startswith("#"):
            m = re.match(r"#\s+(\S+)\s+=\s+([-+0-9.eE]+)", line)
            if m:
                head[m.group(1)] = float(m.group(2))
            continue
        parts = line.split()
        if len(parts) >= 14:
            rows.append([float(x) for x in parts[:14]])
    return head, np.array(rows)


def read_cmp(path):
    vals = []
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2:
            vals.append(float(parts[1]))
    return np.array(vals)


def run_uniform(project, input_text):
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "uniform", f"PROJECT={project}"], check=True)
    exe = os.path.join(REPO, "oracle", "_ref", project, "uniform_init")
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "input.txt")
        open(inp, "w").write(input_text)
        out = os.path.join(td, "out.bin")
        r = subprocess.run([exe, inp, out], cwd=td, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"uniform_init failed ({r.returncode}): {r.stdout[-2000:]}")
        raw = open(out, "rb").read()
    hdr = np.frombuffer(raw[:16], dtype=np.int32)
    d, N, S, sym = (int(x) for x in hdr)
    o = 16
    meta = np.frombuffer(raw[o:o + 96], dtype=np.float64).copy(); o += 96
    En = np.frombuffer(raw[o:o + 8 * S], dtype=np.float64).copy(); o += 8 * S
    nk = {3: 0, 2: S, 1: 2 * S}[d]
    kperp = np.frombuffer(raw[o:o + 8 * nk], dtype=np.float64).copy(); o += 8 * nk
    cnt = np.frombuffer(raw[o:o + 4 * S], dtype=np.int32).copy(); o += 4 * S
    wf = np.frombuffer(raw[o:o + 16 * 2 * S * N], dtype=np.complex128).copy()
    return dict(codedim=d, N=N, nwf=S, spinsymmetry=sym, meta=meta, En=En, kperp=kperp, cnt=cnt, wf=wf)


def compress(proj, u):
    """plane-wave index per axis and amplitudes of every state"""
    d, S, N = u["codedim"], u["nwf"], u["N"]
    shape = {3: (proj.nx, proj.ny, proj.nz), 2: (proj.nx, proj.ny), 1: (proj.nx,)}[d]
    vol = {3: (proj.dx * proj.nx) * (proj.dy * proj.ny) * (proj.dz * proj.nz),
           2: (proj.dx * proj.nx) * (proj.dy * proj.ny), 1: proj.dx * proj.nx}[d]
    wf = u["wf"].reshape(2, S, N)
    kidx = np.zeros((S, 3), dtype=np.int16)
    uk, vk = np.zeros(S), np.zeros(S)
    for n in range(S):
        a = wf[0, n] if np.abs(wf[0, n]).max() >= np.abs(wf[1, n]).max() else wf[1, n]
        spec = np.abs(np.fft.fftn(a.reshape(shape)))
        idx = np.unravel_index(int(np.argmax(spec)), shape)
        kidx[n, :len(idx)] = idx
        uk[n] = wf[0, n, 0].real * np.sqrt(vol)
        vk[n] = wf[1, n, 0].real * np.sqrt(vol)
    return kidx, uk, vk


def make(case, spec):
    refdir, stem, project, dim, extra = spec
    tdir = os.path.join(TESTSUITE, refdir)
    text = open(os.path.join(tdir, f"input.txt.{dim}")).read()
    if extra:
        text = text.rstrip("\n") + "\n" + "\n".join(extra) + "\n"
    proj = P.Project(project)
    assert proj.codedim == dim
    u = run_uniform(project, text)
    kidx, uk, vk = compress(proj, u)
    head, wlog = read_wlog(os.path.join(tdir, "ref", f"{stem}.wlog.ref"))
    cmp = read_cmp(os.path.join(tdir, "ref", f"{stem}.cmp.ref"))
    dt_eF = head["dt*eF"]
    steps = wlog[1, 1] / dt_eF
    fx = dict(project=np.array(project), codedim=np.int32(dim), nwf=np.int32(u["nwf"]),
              spinsymmetry=np.int32(u["spinsymmetry"]), meta=u["meta"], En=u["En"], kperp=u["kperp"],
              cnt=u["cnt"], kidx=kidx, uk=uk, vk=vk, params=read_params(text), dt_eF=np.float64(dt_eF),
              timesteps=np.int32(round(steps)), measurements=np.int32(wlog.shape[0] - 1), wlog=wlog, cmp=cmp,
              ref_kF=np.float64(head["kF"]), ref_Effg=np.float64(head["Effg"]), ref_nwf=np.int32(head["nwf"]))
    # the reconstruction rebuilds the generator's states
    st = initial_states(proj, fx)
    err = np.abs(st - u["wf"]).max() / np.abs(u["wf"]).max()
    assert err < 1e-13, (case, err)
    assert abs(steps - round(steps)) < 1e-6, (case, steps)
    assert int(head["nwf"]) == u["nwf"], (case, head["nwf"], u["nwf"])
    os.makedirs(GOLDEN, exist_ok=True)
    np.savez_compressed(os.path.join(GOLDEN, f"{case}.npz"), **fx)
    print(f"{case}: {project} nwf={u['nwf']} dt*eF={dt_eF} steps/block={round(steps)} rebuild err={err:.1e}")


def main(argv):
    all_cases = cases()
    for case in argv or list(all_cases):
        make(case, all_cases[case])


if __name__ == "__main__":
    main(sys.argv[1:])
