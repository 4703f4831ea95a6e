"""Build one project's library: wslda_b200/_build/<project>/libwtd.so (sm_100a).

    python -m wslda_b200.build <project> [<project> ...]   (or "all")

Mirrors the reference's per-project build (hpc-engine/mk.td: one binary per project, lattice
and functional fixed at compile time) with nvcc only: no cmake, no JIT cache.
"""
import json
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def lib_path(project):
    return os.path.join(HERE, "_build", project, "libwtd.so")


def all_projects():
    d = os.path.join(HERE, "projects")
    return sorted(p for p in os.listdir(d) if os.path.isfile(os.path.join(d, p, "project.json")))


def _sources(project):
    pdir = os.path.join(HERE, "projects", project)
    files = [os.path.join(pdir, "predefines.h"), os.path.join(pdir, "problem-definition.h"),
             os.path.join(REPO, "include", "wtd.h"), os.path.join(REPO, "include", "wslda_td_compat.h")]
    for root in (CSRC, os.path.join(CSRC, "surface")):
        files += [os.path.join(root, f) for f in os.listdir(root) if f.endswith((".cu", ".cuh", ".h"))]
    return [f for f in files if os.path.exists(f)]


def build(project, force=False, verbose=False):
    pdir = os.path.join(HERE, "projects", project)
    with open(os.path.join(pdir, "project.json")) as fh:
        codedim = json.load(fh)["codedim"]
    out = lib_path(project)
    if not force and os.path.exists(out):
        t = os.path.getmtime(out)
        if all(os.path.getmtime(f) <= t for f in _sources(project)):
            return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "--expt-relaxed-constexpr", "-Xptxas", "-v" if verbose else "-O3",
           f"-DCODEDIM={codedim}", f"-I{pdir}", f"-I{os.path.join(CSRC, 'surface')}", f"-I{CSRC}",
           f"-I{os.path.join(REPO, 'include')}", os.path.join(CSRC, "wtd_project.cu"), "-o", out + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {project}:\n{r.stderr[-6000:]}")
    os.replace(out + ".tmp", out)
    if verbose:
        print(r.stderr)
    return out


def main(argv):
    names = argv or ["all"]
    if names == ["all"]:
        names = all_projects()
    force = os.environ.get("WTD_FORCE_BUILD") == "1"
    with ThreadPoolExecutor(max_workers=min(8, len(names))) as ex:
        for name, path in zip(names, ex.map(lambda n: build(n, force=force), names)):
            print(f"{name}: {path}")


if __name__ == "__main__":
    main(sys.argv[1:])
