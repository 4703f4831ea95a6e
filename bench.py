"""Throughput of the TD-(A)SLDA/BdG step on B200: qp-state*steps/s.

Workload: 2D TD-SLDA, 64x64 lattice (dx=1, periodic), 8192 (u, v) states,
seeded Gaussian QR-orthonormalised, harmonic trap omega=0.04, vortex Delta_ext, AB5AM5, FP64.
A step is one full ABM predictor-corrector step of every state (both stream passes, both
density reductions and both functional evaluations).

    python bench.py [--gpus N --steps K --warmup W] [--impl wtd|reference] [--workload c2]

Arms:
  wtd        this library (libwtd.so through its C ABI); prints one JSON line with value
             (device-timed, inputs resident), e2e (host buffers through the public API),
             roofline of the dominant kernel, cpu_baseline (oracle port on host cores),
             the FP32-mixed forms and the reference's own CUDA kernels on the same GPU.
  reference  the reference's step on the host cores (the CPU oracle port, all threads), on a
             bounded sample of the same workload.
Multi-GPU (torchrun): the workload's states are sharded over ranks in contiguous blocks (strong
scaling: one physical system of a fixed state count); after every density reduction NCCL sums
the partial densities over ranks on the context stream (the step's one exchange), and the
per-rank device time is max-reduced.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests"))

WORKLOADS = {
    "c2": dict(project="c2_slda2d", nwf=8192, desc="2D TD-SLDA 64x64, 8192 states, AB5AM5, trap omega=0.04, vortex Delta_ext"),
    "c1": dict(project="c1_bdg1d", nwf=256, desc="1D TD-BdG NX=128, 256 states, AB3AM4"),
    "c4": dict(project="c4_bdg2d", nwf=4608, desc="2D TD-BdG 48x48, 4608 states, AB3AM4, stirrer"),
    "c3": dict(project="c3_aslda3d", nwf=12000, desc="3D TD-ASLDA 32^3, 12000 states, AB5AM5, 5% spin imbalance, "
               "Delta_ext 0.2 with 1% noise (plane/pencil path)", forms=("fp64", "mixed_h64")),
}


# DRAM bytes (read + write) per state of the FP64 passes, from one ncu capture of the same
# kernel on the same lattice (profiles/wtd_fused_pass_c2_slda2d_64x64.md: 1024 states, pass A
# 1203 MB, pass B 437 MB); traffic per launch scales with the states processed
TRAFFIC_PER_STATE = {"c2_slda2d": {"pass_a": 1203152896 / 1024, "pass_b": 436638720 / 1024}}

# bounded CPU samples of each workload (states, steps): about 10-30 s on the host cores
CPU_SAMPLE = {"c2": (1024, 40), "c1": (256, 4000), "c4": (1024, 60), "c3": (128, 12)}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region: the sampler is running (its
    first sample seen) before the region starts, and one sample after its end is kept."""

    def __init__(self, index=0):
        self.index, self.samples, self.proc, self.th = index, [], None, None
        self.t0 = self.t1 = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
            t_wait = time.monotonic() + 5.0
            while not self.samples and time.monotonic() < t_wait:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.monotonic()
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append((time.monotonic(), parts))

    def __exit__(self, *a):
        self.t1 = time.monotonic()
        if self.proc:
            n = len(self.samples)
            t_wait = time.monotonic() + 1.0
            while len(self.samples) == n and time.monotonic() < t_wait:
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        inside = [p for t, p in self.samples if self.t0 is not None and t >= self.t0]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in inside if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in inside if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in inside for k in range(4) if s[3 + k].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside),
                "timed_region_s": round((self.t1 or self.t0) - self.t0, 3)}


def make_inputs(name, nwf, device_qr=True):
    """Seeded inputs; the QR of the (2N x S) Gaussian runs on the GPU for large S."""
    from wslda_b200 import projects as P
    proj = P.Project(name)
    seed = P.config_seed(name)
    n2 = 2 * proj.numel
    if device_qr and nwf * n2 > 4_000_000:
        import torch
        rng = np.random.Generator(np.random.PCG64(seed))
        a = rng.standard_normal((n2, nwf)) + 1j * rng.standard_normal((n2, nwf))
        t = torch.from_numpy(a).cuda()
        del a
        q, _ = torch.linalg.qr(t)
        q = q / np.sqrt(proj.dv)
        y = torch.cat([q[: proj.numel, :].T, q[proj.numel:, :].T], 0).contiguous().reshape(-1).cpu().numpy()
        del t, q
        torch.cuda.empty_cache()
    else:
        y = P.make_states(proj, nwf, seed)
    params = P.stirrer_params(proj, seed) if proj.cfg.get("stirrer_params") else proj.params
    return proj, dict(states=y, pots=P.make_potentials(proj), occ=P.make_occupations(nwf), params=params,
                      extra=P.make_extra(proj, seed))


def pass_bytes(proj, precision):
    """Algorithmic HBM bytes per state of pass A and pass B (compulsory stream traffic)."""
    by = 16 if precision == 0 else 8
    bh = 8 if precision == 2 else 16
    q = proj.nhist - 1
    n2 = 2 * proj.numel
    a = n2 * (by + q * bh + bh + by + bh)  # read y, q history; write f_k, y_pred, P
    b = n2 * (by + bh + by)               # read y_pred, P; write y
    return a, b


def run_wtd(args, rank, world):
    import torch
    from wslda_b200 import TDRun
    wl = WORKLOADS[args.workload]
    name = wl["project"]
    nwf_total = args.nwf or wl["nwf"]
    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    dev = torch.cuda.current_device()
    proj, d = make_inputs(name, nwf_total)
    if world > 1:
        # one system of nwf_total states, a contiguous block per rank (getnwfip); the density
        # partials are summed over ranks by NCCL after every density reduction
        from wslda_b200.sharding import shard_rows, shard_vector
        d["states"] = shard_rows(d["states"], nwf_total, proj.numel, world, rank)
        d["occ"] = shard_vector(d["occ"], nwf_total, world, rank)
    nwf = len(d["occ"])
    res = {}
    forms = [("fp64", 0)] + ([("mixed_h64", 1), ("mixed_h32", 2)] if not args.fp64_only else [])
    forms = [f for f in forms if f[0] in wl.get("forms", ("fp64", "mixed_h64", "mixed_h32"))]
    base_precision = 0
    for label, prec in forms:
        r = TDRun(name, nwf, precision=prec, device=dev)
        r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
        if world > 1:
            from wslda_b200.sharding import attach_nccl
            attach_nccl(r, rank, world)
        r.initial_measurement()
        r.steps(args.warmup)
        r.sync()
        stream = torch.cuda.ExternalStream(r.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        r.set_timing(True)
        launches0 = r.launches()
        with ClockSampler(dev) as clk:
            e0.record(stream)
            r.steps(args.steps)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ta, tb, na, nb = r.pass_times()
        launches = r.launches() - launches0
        t = torch.tensor([ms], device="cuda")
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        dens = r.densities()
        res[label] = dict(ms=ms, ms_a=ta / max(na, 1), ms_b=tb / max(nb, 1), launches=launches,
                          clocks=clk.summary(), dens=dens, energy=r.energy(), prec=prec)
        if label == "fp64":
            # e2e: public API with host buffers, pinned; H2D of the states and D2H of the densities
            # and energies are inside the timed region
            hst = torch.from_numpy(d["states"].view(np.float64)).pin_memory()
            hd = torch.empty(12 * proj.numel, dtype=torch.float64).pin_memory()
            r.set_timing(False)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0.record(stream)
            r.lib.wtd_upload_states(r.h, hst.numpy().ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)))
            r.initial_measurement()
            r.steps(args.steps)
            r.densities(out=hd.numpy())
            en = r.energy()
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_ms = e0.elapsed_time(e1)
            wall = (time.perf_counter() - t0) * 1e3
            res["e2e"] = dict(ms=max(e2e_ms, 0.0), wall_ms=wall, h2d=hst.numel() * 8, d2h=hd.numel() * 8 + 11 * 8)
        if label == "fp64" and world == 1 and (args.adjoint or args.workload == "c4") and proj.cfg.get("stirrer_params"):
            res["adjoint"] = time_adjoint(r, proj, d, stream, args.adjoint_steps)
        r.close()
    return proj, nwf, res


def time_adjoint(r, proj, d, stream, steps=0):
    """device time of the loss-only forward and of the gradient call (forward, segment
    recompute, reverse sweep) over the project's optimal-control horizon: with the checkpoint
    interval chosen by the library (0: records of every step when they fit) and with the
    project's interval; each gradient timed on its second call (workspace already allocated)"""
    import torch
    ns = steps or proj.cfg.get("steps", 200)
    K = min(proj.cfg.get("checkpoint_every", 20), ns)
    npar = proj.cfg["stirrer_params"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(**kw):
        r.upload_states(d["states"])
        torch.cuda.synchronize()
        e0.record(stream)
        loss, g = r.adjoint(ns, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), loss, g

    timed()
    tf, loss, _ = timed()
    out = {"steps": ns, "nparam": npar, "ms_forward_with_loss": tf}
    for label, k in (("auto", 0), (f"K{K}", K)):
        t_first = timed(nparam=npar, checkpoint_every=k)[0]
        tg, loss_g, g = timed(nparam=npar, checkpoint_every=k)
        out[label] = {"checkpoint_every": k or "auto", "ms_gradient": tg, "ms_first_call": t_first,
                      "gradient_over_forward": tg / tf}
        r.adjoint_release()
    out["loss"] = loss
    out["grad_norm"] = float(np.linalg.norm(g))
    return out

def reference_cuda(name, nwf, steps):
    """The reference's own kernels (hpc-engine/*.cu built for sm_100a) on the same GPU."""
    import ctypes
    so = os.path.join(REPO, "oracle", "_ref", name, "libref.so")
    if not os.path.exists(so):
        return None
    from wslda_b200 import projects as P
    proj, d = make_inputs(name, nwf)
    lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.refh_run.argtypes = ([ctypes.c_int] + [dp] * 5 + [ctypes.POINTER(ctypes.c_int)] + [ctypes.c_double] * 7 +
                             [dp, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [dp] * 7)
    c = proj.constants()
    ms = np.zeros(1)
    ex = np.ascontiguousarray(d["extra"])
    y = d["states"]
    rc = lib.refh_run(nwf, y.view(np.float64).ctypes.data_as(dp), d["pots"].ctypes.data_as(dp), d["occ"].ctypes.data_as(dp),
                      None, None, None, c["mu_a"], c["mu_b"], c["ec"], c["t0"], c["dt"], c["kF"], c["sclgth"],
                      np.ascontiguousarray(d["params"]).ctypes.data_as(dp), ex.ctypes.data if ex.size else None, ex.nbytes,
                      steps, 1, 0, None, None, None, None, None, None, ms.ctypes.data_as(dp))
    if rc != 0:
        return {"error": f"refh_run rc={rc}"}
    return {"ms_per_step": float(ms[0]), "value": nwf / (float(ms[0]) * 1e-3)}


def cpu_baseline(name, nwf_sample, steps, threads=None):
    """CPU oracle port on the host cores: bounded sample of the workload."""
    from parity_util import inputs
    from oracle_lib import Oracle
    threads = threads or os.cpu_count()
    proj, d = inputs(name, nwf_sample)
    o = Oracle(name, threads=threads)
    o.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    o.initial_measurement()
    t0 = time.perf_counter()
    o.steps(steps)
    dt = time.perf_counter() - t0
    return {"value": nwf_sample * steps / dt, "unit": "qp-state*steps/s", "cores": threads, "kind": "port",
            "sample": f"{nwf_sample} of the workload's states x {steps} steps, {dt:.1f} s, oracle/wtd_oracle.cpp"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="wtd", choices=["wtd", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--fp64-only", action="store_true")
    ap.add_argument("--nwf", type=int, default=0, help="override the workload's state count (small profiling cases)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-refcuda", action="store_true")
    ap.add_argument("--adjoint", action="store_true", help="also time the adjoint gradient (stirrer projects)")
    ap.add_argument("--adjoint-steps", type=int, default=0, help="adjoint horizon (default: the project's steps)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    wl = WORKLOADS[args.workload]
    metric = "qp-state*steps/s"
    cfg = {"workload": wl["desc"], "project": wl["project"], "states": args.nwf or wl["nwf"], "precision": "fp64",
           "l2": "inputs larger than L2 (state arrays of GBs)", "parallelism": f"states sharded over {world} GPU(s)"}

    if args.impl == "reference":
        if rank != 0:
            return
        sample = CPU_SAMPLE[args.workload]
        vals = []
        for _ in range(args.warmup if False else 0):
            pass
        cb = None
        t0 = time.perf_counter()
        for k in range(max(1, min(args.steps, 3))):
            cb = cpu_baseline(wl["project"], sample[0], sample[1])
            vals.append(cb["value"])
        v = float(np.median(vals))
        cb["value"] = v
        line = {"impl": "reference", "metric": metric, "value": v, "unit": metric, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": wl["nwf"] / v * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": cfg, "cpu_baseline": cb,
                "e2e": {"value": v, "unit": metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference has no CPU implementation of the TD step (td codes require GPUs); this arm "
                        "times the CPU restatement of the reference step (oracle port) on all host threads",
                "wall_s": round(time.perf_counter() - t0, 1)}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    proj, nwf, res = run_wtd(args, rank, world)
    nwf_total = args.nwf or wl["nwf"]
    if rank != 0:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
        return
    hbm, peak_kind = peaks()
    f = res["fp64"]
    value = nwf_total * args.steps / (f["ms"] * 1e-3)
    ba, bb = pass_bytes(proj, 0)
    # the fused path times its passes; the plane/pencil path (3D from 32^3) runs a chain of
    # kernels per half step and reports the whole step against the same compulsory bytes
    fused = f["ms_a"] > 0
    achieved = (ba * nwf / (f["ms_a"] * 1e-3) if fused else (ba + bb) * nwf * args.steps / (f["ms"] * 1e-3)) / 1e9
    line = {
        "metric": metric, "value": value, "unit": metric, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": f["ms"] / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded PCG64 Gaussian states, QR-orthonormalised)", "config": cfg,
        "gpu_launches": int(f["launches"]),
        "roofline": {"bound": "hbm", "kernel": ("wtd_fused_pass<PASS=0> (H psi + ABM predictor)" if fused else
                                                "whole step of the plane/pencil path (compulsory bytes of both half steps)"),
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "traffic": (TRAFFIC_PER_STATE[proj.name]["pass_a"] * nwf if proj.name in TRAFFIC_PER_STATE else None),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of a 1024-state capture, scaled by states",
                     "alg_bytes_per_launch": ba * nwf,
                     "pass_b": ({"achieved": bb * nwf / (f["ms_b"] * 1e-3) / 1e9, "alg_bytes_per_launch": bb * nwf}
                                if fused else None),
                     "ms_pass_a": f["ms_a"], "ms_pass_b": f["ms_b"]},
        "clocks": f["clocks"],
    }
    if "e2e" in res:
        e = res["e2e"]
        line["e2e"] = {"value": nwf_total * args.steps / (e["ms"] * 1e-3), "unit": metric,
                       "h2d_bytes_per_step": e["h2d"] / args.steps, "d2h_bytes_per_step": e["d2h"] / args.steps,
                       "ms": e["ms"], "definition": "upload states (pinned) + initial measurement + K steps + "
                       "download densities + energy, per K steps"}
    forms = {}
    for label in ("mixed_h64", "mixed_h32"):
        if label in res:
            m = res[label]
            d64 = f["dens"]
            n = proj.numel
            rho = np.concatenate([d64[2 * n:3 * n], d64[7 * n:8 * n]])
            rho_m = np.concatenate([m["dens"][2 * n:3 * n], m["dens"][7 * n:8 * n]])
            forms[label] = {"value": nwf_total * args.steps / (m["ms"] * 1e-3),
                            "speedup_vs_fp64": f["ms"] / m["ms"],
                            "density_rel_l2_err_vs_fp64": float(np.linalg.norm(rho_m - rho) / np.linalg.norm(rho)),
                            "energy_rel_err_vs_fp64": float(abs(m["energy"][:7].sum() - f["energy"][:7].sum()) / abs(f["energy"][:7].sum())),
                            "ms_pass_a": m["ms_a"], "ms_pass_b": m["ms_b"]}
    if forms:
        line["precision_forms"] = forms
    if "adjoint" in res:
        line["adjoint"] = res["adjoint"]
    if not args.no_refcuda and world == 1:
        try:
            line["reference_cuda"] = reference_cuda(proj.name, nwf, max(2, min(args.steps, 10)))
            if line["reference_cuda"] and "value" in line["reference_cuda"]:
                line["reference_cuda"]["note"] = "hpc-engine/*.cu compiled for sm_100a + oracle/ref_harness.cu, same GPU, same inputs"
        except Exception as ex:  # reported, not fatal
            line["reference_cuda"] = {"error": str(ex)[:200]}
    if not args.no_cpu and world == 1:
        sample = CPU_SAMPLE[args.workload]
        line["cpu_baseline"] = cpu_baseline(proj.name, *sample)
    print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
