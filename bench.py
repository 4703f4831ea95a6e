"""Throughput of the TD-(A)SLDA/BdG step on B200: qp-state*steps/s.

Workload: 2D TD-SLDA, 64x64 lattice (dx=1, periodic), 8192 (u, v) states,
seeded Gaussian QR-orthonormalised, harmonic trap omega=0.04, vortex Delta_ext, AB5AM5, FP64.
A step is one full ABM predictor-corrector step of every state (both stream passes, both
density reductions and both functional evaluations).

    python bench.py [--gpus N --steps K --warmup W] [--impl wtd|reference] [--workload c2]

Arms:
  wtd        this library (libwtd.so through its C ABI); prints one JSON line with value
             (device-timed, inputs resident), e2e (host buffers through the public API),
             roofline of the dominant kernel, cpu_baseline (the host-core baseline below),
             the FP32-mixed forms, the reference's own CUDA kernels on the same GPU and inputs,
             the 3D comparisons (C3, C5) and the adjoint's cost (C4).
  reference  the step on the host cores with all threads, on a bounded sample of the same
             workload: the state derivatives from the reference's lib/wderiv (compiled
             unmodified over an FFTW-API shim) plus the oracle's local update; the oracle port
             alone where that build is absent.
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
               "Delta_ext 0.2 with 1% noise (3D line path)"),
}
C5 = dict(project="c5_slda3d", nwf=20000, desc="3D TD-SLDA 48^3 vortex with a moving Gaussian stirrer, AB3AM4, "
          "complex64 states and history (3D line path)")


# DRAM bytes (read + write) per state of the FP64 passes, from one ncu capture of the same
# kernels on the same lattice (1024 states: pass A 1203 MB, pass B 437 MB of
# dram__bytes_read.sum + dram__bytes_write.sum); traffic per launch scales with the states processed
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


def total_energy(e):
    """E_kin + E_pot + E_pair + E_curr + E_ext (V, Delta, v): the first 7 of the 11 energy items"""
    return float(np.asarray(e)[:7].sum())


def timed_blocks(r, stream, steps, blocks, dev, world):
    """device time of `blocks` blocks of exactly `steps` steps each (CUDA events on the context
    stream, barrier + synchronize around every block, max over ranks), clocks sampled during
    all blocks; the pass times are accumulated over the blocks"""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms_blocks, launches = [], []
    r.set_timing(True)
    with ClockSampler(dev) as clk:
        for _ in range(blocks):
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            l0 = r.launches()
            e0.record(stream)
            r.steps(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            if world > 1:
                t = torch.tensor([ms], device="cuda")
                torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
                ms = float(t.item())
            ms_blocks.append(ms)
            launches.append(r.launches() - l0)
    ta, tb, na, nb = r.pass_times()
    r.set_timing(False)
    return dict(ms_blocks=ms_blocks, ms=float(np.median(ms_blocks)), ms_a=ta / max(na, 1), ms_b=tb / max(nb, 1),
                launches=int(np.median(launches)), clocks=clk.summary())


def energy_drift(name, nwf, d, precision, steps, dev):
    """|E(t) - E(0)| / |E(0)| over `steps` steps from the initial measurement, scaled to 1000
    steps (time-independent fields conserve E); also returns the final densities"""
    from wslda_b200 import TDRun
    r = TDRun(name, nwf, precision=precision, device=dev)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    r.initial_measurement()
    e0 = total_energy(r.energy())
    r.steps(steps)
    e1 = total_energy(r.energy())
    dens = r.densities()
    r.close()
    return dict(steps=steps, e0=e0, e_t=e1, drift_per_1000_steps=abs(e1 - e0) / abs(e0) * 1000.0 / steps), dens


# nominal CUDA-core peaks of a B200 at its 1965 MHz maximum clock (148 SMs; 64 FP64 and 128
# FP32 fused multiply-adds per SM per clock): the denominators of the flop rooflines below
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e-3
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e-3
DENS_BLOCKS = ("nu", "rho_a", "tau_a", "j_a_x", "j_a_y", "j_a_z", "rho_b", "tau_b", "j_b_x", "j_b_y", "j_b_z")


def dens_errs(dens, ref, n):
    """relative L2 error per density block (the reference's 12-block layout; nu is complex)"""
    out = {}
    offs = [(0, 2 * n)] + [((2 + k) * n, (3 + k) * n) for k in range(10)]
    for name, (a, b) in zip(DENS_BLOCKS, offs):
        nr = float(np.linalg.norm(ref[a:b]))
        if nr > 0:
            out[name] = float(np.linalg.norm(dens[a:b] - ref[a:b]) / nr)
    return out


def fft_flops(proj):
    """algorithmic flops of one qp-state-step's transforms: 5 N log2 N per complex transform,
    14 transforms per component and step with variable mass (ASLDA), 4 with constant mass"""
    import math
    n = proj.numel
    per = 14 if not proj.const_mass else 4
    return 5.0 * n * math.log2(n) * per * 2


def rho_err(dens, ref, n):
    """relative L2 error of (rho_a, rho_b)"""
    rho = np.concatenate([ref[2 * n:3 * n], ref[7 * n:8 * n]])
    got = np.concatenate([dens[2 * n:3 * n], dens[7 * n:8 * n]])
    return float(np.linalg.norm(got - rho) / np.linalg.norm(rho))


def run_wtd(args, rank, world):
    import torch
    from wslda_b200 import TDRun, WtdError
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
    for label, prec in forms:
        try:
            r = TDRun(name, nwf, precision=prec, device=dev)
        except WtdError as ex:
            res[label] = {"unsupported": str(ex)}
            continue
        r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
        if world > 1:
            from wslda_b200.sharding import attach_nccl
            attach_nccl(r, rank, world)
        r.initial_measurement()
        r.steps(args.warmup)
        r.sync()
        stream = torch.cuda.ExternalStream(r.stream())
        t = timed_blocks(r, stream, args.steps, args.blocks, dev, world)
        t.update(dens=r.densities(), energy=r.energy(), prec=prec)
        res[label] = t
        if label == "fp64":
            # e2e: public API with host buffers, pinned; H2D of the states and D2H of the densities
            # and energies are inside the timed region
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            hst = torch.from_numpy(d["states"].view(np.float64)).pin_memory()
            hd = torch.empty(12 * proj.numel, dtype=torch.float64).pin_memory()
            e2e_blocks = []
            for _ in range(args.blocks):
                torch.cuda.synchronize()
                e0.record(stream)
                r.lib.wtd_upload_states(r.h, hst.numpy().ctypes.data_as(__import__("ctypes").POINTER(__import__("ctypes").c_double)))
                r.initial_measurement()
                r.steps(args.steps)
                r.densities(out=hd.numpy())
                r.energy()
                e1.record(stream)
                torch.cuda.synchronize()
                e2e_blocks.append(max(e0.elapsed_time(e1), 0.0))
            res["e2e"] = dict(ms=float(np.median(e2e_blocks)), ms_blocks=e2e_blocks, h2d=hst.numel() * 8,
                              d2h=hd.numel() * 8 + 11 * 8)
        if label == "fp64" and world == 1 and (args.adjoint or args.workload == "c4") and proj.cfg.get("stirrer_params"):
            res["adjoint"] = time_adjoint(r, proj, d, stream, args.adjoint_steps)
        r.close()
        if world == 1 and args.drift_steps > 0 and wl.get("drift", False):
            res[label]["drift"], res[label]["drift_dens"] = energy_drift(name, nwf, d, prec, args.drift_steps, dev)
    return proj, nwf, d, res


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
        # the call split at the loss: the forward with its checkpoints, and the reverse sweep
        # (segment recomputation and adjoint steps) — the adjoint proper
        ms_fwd, ms_rev = r.adjoint_times()
        out[label] = {"checkpoint_every": k or "auto", "ms_gradient": tg, "ms_first_call": t_first,
                      "gradient_over_forward": tg / tf, "ms_forward_in_call": ms_fwd, "ms_reverse_sweep": ms_rev,
                      "adjoint_over_forward": ms_rev / tf}
        r.adjoint_release()
    out["loss"] = loss
    out["grad_norm"] = float(np.linalg.norm(g))
    return out

def reference_cuda(name, nwf, steps, inp=None):
    """The reference's own kernels (hpc-engine/*.cu built for sm_100a) on the same GPU and the same
    inputs: initial measurement and one measurement block of `steps` steps (gradients on its last
    step), as the reference driver runs them (pca.c:939-1586).  Returns the device time per step
    and the block's densities and energies."""
    import ctypes
    so = os.path.join(REPO, "oracle", "_ref", name, "libref.so")
    if not os.path.exists(so):
        return None
    proj, d = inp if inp is not None else make_inputs(name, nwf)
    lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.refh_run.argtypes = ([ctypes.c_int] + [dp] * 5 + [ctypes.POINTER(ctypes.c_int)] + [ctypes.c_double] * 7 +
                             [dp, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [dp] * 7)
    c = proj.constants()
    ms = np.zeros(1)
    dens = np.zeros(12 * proj.numel)
    energy = np.zeros(11)
    ex = np.ascontiguousarray(d["extra"])
    y = d["states"]
    rc = lib.refh_run(nwf, y.view(np.float64).ctypes.data_as(dp), d["pots"].ctypes.data_as(dp), d["occ"].ctypes.data_as(dp),
                      None, None, None, c["mu_a"], c["mu_b"], c["ec"], c["t0"], c["dt"], c["kF"], c["sclgth"],
                      np.ascontiguousarray(d["params"]).ctypes.data_as(dp), ex.ctypes.data if ex.size else None, ex.nbytes,
                      steps, 1, 0, None, dens.ctypes.data_as(dp), None, energy.ctypes.data_as(dp), None, None,
                      ms.ctypes.data_as(dp))
    if rc != 0:
        return {"error": f"refh_run rc={rc}"}
    return {"ms_per_step": float(ms[0]), "value": nwf / (float(ms[0]) * 1e-3), "steps": steps, "dens": dens,
            "energy": energy}


def parity_full_size(name, nwf, steps, dev, inp=None, ref=None):
    """This library (FP64) against the reference's own kernels at the benchmarked state count:
    the same seeded inputs, initial measurement and `steps` steps each; densities (relative L2
    per block), the 11 energy items and the particle numbers.  The reference is the one-rank
    restatement of pca.c:939-1586 over its unmodified kernels."""
    from wslda_b200 import TDRun
    from parity_util import density_errors
    proj, d = inp if inp is not None else make_inputs(name, nwf)
    if ref is None:
        ref = reference_cuda(name, nwf, steps, (proj, d))
    if not ref or "dens" not in ref:
        return {"error": "reference kernels unavailable" if not ref else ref.get("error")}
    r = TDRun(name, nwf, precision=0, device=dev)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    r.initial_measurement()
    r.steps(steps)
    dens, en = r.densities(), r.energy()
    r.close()
    derr = density_errors(dens, ref["dens"], proj.numel)
    e_ref = ref["energy"]
    eterm = {k: float(abs(en[i] - e_ref[i]) / max(abs(e_ref[i]), 1e-300))
             for i, k in enumerate(["E_kin", "E_pot", "E_pair", "E_curr", "E_ext_V", "E_ext_delta", "E_ext_v",
                                    "N_a", "N_b", "L_za", "L_zb"]) if abs(e_ref[i]) > 1e-12 * abs(e_ref[:7]).max()}
    worst = max(max(derr.values()), max(eterm.values()))
    return {"states": nwf, "steps": steps, "density_rel_l2": {k: float(v) for k, v in derr.items()},
            "energy_rel": eterm, "worst": worst, "tolerance": 1e-10, "pass": bool(worst < 1e-10),
            "against": "the reference's CUDA kernels (hpc-engine/*.cu, sm_100a) through oracle/ref_harness.cu, "
                       "same GPU, same inputs"}


def c3_comparison(args, dev):
    """The 3D TD-ASLDA workload (32^3, 12,000 states, AB5AM5): FP64 against the FP32-mixed forms.
    Each form is timed over `blocks` blocks of `c3_steps` steps at the full state count; its
    density error against FP64 after those steps, and the energy drift of every form over
    `c3_drift_steps` steps on a reduced state count (a smaller system of the same lattice and
    functional, stated in the result)."""
    import torch
    from wslda_b200 import TDRun, WtdError
    wl = WORKLOADS["c3"]
    name, nwf = wl["project"], args.c3_nwf or wl["nwf"]
    proj, d = make_inputs(name, nwf)
    hbm, peak_kind = peaks()
    out = {"workload": wl["desc"], "states": nwf, "steps": args.c3_steps, "blocks": args.blocks, "forms": {}}
    dens64 = None
    for label, prec in (("fp64", 0), ("mixed_h64", 1), ("mixed_h32", 2)):
        try:
            r = TDRun(name, nwf, precision=prec, device=dev)
            r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
            r.initial_measurement()
            r.steps(args.warmup)
            r.sync()
        except WtdError as ex:
            out["forms"][label] = {"unsupported": str(ex)}
            try:
                r.close()
            except Exception:
                pass
            continue
        stream = torch.cuda.ExternalStream(r.stream())
        t = timed_blocks(r, stream, args.c3_steps, args.blocks, dev, 1)
        dens = r.densities()
        r.close()
        ba, bb = pass_bytes(proj, prec)
        f = {"value": nwf * args.c3_steps / (t["ms"] * 1e-3), "ms_per_step": t["ms"] / args.c3_steps,
             "ms_blocks": t["ms_blocks"], "hbm_gbs_compulsory": (ba + bb) * nwf * args.c3_steps / (t["ms"] * 1e-3) / 1e9,
             "launches_per_block": t["launches"], "clocks": t["clocks"]}
        f["roofline_frac"] = f["hbm_gbs_compulsory"] / hbm
        # the transforms' flops against the CUDA-core peak of the arithmetic precision (FP64 for
        # the FP64 form, FP32 for the mixed forms): the C3 step is transform- and latency-bound
        tf = fft_flops(proj) * f["value"] / 1e12
        fpk = FP64_PEAK_TFLOPS if prec == 0 else FP32_PEAK_TFLOPS
        f["flops"] = {"alg_flops_per_state_step": fft_flops(proj), "achieved_tflops": tf, "peak_tflops": fpk,
                      "peak_source": "nominal (148 SMs x FMA/clk x 1965 MHz)", "frac": tf / fpk}
        if label == "fp64":
            dens64 = dens
        else:
            f["speedup_vs_fp64"] = out["forms"]["fp64"]["value"] and f["value"] / out["forms"]["fp64"]["value"]
            f["density_rel_l2_err_vs_fp64"] = rho_err(dens, dens64, proj.numel)
            f["density_rel_l2_err_vs_fp64_by_block"] = dens_errs(dens, dens64, proj.numel)
        out["forms"][label] = f
        torch.cuda.empty_cache()
    out["peak_gbs"] = hbm
    out["peak_source"] = peak_kind
    if args.c3_drift_steps > 0:
        nd = args.c3_drift_nwf
        pd, dd = make_inputs(name, nd)
        drift = {"states": nd, "steps": args.c3_drift_steps}
        d64 = None
        for label, prec in (("fp64", 0), ("mixed_h64", 1), ("mixed_h32", 2)):
            if "unsupported" in out["forms"].get(label, {}):
                continue
            res, dens = energy_drift(name, nd, dd, prec, args.c3_drift_steps, dev)
            if label == "fp64":
                d64 = dens
            else:
                res["density_rel_l2_err_vs_fp64"] = rho_err(dens, d64, pd.numel)
            drift[label] = res
        out["drift"] = drift
    if args.c3_parity_nwf > 0 and not args.no_refcuda:
        np_ = args.c3_parity_nwf
        inp = make_inputs(name, np_)
        ref = reference_cuda(name, np_, args.c3_parity_steps, inp)
        out["parity_full_size"] = parity_full_size(name, np_, args.c3_parity_steps, dev, inp, ref)
        if ref and "value" in ref:
            out["reference_cuda"] = {"value": ref["value"], "ms_per_step": ref["ms_per_step"], "states": np_,
                                     "steps": ref["steps"]}
    return out


def cpu_baseline(name, nwf_sample, steps, threads=None, single_thread=True):
    """The step on the host cores, bounded sample of the workload.  Where it is built (it ships
    in oracle/_ref/<project>/liboracle_wderiv.so), the spectral derivatives are the reference's
    own CPU library, lib/wderiv/c/wderiv.c compiled unmodified over an in-repo FFTW3-API shim
    (FFTW is not installed), with the oracle's restatement of the local update, densities,
    functional and ABM; else the oracle port alone.  OpenMP over states on all host threads,
    and a one-thread figure of the same sample."""
    import platform
    from parity_util import inputs
    from oracle_lib import Oracle
    threads = threads or os.cpu_count()
    so = os.path.join(REPO, "oracle", "_ref", name, "liboracle_wderiv.so")
    variant = "wderiv" if os.path.exists(so) else None
    proj, d = inputs(name, nwf_sample)

    def run(th, nsteps):
        o = Oracle(name, threads=th, variant=variant)
        o.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
        o.initial_measurement()
        t0 = time.perf_counter()
        o.steps(nsteps)
        return time.perf_counter() - t0

    dt = run(threads, steps)
    cpu = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as fh:
            cpu = next((l.split(":", 1)[1].strip() for l in fh if l.startswith("model name")), cpu)
    except Exception:
        pass
    out = {"value": nwf_sample * steps / dt, "unit": "qp-state*steps/s", "cores": threads,
           "kind": "reference" if variant else "port", "cpu": cpu,
           "sample": f"{nwf_sample} of the workload's states x {steps} steps, {dt:.1f} s, " +
                     ("wderiv (lib/wderiv/c/wderiv.c) + in-repo FFT shim (FFTW unavailable) + the oracle's local update"
                      if variant else "oracle/wtd_oracle.cpp")}
    if single_thread:
        s1 = max(1, steps // 8)
        dt1 = run(1, s1)
        out["value_1_thread"] = nwf_sample * s1 / dt1
        out["sample_1_thread"] = f"{nwf_sample} states x {s1} steps, {dt1:.1f} s"
    return out


def c5_scale(args, dev):
    """The 3D TD-SLDA vortex workload (48^3, AB3AM4) in the all-FP32 storage form (complex64
    states and history, FP32 transforms, FP64 sums) at the largest state count that fits the
    GPU, up to the workload's 20,000; and its error against FP64 on a subset of states."""
    import torch
    from wslda_b200 import TDRun, projects as P
    name = C5["project"]
    proj = P.Project(name)
    free, _ = torch.cuda.mem_get_info(dev)
    per_state = 2 * proj.numel * 8 * (1 + proj.nhist + 1)     # y, the ring, K_yz (complex64)
    nwf = int(min(C5["nwf"], args.c5_nwf or C5["nwf"], (free - (6 << 30)) // per_state))
    out = {"workload": C5["desc"], "states_requested": C5["nwf"], "states": nwf,
           "resident_bytes_per_state": per_state, "steps": args.c5_steps, "blocks": args.blocks}
    # the full state count as host FP64 would be 2 x 20,000 x 110,592 complex128 (70 GB) and its
    # QR beyond one GPU: the states are seeded Gaussian complex64 drawn on the device in chunks
    # (torch Philox, seed 20261203 + 5) straight into the context's state array; the initial
    # measurement normalises each state
    import ctypes
    seed = P.config_seed(name)
    hbm, _ = peaks()

    def timed_form(prec, ns):
        r = TDRun(name, ns, precision=prec, device=dev)
        sp = ctypes.c_void_p()
        r._check(r.lib.wtd_device_pointers(r.h, ctypes.byref(sp), None, None))
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        n2 = 2 * ns * proj.numel
        chunk = 1 << 27
        dt_, eb = (torch.float32, 8) if prec else (torch.float64, 16)
        for o in range(0, n2, chunk):
            m = min(chunk, n2 - o)
            z = torch.randn(2 * m, device="cuda", dtype=dt_, generator=g)
            r.lib.memcopy_gpu2gpu(ctypes.c_void_p(z.data_ptr()), ctypes.c_void_p(sp.value + eb * o), ctypes.c_size_t(eb * m))
            del z
        torch.cuda.synchronize()
        r.setup_fields(P.make_potentials(proj), P.make_occupations(ns), proj.params, P.make_extra(proj, seed))
        r.initial_measurement()
        r.steps(args.warmup)
        r.sync()
        stream = torch.cuda.ExternalStream(r.stream())
        t = timed_blocks(r, stream, args.c5_steps, args.blocks, dev, 1)
        r.close()
        torch.cuda.empty_cache()
        ba, bb = pass_bytes(proj, prec)
        res = {"states": ns, "value": ns * args.c5_steps / (t["ms"] * 1e-3), "ms_per_step": t["ms"] / args.c5_steps,
               "ms_blocks": t["ms_blocks"], "hbm_gbs_compulsory": (ba + bb) * ns * args.c5_steps / (t["ms"] * 1e-3) / 1e9,
               "clocks": t["clocks"]}
        res["roofline_frac"] = res["hbm_gbs_compulsory"] / hbm
        return res

    f32 = timed_form(2, nwf)
    f32.pop("states")
    out.update(f32)
    # the FP64 form on the same GPU, at the state count its resident arrays allow (the staged
    # path: states, ring and the derivative arrays); qp-state*steps/s is per state, so the two
    # rates compare directly
    if args.c5_fp64_nwf > 0:
        f64 = timed_form(0, args.c5_fp64_nwf)
        out["fp64"] = f64
        out["speedup_vs_fp64"] = out["value"] / f64["value"]
    # accuracy against FP64 on a subset of the workload
    ns = args.c5_err_nwf
    pe, de = make_inputs(name, ns)
    res = {}
    for label, prec in (("fp64", 0), ("mixed_h32", 2)):
        rr = TDRun(name, ns, precision=prec, device=dev)
        rr.setup(de["states"], de["pots"], de["occ"], de["params"], de["extra"])
        rr.initial_measurement()
        rr.steps(args.c5_err_steps)
        res[label] = (rr.densities(), rr.energy())
        rr.close()
    out["error_vs_fp64"] = {"states": ns, "steps": args.c5_err_steps,
                            "density_rel_l2": rho_err(res["mixed_h32"][0], res["fp64"][0], pe.numel),
                            "energy_rel": abs(total_energy(res["mixed_h32"][1]) - total_energy(res["fp64"][1])) /
                                          abs(total_energy(res["fp64"][1]))}
    return out


def adjoint_c4(args, dev):
    """Cost of the optimal-control gradient on the C4 workload (2D TD-BdG 48x48, 4608 states,
    200 steps, checkpoints every 20): the gradient call over the loss-only forward"""
    import torch
    from wslda_b200 import TDRun
    wl = WORKLOADS["c4"]
    proj, d = make_inputs(wl["project"], wl["nwf"])
    r = TDRun(wl["project"], wl["nwf"], precision=0, device=dev)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    stream = torch.cuda.ExternalStream(r.stream())
    out = time_adjoint(r, proj, d, stream, args.adjoint_steps)
    r.close()
    out["workload"] = wl["desc"]
    out["states"] = wl["nwf"]
    return out


def probe(args):
    """one form of one workload on one GPU: device time of --steps steps after the initial
    measurement and --warmup steps (the case the ncu captures of the line path run)"""
    import torch
    from wslda_b200 import TDRun
    wl = C5 if args.workload == "c5" else WORKLOADS[args.workload]
    nwf = args.nwf or wl["nwf"]
    proj, d = make_inputs(wl["project"], nwf)
    r = TDRun(wl["project"], nwf, precision=args.probe, device=0)
    r.setup(d["states"], d["pots"], d["occ"], d["params"], d["extra"])
    r.initial_measurement()
    r.steps(args.warmup)
    r.sync()
    stream = torch.cuda.ExternalStream(r.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    l0 = r.launches()
    e0.record(stream)
    r.steps(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"probe": wl["project"], "states": nwf, "precision": args.probe, "steps": args.steps,
           "path_3d": os.environ.get("WTD_3D_PATH", "default"), "ms_per_step": ms / args.steps,
           "value": nwf * args.steps / (ms * 1e-3), "unit": "qp-state*steps/s",
           "launches_per_step": (r.launches() - l0) / args.steps}
    r.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--blocks", type=int, default=3, help="timed blocks of --steps steps each; value is the median block")
    ap.add_argument("--impl", default="wtd", choices=["wtd", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS) + ["c5"],
                    help="c5 (reported inside the default run's line) only with --probe")
    ap.add_argument("--fp64-only", action="store_true")
    ap.add_argument("--nwf", type=int, default=0, help="override the workload's state count (small profiling cases)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-refcuda", action="store_true")
    ap.add_argument("--adjoint", action="store_true", help="also time the adjoint gradient (stirrer projects)")
    ap.add_argument("--adjoint-steps", type=int, default=0, help="adjoint horizon (default: the project's steps)")
    ap.add_argument("--drift-steps", type=int, default=1000, help="energy-drift run of every form (0: skip)")
    ap.add_argument("--parity-steps", type=int, default=10, help="full-size parity against the reference kernels (0: skip)")
    ap.add_argument("--extras", type=int, default=1, help="with the C2 workload at N=1: the C3 FP64-vs-mixed comparison "
                    "and the C4 adjoint cost (0: skip)")
    ap.add_argument("--c3-nwf", type=int, default=0)
    ap.add_argument("--c3-steps", type=int, default=10)
    ap.add_argument("--c3-drift-steps", type=int, default=1000)
    ap.add_argument("--c3-drift-nwf", type=int, default=1024)
    ap.add_argument("--c3-parity-nwf", type=int, default=4000)
    ap.add_argument("--c3-parity-steps", type=int, default=10)
    ap.add_argument("--c5-nwf", type=int, default=0)
    ap.add_argument("--c5-steps", type=int, default=3)
    ap.add_argument("--c5-err-nwf", type=int, default=256)
    ap.add_argument("--c5-err-steps", type=int, default=20)
    ap.add_argument("--c5-fp64-nwf", type=int, default=2000, help="states of the C5 FP64 comparison (0: skip)")
    ap.add_argument("--probe", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="time one precision form (0 FP64, 1 mixed H64, 2 mixed H32) of the workload for --steps "
                         "steps after --warmup, print one short JSON line and exit (the profiling case)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    args.blocks = max(args.blocks, 1)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    wl = WORKLOADS.get(args.workload, C5)
    metric = "qp-state*steps/s"
    cfg = {"workload": wl["desc"], "project": wl["project"], "states": args.nwf or wl["nwf"], "precision": "fp64",
           "l2": "inputs larger than L2 (state arrays of GBs)", "parallelism": f"states sharded over {world} GPU(s)"}

    if args.impl == "reference":
        if rank != 0:
            return
        sample = CPU_SAMPLE[args.workload]
        vals = []
        cb = None
        t0 = time.perf_counter()
        for k in range(max(1, min(args.steps, 3))):
            cb = cpu_baseline(wl["project"], sample[0], sample[1], single_thread=False)
            vals.append(cb["value"])
        v = float(np.median(vals))
        cb["value"] = v
        line = {"impl": "reference", "metric": metric, "value": v, "unit": metric, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": wl["nwf"] / v * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": cfg, "cpu_baseline": cb,
                "e2e": {"value": v, "unit": metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference has no CPU implementation of the TD step (td codes require GPUs); this arm "
                        "times the step on all host threads with the reference's own CPU derivative library "
                        "(lib/wderiv) and the oracle's restatement of the rest of the step",
                "wall_s": round(time.perf_counter() - t0, 1)}
        print(json.dumps(line))
        return

    if args.probe >= 0:
        print(json.dumps(probe(args)))
        return
    if args.workload == "c5":
        ap.error("--workload c5 needs --probe")

    if world > 1:
        import torch
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    t_start = time.perf_counter()
    wl["drift"] = args.workload == "c2"
    proj, nwf, d, res = run_wtd(args, rank, world)
    nwf_total = args.nwf or wl["nwf"]
    if rank != 0:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
        return
    import torch
    dev = torch.cuda.current_device()
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
        "blocks": args.blocks, "ms_blocks": f["ms_blocks"],
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
                       "ms": e["ms"], "ms_blocks": e["ms_blocks"],
                       "definition": "upload states (pinned) + initial measurement + K steps + download densities + "
                                     "energy, per K steps (median of the blocks)"}
    forms = {}
    n = proj.numel
    if "drift" in f:
        forms["fp64"] = {"energy_drift": f["drift"]}
    for label in ("mixed_h64", "mixed_h32"):
        if label in res and "unsupported" not in res[label]:
            m = res[label]
            forms[label] = {"value": nwf_total * args.steps / (m["ms"] * 1e-3), "ms_blocks": m["ms_blocks"],
                            "speedup_vs_fp64": f["ms"] / m["ms"],
                            "density_rel_l2_err_vs_fp64": rho_err(m["dens"], f["dens"], n),
                            "density_rel_l2_err_vs_fp64_by_block": dens_errs(m["dens"], f["dens"], n),
                            "energy_rel_err_vs_fp64": float(abs(total_energy(m["energy"]) - total_energy(f["energy"])) /
                                                            abs(total_energy(f["energy"]))),
                            "ms_pass_a": m["ms_a"], "ms_pass_b": m["ms_b"]}
            if "drift" in m:
                forms[label]["energy_drift"] = m["drift"]
                forms[label]["density_rel_l2_err_vs_fp64_after_drift_run"] = rho_err(m["drift_dens"], f["drift_dens"], n)
    if forms:
        line["precision_forms"] = forms
    if "adjoint" in res:
        line["adjoint"] = res["adjoint"]
    if not args.no_refcuda and world == 1:
        try:
            rsteps = max(2, args.parity_steps if args.parity_steps > 0 else min(args.steps, 10))
            ref = reference_cuda(proj.name, nwf, rsteps, (proj, d))
            if ref and "value" in ref:
                line["reference_cuda"] = {"value": ref["value"], "ms_per_step": ref["ms_per_step"], "steps": rsteps,
                                          "note": "hpc-engine/*.cu compiled for sm_100a + oracle/ref_harness.cu, same GPU, "
                                                  "same inputs"}
                if args.parity_steps > 0:
                    line["parity_full_size"] = parity_full_size(proj.name, nwf, rsteps, dev, (proj, d), ref)
            else:
                line["reference_cuda"] = ref
        except Exception as ex:  # reported, not fatal
            line["reference_cuda"] = {"error": str(ex)[:200]}
    if args.extras and args.workload == "c2" and world == 1 and not args.nwf:
        for key, fn in (("adjoint", adjoint_c4), ("c3", c3_comparison), ("c5", c5_scale)):
            try:
                line[key] = fn(args, dev)
            except Exception as ex:  # reported, not fatal
                line[key] = {"error": f"{type(ex).__name__}: {str(ex)[:300]}"}
            torch.cuda.empty_cache()
    if not args.no_cpu and world == 1:
        sample = CPU_SAMPLE[args.workload]
        line["cpu_baseline"] = cpu_baseline(proj.name, *sample)
    line["wall_s"] = round(time.perf_counter() - t_start, 1)
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
