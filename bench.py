#!/usr/bin/env python
"""Benchmark of the B200 Lanczos stage: Lanczos iterations/s on the drop-in size system.

Workload (one step = one Lanczos iteration = H.v + alpha reduction + residual update +
beta reduction): the 3-state, 8-mode vibronic Hamiltonian with basis [20,16,12,10,8,8,6,6]
(88,473,600 functions per state, 265,420,800 in total), quadratic expansion, seeded
synthetic coefficients (numpy default_rng(1002); the reference ships no input for it).
The headline value is the plain FP64 path; the same line carries the mixed-precision
(FP32 vectors, FP64 recurrence) rate, their ratio, and H.v bandwidth for both.

Every vector (2.1 GB FP64) is larger than the 126 MB L2, so no cache flush is needed
between steps.  Multi-GPU runs are replicas (the stage does not shard): each rank runs its
own copy; value = total iterations/s over all ranks, timed as the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --hv-only --precision mixed --steps 1 --warmup 1   (one H.v, for profiling)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Lanczos iter/s & H.v HBM GB/s: mixed vs FP64 at <=0.1 cm^-1; grad/fwd time"
CONFIG_NUMBER = 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="both")
    ap.add_argument("--hv-only", action="store_true", help="run H.v launches only (profiling)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run the adjoint contraction d<u|H|v>/dtheta only (FP64 vectors; profiling)")
    ap.add_argument("--grad-only", action="store_true",
                    help="run the gradient leg only and print its JSON (profiling)")
    ap.add_argument("--config", type=int, default=CONFIG_NUMBER)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradient (grad/fwd) measurement")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the mixed-vs-FP64 Ritz comparison")
    ap.add_argument("--no-fma", action="store_true", help="skip the measured FMA and tile-stream ceilings")
    ap.add_argument("--no-config5", action="store_true",
                    help="skip the short literal-size run of the cubic system (config 5)")
    ap.add_argument("--no-reorth", action="store_true",
                    help="skip the re-orthogonalised mixed run with the host-memory archive")
    ap.add_argument("--reorth-iters", type=int, default=150,
                    help="iterations of the re-orthogonalised run (capped by host memory)")
    ap.add_argument("--config5", action="store_true",
                    help="also run the large cubic system (config 5): literal-size mixed forward and the "
                         "budgeted gradient (minutes; not part of the default run)")
    ap.add_argument("--basis", type=str, default=None,
                    help="comma-separated basis overriding the config's (same coefficients; profiling of "
                         "reduced sizes)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.th = None

    def _run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.th:
            self.th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_for(kernel: str, precision: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "hv_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(f"{kernel}:{precision}")


def make_inputs(cfgn: int, tmpdir: str, basis: str | None = None):
    from nadvibs_b200 import synth
    cfg = synth.config(cfgn)
    if basis:
        b = [int(v) for v in basis.split(",")]
        if len(b) != cfg.nmodes:
            raise SystemExit(f"--basis needs {cfg.nmodes} values")
        cfg.basis = b
    return cfg, synth.write_inputs(tmpdir, cfg)


def run_ours(args, rank, world, dev):
    import torch
    from nadvibs_b200 import _lib as L

    torch.cuda.set_device(dev)
    tmp = tempfile.mkdtemp(prefix=f"nvb_bench_{rank}_")
    cfg, (basis, nadvibs) = make_inputs(args.config, tmp, args.basis)
    N = cfg.dimen * cfg.nstates
    from nadvibs_b200 import replicas
    results = {}
    precs = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    barrier = replicas.barrier
    maxall = replicas.max_over_ranks

    for prec in precs:
        pflag = L.NVB_FP64 if prec == "fp64" else L.NVB_MIXED
        eb = 8 if prec == "fp64" else 4
        h = L.Handle.from_files(basis, nadvibs, device=dev, precision=pflag)
        kname = h.hv_kernel(L.DTYPE_F64 if prec == "fp64" else L.DTYPE_F32)
        st = torch.cuda.Stream(device=dev)
        h.set_stream(st.cuda_stream)
        if args.hv_only:
            dt = torch.float64 if prec == "fp64" else torch.float32
            x = torch.randn(N, device=f"cuda:{dev}", dtype=dt)
            y = torch.empty_like(x)
            torch.cuda.synchronize()
            with torch.cuda.stream(st):
                for _ in range(args.warmup + args.steps):
                    h.hv_ptr(x.data_ptr(), y.data_ptr(), L.DTYPE_F64 if prec == "fp64" else L.DTYPE_F32)
            torch.cuda.synchronize()
            h.close()
            del x, y
            torch.cuda.empty_cache()
            continue
        h.seed()
        if args.warmup:
            h.lanczos(args.warmup)
        torch.cuda.synchronize()
        barrier()
        h.set_timing(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clk:
            e0.record(st)
            a, b = h.lanczos(args.steps)
            e1.record(st)
            torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        ms_max = maxall(ms)
        hv_ms, it_ms, n = h.timing()
        results[prec] = dict(ms=ms_max, hv_ms_per=hv_ms / max(n, 1), it_ms_per=it_ms / max(n, 1),
                             clocks=clk.summary(), bytes_hv=2 * N * eb, alpha=a[-3:].tolist(),
                             beta=b[-3:].tolist(), launches=4 * args.steps, kernel=kname,
                             stream=h.hv_tile_stream(L.DTYPE_F64 if prec == "fp64" else L.DTYPE_F32))
        h.close()
        torch.cuda.empty_cache()
    # end-to-end through the public API with host buffers: create from files (host input),
    # seed, K iterations with alpha/beta returned to host memory, per iteration
    e2e = None
    if not args.hv_only:
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        h = L.Handle.from_files(basis, nadvibs, device=dev, precision=L.NVB_FP64)
        h.seed()
        a, b = h.lanczos(args.steps)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        h.close()
        wall = maxall(t1 - t0)
        h2d = os.path.getsize(basis) + os.path.getsize(nadvibs)
        e2e = {"value": world * args.steps / wall, "unit": "iter/s",
               "h2d_bytes_per_step": int(round(h2d / args.steps)), "d2h_bytes_per_step": 16}
    return cfg, N, results, e2e


def mixed_accuracy(basis: str, nadvibs: str, dev: int, iters: int = 2000, nroots: int = 50):
    """Mixed precision against FP64 on the benchmark system: both precisions run `iters` plain
    Lanczos iterations from the same seed.  The FP64 Ritz values converged to 1e-8 (bji,
    hartree) are grouped into distinct roots (ghost copies within 0.5 cm^-1 of each other are
    one root).  A root counts as converged in both runs when the nearest mixed Ritz value has
    bji < 1e-6; for the lowest `nroots` such roots the report gives the energy difference
    (cm^-1) and, for lines of intensity >= 1e-3, the relative difference of the intensities,
    each summed over the Ritz values within 0.5 cm^-1 (ghost copies split a line).  Roots that
    converged in the FP64 run only (the FP32 run converges fewer distinct roots in the same
    number of iterations) are counted, with the distance to their nearest mixed Ritz value."""
    import numpy as np
    from nadvibs_b200 import _lib as L
    au2cm = 219474.6313705
    out, secs = {}, {}
    for prec in (L.NVB_FP64, L.NVB_MIXED):
        h = L.Handle.from_files(basis, nadvibs, device=dev, precision=prec)
        t0 = time.perf_counter()
        h.seed()
        h.lanczos(iters)
        out[prec] = h.ritz(iters)
        secs[prec] = time.perf_counter() - t0
        h.close()
    E, bji, inten = out[L.NVB_FP64][:3]
    Em, bjim, intm = out[L.NVB_MIXED][:3]
    roots = []
    for e in np.sort(E[bji < 1e-8]):
        if not roots or (e - roots[-1]) * au2cm > 0.5:
            roots.append(e)
    both, only64 = [], []
    for e in roots:
        k = int(np.argmin(np.abs(Em - e)))
        (both if bjim[k] < 1e-6 else only64).append((e, abs(Em[k] - e) * au2cm))
    sel = both[:nroots]
    dE = [d for _, d in sel]
    dI = []
    for e, _ in sel:
        i64 = inten[np.abs(E - e) * au2cm < 0.5].sum()
        i32 = intm[np.abs(Em - e) * au2cm < 0.5].sum()
        if i64 >= 1e-3:
            dI.append(abs(i32 - i64) / i64)
    e0 = roots[0] if roots else 0.0
    return {"iterations": iters, "fp64_converged_roots": len(roots), "converged_in_both": len(both),
            "roots_compared": len(sel), "lines_compared": len(dI),
            "compared_span_cm": float((sel[-1][0] - sel[0][0]) * au2cm) if sel else None,
            "max_abs_dE_cm": float(max(dE)) if dE else None,
            "max_rel_dI": float(max(dI)) if dI else None,
            "target_dE_cm": 0.1, "target_rel_dI": 1e-4,
            "fp64_only_roots": len(only64),
            "fp64_only_lowest_above_e0_cm": float((only64[0][0] - e0) * au2cm) if only64 else None,
            "fp64_only_max_dist_cm": float(max(d for _, d in only64)) if only64 else None,
            "wall_s": {"fp64": secs[L.NVB_FP64], "mixed": secs[L.NVB_MIXED]}}


def host_available_bytes() -> int:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def reorth_leg(basis: str, nadvibs: str, dev: int, iters: int = 150, host_frac: float = 0.6):
    """The re-orthogonalised mixed-precision run (the config-2 Hamiltonian with FP32 vectors,
    reorthog=1: the omega recurrence with exact checks every chkorthog=100 iterations, partial
    re-orthogonalisation), its Lanczos-vector archive in pinned host memory streamed back to the
    GPU in chunks.  One vector is 1.06 GB, so the run is as long as `host_frac` of the host's
    available memory allows (at most `iters`); the reference keeps the same archive on disk.
    Reports iter/s (including pinning the archive), the re-orthogonalisation events, and the
    converged roots with the smallest gap between two of them (no ghost copies)."""
    import numpy as np
    from nadvibs_b200 import _lib as L
    au2cm = 219474.6313705
    h = L.Handle.from_files(basis, nadvibs, device=dev, precision=L.NVB_MIXED)
    try:
        sz = h.sizes()
        per = int(sz["dimen"]) * int(sz["nstates"]) * 4
        fit = int(host_frac * host_available_bytes() // per)
        n = max(0, min(iters, fit))
        if n < 10:
            return {"skipped": f"host memory for {n} archived vectors only"}
        h.set_archive(1, n)
        h.set_reorthog(1, 100)
        t0 = time.perf_counter()
        h.seed()
        h.lanczos(n)
        dt = time.perf_counter() - t0
        log = h.reorth_log()
        E, bji, inten = h.ritz(n)[:3]
    finally:
        h.close()
    conv = np.sort(E[bji < 1e-8])
    return {"iterations": n, "archive": "pinned host memory", "archive_gb": n * per / 1e9,
            "host_available_gb": host_available_bytes() / 1e9, "host_fraction_used": host_frac,
            "wall_s": dt, "iter_per_s": n / dt,
            "reorth_events": int(len(set(int(r[0]) for r in log))),
            "vectors_reorthogonalised": int(sum(int(r[2]) - int(r[1]) + 1 for r in log)),
            "converged_roots": int(conv.size),
            "min_gap_converged_cm": float(np.diff(conv).min() * au2cm) if conv.size > 1 else None}


def grad_timing(dev: int):
    """grad/fwd on the gradient system (config 4): forward = seed + 400 plain Lanczos
    iterations, recording every Lanczos vector and H v for the reverse sweep (checkpoint
    interval -1, which fits here); backward = eigen-derivatives of T_400 for a loss
    (Gaussian-convolved spectrum of the converged Ritz values, sigma 20 cm^-1, 2048 points, plus
    the lowest 20 Ritz energies; loss and eigen-derivative products on the GPU, the tridiagonal
    eigensolve on the host) and the reverse sweep (nvb_lanczos_backward from the record).  Host
    wall times around synchronised calls, best of 3."""
    import numpy as np
    import torch
    from nadvibs_b200 import _lib as L
    from nadvibs_b200 import synth
    from nadvibs_b200.autograd import AU2WAVE, converged_spectrum, tridiag_eig_backward, tridiag_eigh
    cfg = synth.config(4)
    om, cc, pot = synth.draw(cfg)
    potf = synth.flatten_pot(pot)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr, p.niter = cfg.nstates, cfg.nmodes, cfg.ordr, cfg.niter
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    n, k = 400, -1  # the forward records every vector when it fits (as autograd.ritz does)
    cuda = torch.device("cuda", dev)
    # the loss and the eigen-derivatives of T_n run on the same GPU (FP64)
    grid = torch.linspace(-200.0, 8000.0, 2048, dtype=torch.float64, device=cuda)
    w = torch.from_numpy(np.random.default_rng(4).normal(size=2048)).to(cuda)
    fwd, bwd, sweep, host = [], [], [], []
    plan = None
    for _ in range(3):
        h = L.Handle.from_arrays(p, om, cc, potf, device=dev)
        h.set_checkpoints(k)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h.seed()
        a, b = h.lanczos(n)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        E, S = tridiag_eigh(a[:n], b[1:n])
        conv = torch.from_numpy(np.abs(b[n] * S[-1]) < 1e-9).to(cuda)
        Et = torch.from_numpy(E).to(cuda).requires_grad_(True)
        It = torch.from_numpy(S[0] ** 2).to(cuda).requires_grad_(True)
        ((w * converged_spectrum(Et, It, conv, grid, 20.0)).sum() + (Et[:20] * AU2WAVE).sum()).backward()
        abar, boff = tridiag_eig_backward(E, S, Et.grad.cpu().numpy(), It.grad.cpu().numpy(), device=cuda)
        bbar = np.zeros(n)
        bbar[: n - 1] = boff
        th = time.perf_counter()
        h.lanczos_backward(n, abar, bbar, k)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        plan = h.backward_plan()
        h.close()
        fwd.append(t1 - t0)
        bwd.append(t2 - t1)
        sweep.append(t2 - th)
        host.append(th - t1)
    f, g = min(fwd), min(bwd)
    return {"workload": "config4: 2 states, basis [14,12,10,8,8,6], 1,290,240 functions, ordr 2, 400 plain "
                        "Lanczos iterations, forward recorded for the sweep (checkpoint interval -1), FP64",
            "backward_plan": plan,
            "loss": "Gaussian-convolved spectrum of the converged Ritz values (bji < 1e-9; sigma 20 cm^-1, "
                    "2048 points) + lowest 20 Ritz energies",
            "ncoef": int(len(potf) + len(cc) + len(om)), "fwd_ms": 1e3 * f, "grad_ms": 1e3 * g,
            "reverse_sweep_ms": 1e3 * min(sweep), "host_eig_and_loss_ms": 1e3 * min(host),
            "grad_over_fwd": g / f}


def adjoint_timing(args, dev: int) -> dict:
    """warmup + steps calls of the adjoint contraction (nvb_hv_adjoint_coeffs) of the chosen
    system with random FP64 u, v; host wall time per call around synchronised calls."""
    import numpy as np
    import torch
    from nadvibs_b200 import _lib as L
    from nadvibs_b200 import synth
    torch.cuda.set_device(dev)
    cfg = synth.config(args.config)
    if args.basis:
        cfg.basis = [int(b) for b in args.basis.split(",")]
    om, cc, pot = synth.draw(cfg)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr, p.niter = cfg.nstates, cfg.nmodes, cfg.ordr, 10
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    n = int(np.prod(cfg.basis)) * cfg.nstates
    h = L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot), device=dev, precision=L.NVB_MIXED, quirk_lower=0)
    try:
        g = torch.Generator(device=f"cuda:{dev}").manual_seed(1)
        u = torch.randn(n, generator=g, device=f"cuda:{dev}", dtype=torch.float64)
        v = torch.randn(n, generator=g, device=f"cuda:{dev}", dtype=torch.float64)
        for _ in range(args.warmup):
            h.adjoint_ptr(u.data_ptr(), v.data_ptr(), L.DTYPE_F64)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            h.adjoint_ptr(u.data_ptr(), v.data_ptr(), L.DTYPE_F64)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / max(args.steps, 1)
    finally:
        h.close()
    return {"basis": list(cfg.basis), "elements": n, "ms_per_call": ms}


def tile_stream(stream: dict | None, hv_ms: float, seconds: float = 1.0):
    """The factorised H.v's neighbour-tile stream (bytes copied L2 -> shared memory per product)
    against its measured ceiling: whole tiles of the same size streamed into a ring of the same
    slots and CTAs per multiprocessor with no arithmetic (nvb_measure_tile_stream)."""
    from nadvibs_b200 import _lib as L
    if not stream or stream["bytes_per_hv"] <= 0:
        return None
    ceiling = L.measure_tile_stream(stream["tile_bytes"], stream["slots"], stream["ctas_per_sm"], seconds)
    achieved = stream["bytes_per_hv"] / (hv_ms / 1e3)
    return {"bytes_per_hv": stream["bytes_per_hv"], "tile_bytes": stream["tile_bytes"], "slots": stream["slots"],
            "ctas_per_sm": stream["ctas_per_sm"], "achieved_gbs": achieved / 1e9, "ceiling_gbs": ceiling / 1e9,
            "frac": achieved / ceiling, "ceiling_kind": "measured (nvb_measure_tile_stream)"}


def large_cubic(dev: int, iters: int = 4, warm: int = 2, grad_iters: int = 60, budget: float = 150e9,
                with_grad: bool = True):
    """Config 5, ordr 3 (cubic terms N(0,10 cm^-1)), 3 states, 10 modes, FP32 vectors / FP64
    recurrence.  (1) The literal basis [16,14,12,10,8,8,6,6,4,4]: 990,904,320 functions per
    state, 2,972,712,960 elements, 11.9 GB per FP32 vector; `warm` + `iters` mixed iterations,
    iter/s and the H.v kernel in use.  (2) The gradient at the size the benchmark description
    states (~124M per state, 372M total): basis [8,7,6,10,8,8,6,6,4,4] with the same coefficient
    draws; `grad_iters` mixed iterations, loss = Gaussian-convolved spectrum (sigma 20 cm^-1,
    2048 points) + lowest 20 Ritz energies, reverse sweep with the automatic checkpoint plan
    under a `budget`-byte device-memory budget.  Host wall times around synchronised calls."""
    import numpy as np
    import torch
    from nadvibs_b200 import _lib as L
    from nadvibs_b200 import synth
    from nadvibs_b200.autograd import AU2WAVE, convolved_spectrum, tridiag_eig_backward, tridiag_eigh
    cfg = synth.config(5)
    om, cc, pot = synth.draw(cfg)
    potf = synth.flatten_pot(pot)

    def params(basis, niter):
        p = L.default_params()
        p.nstates, p.nmodes, p.ordr, p.niter = cfg.nstates, cfg.nmodes, cfg.ordr, niter
        for i, b in enumerate(basis):
            p.basis[i] = b
        return p

    out = {}
    h = L.Handle.from_arrays(params(cfg.basis, warm + iters), om, cc, potf, device=dev, precision=L.NVB_MIXED)
    try:
        free, total = torch.cuda.mem_get_info(dev)
        h.seed()
        h.lanczos(warm)
        torch.cuda.synchronize()
        h.set_timing(True)
        t0 = time.perf_counter()
        h.lanczos(iters)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        hv_ms, _, nt = h.timing()
        hv_ms /= max(nt, 1)
        n_el = int(np.prod(cfg.basis)) * cfg.nstates
        out["literal"] = {"basis": list(cfg.basis), "elements": n_el,
                          "kernel": h.hv_kernel(L.DTYPE_F32), "iter_per_s": iters / dt, "ms_per_iter": 1e3 * dt / iters,
                          "hv_ms": hv_ms, "hv_gbs": 2 * n_el * 4 / (hv_ms / 1e3) / 1e9,
                          "tile_stream": tile_stream(h.hv_tile_stream(L.DTYPE_F32), hv_ms),
                          "device_gb_in_use_after_create": (total - free) / 1e9, "iterations_timed": iters}
    finally:
        h.close()
    if not with_grad:
        return out
    basis = [8, 7, 6, 10, 8, 8, 6, 6, 4, 4]
    n = grad_iters
    h = L.Handle.from_arrays(params(basis, n), om, cc, potf, device=dev, precision=L.NVB_MIXED)
    try:
        # the forward records its vectors for the sweep when they fit the budget (n + 2 FP32
        # vectors beside the sweep's work vectors); otherwise the sweep takes the automatic plan
        h.set_backward_memory(int(budget))
        h.set_checkpoints(-1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h.seed()
        a, b = h.lanczos(n)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        E, S = tridiag_eigh(a[:n], b[1:n])
        grid = torch.linspace(-200.0, 8000.0, 2048, dtype=torch.float64)
        w = torch.from_numpy(np.random.default_rng(5).normal(size=2048))
        Et = torch.from_numpy(E).requires_grad_(True)
        It = torch.from_numpy(S[0] ** 2).requires_grad_(True)
        ((w * convolved_spectrum(Et, It, grid, 20.0)).sum() + (Et[:20] * AU2WAVE).sum()).backward()
        abar, boff = tridiag_eig_backward(E, S, Et.grad.numpy(), It.grad.numpy())
        bbar = np.zeros(n)
        bbar[: n - 1] = boff
        g = h.lanczos_backward(n, abar, bbar, -1)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        out["gradient"] = {"basis": basis, "elements": int(np.prod(basis)) * cfg.nstates, "iterations": n,
                           "budget_gb": budget / 1e9, "backward_plan": h.backward_plan(), "ncoef": int(g.size),
                           "finite": bool(np.isfinite(g).all()), "fwd_s": t1 - t0, "grad_s": t2 - t1,
                           "grad_over_fwd": (t2 - t1) / (t1 - t0)}
    finally:
        h.close()
    return out


def workload_name(cfgn: int, basis=None) -> str:
    """The benchmark system's description as both arms' JSON lines name it."""
    import math
    from nadvibs_b200 import synth
    cfg = synth.config(cfgn)
    basis = list(basis) if basis else list(cfg.basis)
    n = math.prod(basis) * cfg.nstates
    return (f"config{cfgn}: {cfg.nstates} states, {cfg.nmodes} modes, basis [{','.join(str(b) for b in basis)}], "
            f"{n:,} functions, ordr {cfg.ordr}, plain Lanczos (reorthog=0)")


def hv_flops(cfg) -> float:
    """Reference-equivalent arithmetic of one H.v, from the term table (the reference's pass
    structure, Source/top.f90:717-806): 2 flops per row for every nonzero (monomial, nonzero
    shift, ordered state pair) and for every diagonal-section term (one fused harmonic energy +
    constant per state, plus the zero shift of each all-even monomial).  Rows where a shift
    leaves the basis are counted too, so this is an upper bound of the reference's work."""
    import math
    from nadvibs_b200 import synth
    _, _, pot = synth.draw(cfg)
    S, M = cfg.nstates, cfg.nmodes
    dimen = math.prod(cfg.basis)
    shift_terms, diag_terms = 0, S
    k = 0
    for i in range(1, S + 1):
        for j in range(1, i + 1):
            mult = 1 if i == j else 2
            for d in range(1, cfg.ordr + 1):
                for t, mono in enumerate(synth.monomials(M, d)):
                    if pot[k][d - 1][t] == 0.0:
                        continue
                    pows = [mono.count(q) for q in set(mono)]
                    even = all(p % 2 == 0 for p in pows)
                    shift_terms += mult * (math.prod(p + 1 for p in pows) - (1 if even else 0))
                    diag_terms += mult if even else 0
            k += 1
    return 2.0 * dimen * (shift_terms + diag_terms)


def cpu_baseline_sample(cfgn: int, iters: int):
    """The oracle's restatement of the reference (one streaming pass per term and shift,
    Source/top.f90:672-818, and lanczos_step) on all host cores, bounded sample."""
    from nadvibs_b200 import synth
    from oracle import oracle as O
    O.build()
    cfg = synth.config(cfgn)
    om, cc, pot = synth.draw(cfg)
    S = O.system_from_arrays(cfg.basis, cfg.nstates, cfg.ordr, om, cc, pot)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    S.lanczos(iters, nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": iters / dt, "unit": "iter/s", "cores": cores, "kind": "port",
            "sample": f"{iters} Lanczos iteration(s) of the {cfg.dimen * cfg.nstates:,}-element system "
                      f"(seed + recurrence) by the C oracle, OpenMP on {cores} threads, {dt:.1f} s"}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        # one iteration of the benchmark system takes seconds of CPU time per core count, so
        # the CPU arm times a bounded sample of at most 3 iterations, whatever --steps asks
        iters = max(1, min(args.steps, 3))
        cb = cpu_baseline_sample(args.config, iters)
        cb["iterations_timed"] = iters
        cb["why_fewer_than_steps"] = (None if iters == args.steps else
                                      f"bounded CPU sample: {iters} of the {args.steps} requested iterations, so "
                                      f"that the arm ends within a few minutes (rate in iter/s is per iteration)")
        line = {"metric": METRIC, "value": cb["value"], "unit": "iter/s", "impl": "reference", "n_gpus": args.gpus,
                "steps": iters, "warmup": 0, "ms_per_step": 1e3 / cb["value"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": workload_name(args.config), "precision": "fp64",
                           "cache": "inputs larger than L2" if args.config in (2, 3, 5) else "inputs in L2"},
                "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "iter/s", "h2d_bytes_per_step": 0,
                                            "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    if args.adjoint_only:
        if rank == 0:
            print(json.dumps({"adjoint_only": adjoint_timing(args, local)}))
        return 0
    if args.grad_only:
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            print(json.dumps({"grad": grad_timing(local)}))
        return 0
    if world > 1:
        from nadvibs_b200 import replicas
        replicas.init("nccl", timeout_s=120)
    cfg, N, res, e2e = run_ours(args, rank, world, local)
    if args.hv_only:
        if rank == 0:
            print(json.dumps({"hv_only": True, "launches": args.warmup + args.steps}))
        return 0
    peak, peak_kind = peaks()
    main_prec = "fp64" if "fp64" in res else "mixed"
    r = res[main_prec]
    value = world * args.steps / (r["ms"] / 1e3)
    hv_gbs = r["bytes_hv"] / (r["hv_ms_per"] / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if main_prec == "fp64" else "f32+f64",
        "data": f"synthetic (seeded basis.in/nadvibs.in, numpy default_rng({cfg.seed}))",
        "config": {"workload": workload_name(args.config, cfg.basis), "precision": main_prec,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "cache": "inputs larger than L2 (2.1 GB FP64 vectors), no flush"},
        "roofline": {"bound": "hbm", "achieved": hv_gbs, "peak": peak, "unit": "GB/s", "frac": hv_gbs / peak,
                     "traffic": traffic_for("hv_" + r["kernel"], main_prec), "kernel": f"H.v (k_hv_{r['kernel']})",
                     "algorithmic_bytes": r["bytes_hv"], "peak_kind": peak_kind},
        "clocks": r["clocks"], "gpu_launches": r["launches"], "e2e": e2e,
    }
    if "mixed" in res and "fp64" in res:
        m = res["mixed"]
        mixed_rate = world * args.steps / (m["ms"] / 1e3)
        line["mixed"] = {"value": mixed_rate, "unit": "iter/s", "ratio_vs_fp64": mixed_rate / value,
                         "hv_ms": m["hv_ms_per"], "hv_gbs": m["bytes_hv"] / (m["hv_ms_per"] / 1e3) / 1e9,
                         "hv_frac": m["bytes_hv"] / (m["hv_ms_per"] / 1e3) / 1e9 / peak,
                         "hv_traffic": traffic_for("hv_" + m["kernel"], "mixed"), "kernel": f"k_hv_{m['kernel']}"}
        line["fp64_hv_ms"] = r["hv_ms_per"]
    if rank == 0:
        # the arithmetic side of the roofline, reference-equivalent flops (the factorised
        # kernels execute fewer; see hv_flops)
        fl = hv_flops(cfg)
        line["alu"] = {"algorithmic_gflop_per_hv": fl / 1e9,
                       "achieved_tflops": fl / (r["hv_ms_per"] / 1e3) / 1e12, "precision": main_prec}
        if "mixed" in res and main_prec != "mixed":
            line["alu"]["mixed_achieved_tflops"] = fl / (res["mixed"]["hv_ms_per"] / 1e3) / 1e12
        if not args.no_fma:
            # measured FMA ceilings of this GPU (seconds-long register-only FMA loops), against
            # which the reference-equivalent flop rates above are compared
            import torch
            from nadvibs_b200 import _lib as L
            torch.cuda.set_device(local)
            f64 = L.measure_fma(L.DTYPE_F64, 2.0)
            f32 = L.measure_fma(L.DTYPE_F32, 2.0)
            line["alu"]["measured_fp64_tflops"] = f64 / 1e12
            line["alu"]["measured_fp32_tflops"] = f32 / 1e12
            line["alu"]["frac_of_measured_fp64"] = line["alu"]["achieved_tflops"] / (f64 / 1e12)
            if "mixed_achieved_tflops" in line["alu"]:
                line["alu"]["mixed_frac_of_measured_fp32"] = line["alu"]["mixed_achieved_tflops"] / (f32 / 1e12)
            # the factorised kernel's own bound: its neighbour-tile stream against the measured
            # ceiling of that stream
            line["roofline"]["tile_stream"] = tile_stream(r.get("stream"), r["hv_ms_per"])
            if "mixed" in line:
                line["mixed"]["tile_stream"] = tile_stream(res["mixed"].get("stream"), res["mixed"]["hv_ms_per"])
    if rank == 0 and not args.no_grad:
        line["grad"] = grad_timing(local)
    if rank == 0 and args.config5:
        line["config5"] = large_cubic(local)
    elif rank == 0 and not args.no_config5:
        # the cubic system at its literal size: a few mixed iterations (the gradient at the
        # stated size runs with --config5)
        try:
            line["config5"] = large_cubic(local, iters=2, warm=1, with_grad=False)
        except Exception as e:
            line["config5"] = {"error": str(e)}
    if rank == 0 and "mixed" in res and not args.no_accuracy:
        tmp = tempfile.mkdtemp(prefix="nvb_acc_")
        _, (b_in, n_in) = make_inputs(args.config, tmp, args.basis)
        line["accuracy"] = mixed_accuracy(b_in, n_in, local)
    if rank == 0 and "mixed" in res and not args.no_reorth:
        tmp = tempfile.mkdtemp(prefix="nvb_reorth_")
        _, (b_in, n_in) = make_inputs(args.config, tmp, args.basis)
        try:
            line["reorth"] = reorth_leg(b_in, n_in, local, args.reorth_iters)
        except Exception as e:  # reported, not fatal: the leg needs ~100 GB of pinned host memory
            line["reorth"] = {"error": str(e)}
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(args.config, 1)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        from nadvibs_b200 import replicas
        replicas.shutdown()
    return 0


if __name__ == "__main__":
    sys.exit(main())
