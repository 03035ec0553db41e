"""The Lanczos stage end to end on the B200 library: the role of ``program main``
(Source/main.f90:25-88) for one GPU.

    python -m nadvibs_b200.driver [-m MB] [-o scratch_dir] [--precision fp64|mixed] [--device N]

reads ``basis.in`` and ``nadvibs.in`` from the working directory, and writes ``output.dat``
(header and eigenvalue table), ``restart.log`` (working directory) with ``nadvibs.35.0``
(scratch directory), ``rootinfo.dat`` when ``idroots``/``soroots`` ask for root
identification, and ``sodata.in`` (spin-orbit parameters) when ``soroots > 0``.  ``restart != 0`` in basis.in resumes from restart.log / nadvibs.35.0 and
runs ``niter`` further iterations, as the reference does (Source/secondary.f90:857-861).
``-m`` is accepted for compatibility (the reference only prints it).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

from . import _lib as L


def _archive_budget(params, niter_total: int, elem_bytes: int, device: int) -> int:
    """Number of Lanczos vectors to keep on the device: all of them when re-orthogonalising
    (required) or when they fit in half of the free device memory (Ritz vectors without a
    replay); 0 otherwise (two-pass Ritz vectors)."""
    dimen = 1
    for i in range(params.nmodes):
        dimen *= params.basis[i]
    per = dimen * params.nstates * elem_bytes
    if params.reorthog > 0:
        return niter_total
    if params.idroots <= 0 and params.soroots <= 0:
        return 0
    try:
        import torch
        free, _ = torch.cuda.mem_get_info(device)
    except Exception:  # no torch: be conservative
        free = 0
    return niter_total if per * niter_total < 0.5 * free else 0


def run(workdir: str = ".", outdir: str | None = None, precision: str = "fp64", device: int = 0,
        basis: str = "basis.in", nadvibs: str = "nadvibs.in", log=print) -> dict:
    t0 = time.time()
    outdir = outdir or workdir
    bpath = os.path.join(workdir, basis)
    npath = os.path.join(workdir, nadvibs)
    out = os.path.join(workdir, "output.dat")
    params = L.read_basis(bpath)
    restart = params.restart != 0
    prec = L.NVB_MIXED if precision == "mixed" else L.NVB_FP64
    iters_before = 0
    if restart:
        with open(os.path.join(workdir, "restart.log")) as f:
            lines = f.read().splitlines()
        iters_before = int(lines[3].split()[0])
    total = iters_before + params.niter
    archive = _archive_budget(params, total, 4 if prec == L.NVB_MIXED else 8, device)
    h = L.Handle.from_files(bpath, npath, precision=prec, device=device, archive_max=archive)
    try:
        h.set_reorthog(params.reorthog, max(params.chkorthog, 1))
        h.write_header(out)
        if restart:
            h.load_restart(workdir, outdir)
            log(f"Restarting Lanczos procedure on step {iters_before + 1}")
        else:
            h.seed()
            h.write_seed_report(out)
        h.set_timing(True)
        a, b = h.lanczos(params.niter)
        hv_ms, it_ms, n = h.timing()
        with open(out, "a") as f:
            f.write("\n   >>>>>>>> Running Lanczos Iterations <<<<<<<<< \n\n")
            f.write(f"   ITERATIONS: {iters_before + 1:5d} - {iters_before + params.niter:5d}\n")
            f.write(f"   - Total matrix-vector product:          {hv_ms / 1e3:14.3f} secs.\n")
            f.write(f"   Time to complete iterations:            {it_ms / 1e3:14.3f} secs.\n")
            f.write("  - Lanczos Iterations Completed - \n")
        h.save_restart(workdir, outdir)
        h.write_eigenvalues(out)
        nroots = max(params.idroots, params.soroots)
        leads = None
        if nroots > 0:
            leads = h.lead_contributors(nroots, params.idroots, os.path.join(workdir, "rootinfo.dat"))
        if params.soroots > 0:
            h.spin_orbit(params.soroots, nroots, os.path.join(workdir, "sodata.in"))
        with open(out, "a") as f:
            f.write(" \nCalculation completed.\n")
        return dict(alpha=a, beta=b, leads=leads, seconds=time.time() - t0)
    finally:
        h.close()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("-m", type=float, default=30.0, help="memory in MB (accepted, not used)")
    ap.add_argument("-o", default=None, help="scratch directory for nadvibs.35.0")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--workdir", default=".")
    a = ap.parse_args(argv)
    res = run(a.workdir, a.o, a.precision, a.device)
    print(f"NadVibS Lanczos stage finished in {res['seconds']:.2f} s")
    return 0


if __name__ == "__main__":
    sys.exit(main())
