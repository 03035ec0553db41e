"""The stage end to end from basis.in / nadvibs.in (the role of Source/main.f90) on the GPU:
the Python driver and the C driver, output.dat's eigenvalue table against the oracle's
restatement of compute_eigenvalues (Source/top.f90:1051-1113) and extract.py's parser, and a
restart run."""
import os
import re
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import driver, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_python_driver_output_tables_and_restart(tmp_path):
    cfg = synth.config(1)
    synth.write_inputs(str(tmp_path), cfg, niter=300, idroots=3)
    res = driver.run(str(tmp_path))
    text = (tmp_path / "output.dat").read_text().splitlines()
    om, cc, pot = synth.draw(cfg)
    # same alpha/beta into the oracle's table: the lines must be identical (drop-in format)
    ref = O.eigen_table_lines(res["alpha"], res["beta"], om, 1.0)
    i0 = next(i for i, l in enumerate(text) if l.startswith("  ZPVE from nadvibs.in"))
    got = [l for l in text[i0:i0 + 4 + len(ref)] if l.strip()]
    assert got[:len(ref)] == ref
    spec = O.extract_spectrum(str(tmp_path / "output.dat"), threshold=1.0)
    rows = [r.split() for r in ref[4:]]
    assert len(spec) == sum(1 for r in rows if float(r[2]) < 1.0 and float(r[5]) != 0.0)
    assert (tmp_path / "restart.log").exists() and (tmp_path / "nadvibs.35.0").exists()
    assert (tmp_path / "rootinfo.dat").read_text().count("************ ROOT") == 3
    # restart: 50 more iterations
    b = (tmp_path / "basis.in").read_text()
    b = re.sub(r"restart = 0", "restart = 1", b)
    b = re.sub(r"niter = 300", "niter = 50", b)
    (tmp_path / "basis.in").write_text(b)
    res2 = driver.run(str(tmp_path))
    assert len(res2["alpha"]) == 350
    np.testing.assert_array_equal(res2["alpha"][:300], res["alpha"])
    assert (tmp_path / "restart.log.old").exists()


def test_c_driver_runs_on_the_gpu(tmp_path):
    cfg = synth.config(1)
    synth.write_inputs(str(tmp_path), cfg)
    exe = tmp_path / "drv"
    subprocess.check_call(["gcc", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "nadvibs_b200", "examples", "nadvibs_driver.c"), "-o", str(exe),
                           "-L", os.path.join(ROOT, "nadvibs_b200"), "-lnadvibs_gpu",
                           f"-Wl,-rpath,{os.path.join(ROOT, 'nadvibs_b200')}"])
    out = subprocess.run([str(exe), str(tmp_path), "20"], capture_output=True, text=True, check=True).stdout
    a1 = float(out.split()[2])
    om, cc, pot = synth.draw(cfg)
    ao, bo, _, _ = O.system_from_arrays(cfg.basis, cfg.nstates, cfg.ordr, om, cc, pot).lanczos(20)
    assert a1 == pytest.approx(ao[0], rel=1e-12)
    assert "COMPUTED EIGENVALUES" in (tmp_path / "output.dat").read_text()
