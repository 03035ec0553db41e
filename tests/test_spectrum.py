"""Spectrum post-step: the extract.py filter (host, no GPU) and the GPU broadening
(nvb_convolve) against the reference's own broadened fixtures (convolve/spec.line -> output,
printed with f15.8) and the oracle's restatement of convolve.py."""
import json
import os

import numpy as np
import pytest

from nadvibs_b200 import spectrum
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _fixtures():
    with open(os.path.join(HERE, "golden", "convolve_fwhm.json")) as f:
        return json.load(f)


def test_extract_filter_matches_oracle(tmp_path):
    rng = np.random.default_rng(3)
    n = 40
    conv = 10.0 ** rng.uniform(-20, -1, size=n)
    conv[::7] = 0.0
    inten = np.round(rng.uniform(0, 1, size=n), 7)
    inten[::5] = 0.0
    ecm = np.sort(rng.uniform(0, 8000, size=n))
    lines = ["  header line", " ", "  Root  Index  Convergence     E(cm-1)        E(eV)     Intensity"]
    for k in range(n):
        lines.append(O._I(k + 1, 6) + O._I(k + 1, 7) + O._ES(conv[k], 13, 4) + O._F(ecm[k], 15, 5)
                     + O._F(ecm[k] / 8065.54, 12, 5) + O._F(inten[k], 12, 7))
    lines += [" ", "   All requested eigenvalues computed."]
    path = tmp_path / "output.dat"
    path.write_text("\n".join(lines) + "\n")
    for thr in [1e-15, 1e-6, 1.0]:
        x, y, c = spectrum.extract(str(path), threshold=thr)
        ref = O.extract_spectrum(str(path), threshold=thr)
        assert len(x) == len(ref)
        if len(ref):
            ref = np.array(ref)
            np.testing.assert_allclose(x, ref[:, 0])
            np.testing.assert_allclose(y, ref[:, 1])


def test_extract_reads_three_digit_exponents(tmp_path):
    rows = ["  Root  Index  Convergence     E(cm-1)        E(eV)     Intensity",
            "     1      1   1.0227-321        0.00000     0.00000   1.0000000",
            "     2      2   2.5000E-03      619.95484     0.07686   0.0011396",
            " ", "   All requested eigenvalues computed."]
    path = tmp_path / "output.dat"
    path.write_text("\n".join(rows) + "\n")
    x, y, c = spectrum.extract(str(path), threshold=1e-2)
    np.testing.assert_allclose(c, [1.0227e-321, 2.5e-3])
    np.testing.assert_allclose(y, [1.0, 0.0011396])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["dia", "adia"])
def test_gpu_fwhm_broadening_reproduces_the_reference_fixture(name):
    fx = _fixtures()[name]
    lines = np.array(fx["lines"])
    want = np.array(fx["spectrum"])
    x, y = spectrum.convolve_fwhm(lines[:, 0], lines[:, 1])
    assert len(x) == len(want)
    np.testing.assert_allclose(x, want[:, 0], atol=5e-9)
    np.testing.assert_allclose(y, want[:, 1], atol=5e-9)
    xo, yo = O.convolve_fwhm(lines[:, 0], lines[:, 1])
    np.testing.assert_allclose(y, yo, rtol=1e-13, atol=1e-15)


@pytest.mark.gpu
@pytest.mark.parametrize("aperture", ["Gaussian", "Lorentzian"])
def test_gpu_sigma_broadening_matches_convolve_py(aperture):
    rng = np.random.default_rng(5)
    c = rng.uniform(0.0, 1.0, size=300)
    h = rng.uniform(0.0, 1.0, size=300)
    grid = np.linspace(-0.2, 1.2, 1000)
    env = spectrum.convolve(c, h, grid, 0.01, aperture)
    ref = O.convolve_sigma(c, h, 0.01, grid, aperture)
    np.testing.assert_allclose(env, ref, rtol=1e-12, atol=1e-14)
