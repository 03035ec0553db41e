"""Regenerate the golden fixtures of tests/golden/ from the reference checkout.

The reference's only known-answer data are the Gaussian-broadening fixtures of its
``convolve/`` directory: line spectra ``spec.line`` / ``spec.line.adia`` and the broadened
spectra ``output`` / ``output.adia`` produced from them by ``convolve/main.f90`` (FWHM 5e-3 eV,
grid -0.1..0.4 eV with 2002 points, shift 2.7807 eV).  This script copies those numbers
into JSON so the tests can run without the reference checkout.

Usage: python tests/golden/make_golden.py <path of the reference checkout>
"""
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
ref = sys.argv[1]
here = os.path.dirname(os.path.abspath(__file__))


def cols(path):
    out = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if len(t) >= 2:
                out.append([float(t[0]), float(t[1])])
    return out


fixtures = {}
for name, spec, outp in [("dia", "spec.line", "output"), ("adia", "spec.line.adia", "output.adia")]:
    fixtures[name] = {
        "source": f"convolve/{spec} -> convolve/{outp}",
        "lines": cols(os.path.join(ref, "convolve", spec)),
        "spectrum": cols(os.path.join(ref, "convolve", outp)),
    }
with open(os.path.join(here, "convolve_fwhm.json"), "w") as f:
    json.dump(fixtures, f)
print("wrote", os.path.join(here, "convolve_fwhm.json"))
