"""The identity the reverse sweep uses instead of storing H v_j (csrc/grad.cu): the Lanczos
recurrence (Source/top.f90:646-670,820-842) r_j = H v_j - alpha_j v_j - beta_{j-1} v_{j-1},
v_{j+1} = r_j / beta_j gives H v_j = beta_j v_{j+1} + alpha_j v_j + beta_{j-1} v_{j-1}.  Checked
on the oracle's own recurrence (plain Lanczos, FP64) for a quadratic and a cubic system."""
import numpy as np
import pytest

from nadvibs_b200 import synth
from oracle import oracle as O


@pytest.mark.parametrize("seed,nstates,basis,ordr", [(61, 2, [4, 3, 3], 3), (62, 3, [5, 4, 3], 2)])
def test_hv_rebuilt_from_three_lanczos_vectors(seed, nstates, basis, ordr):
    cfg = synth.random_small(seed, nstates, basis, ordr)
    om, cc, pot = synth.draw_small(cfg)
    S = O.system_from_arrays(basis, nstates, ordr, om, cc, pot, quirk_lower=False)
    n = 40
    alpha, beta, V, _ = S.lanczos(n, keep_vectors=True)  # V[j - 1] = v_j, beta[j] = ||r_j||
    for j in range(1, n):
        w = S.hv(V[j - 1])
        rebuilt = beta[j] * V[j] + alpha[j - 1] * V[j - 1]
        if j > 1:
            rebuilt = rebuilt + beta[j - 1] * V[j - 2]
        assert np.abs(w - rebuilt).max() <= 1e-13 * np.abs(w).max(), j
