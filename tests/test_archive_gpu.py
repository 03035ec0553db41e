"""The Lanczos-vector archive in device memory, pinned host memory and a file in the
reference's nadvibs.34 layout (Source/secondary.f90:273-308), driving partial
re-orthogonalisation (Source/top.f90:844-1005): the three give the same recurrence, the
Gram-Schmidt intervals of the exact-overlap mode match the oracle's step by step, the file
holds the vectors in the reference's FP64 layout, and re-orthogonalisation resumes after a
restart from the file archive (Source/top.f90:572-575,582-587)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth
from oracle import oracle as O
from oracle import reorth

pytestmark = pytest.mark.gpu


def _handle(n=1, precision=L.NVB_FP64):
    cfg = synth.config(n)
    om, cc, pot = synth.draw(cfg)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr, p.niter = cfg.nstates, cfg.nmodes, cfg.ordr, cfg.niter
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    S = O.system_from_arrays(cfg.basis, cfg.nstates, cfg.ordr, om, cc, pot)
    return L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot), precision=precision), S


def _run(kind, niter, reorthog, tmp_path, precision=L.NVB_FP64, chk=50):
    h, _ = _handle(precision=precision)
    with h:
        h.set_archive(kind, niter, str(tmp_path / f"nadvibs.34.k{kind}") if kind == 2 else None)
        h.set_reorthog(reorthog, chk)
        h.seed()
        a, b = h.lanczos(niter)
        return a, b, h.reorth_log(), h.ritz(niter)[0]


@pytest.mark.parametrize("reorthog", [1, 2])
@pytest.mark.parametrize("precision", [L.NVB_FP64, L.NVB_MIXED])
def test_archive_kinds_give_the_same_recurrence(reorthog, precision, tmp_path):
    """Device, pinned-host and file archives (the last two streamed in chunks of 16 vectors):
    the same alpha/beta (1e-12 relative FP64; FP32 vectors round between chunks, 1e-5) and the
    same re-orthogonalisation intervals over 200 iterations of the 4,608-function system."""
    n = 200
    runs = [_run(k, n, reorthog, tmp_path, precision) for k in (0, 1, 2)]
    tol = 1e-12 if precision == L.NVB_FP64 else 1e-5
    a0, b0, log0, _ = runs[0]
    assert len(log0) > 0
    for a, b, log, _ in runs[1:]:
        assert np.abs(a - a0).max() <= tol * np.abs(a0).max()
        assert np.abs(b - b0).max() <= tol * np.abs(b0).max()
        if precision == L.NVB_FP64:
            assert np.array_equal(log, log0)


class _DevArray:
    """A device FP64 vector at a raw address, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}


def test_exact_overlaps_and_intervals_against_the_oracle(tmp_path):
    """reorthog=2, one iteration at a time for 200 iterations, the archive in a file.  At every
    iteration the intervals the GPU orthogonalised against equal oracle/reorth.py's rule
    (choose_intervals, partial_orthog's) applied to the GPU's omega(2, 1:it), the repeat step of
    each pair included; at every iteration without a Gram-Schmidt step, omega(2, 1:it) equals
    <r_it, v_i> computed in numpy from the residual and the file's vectors (1e-13 |r|).  (The
    GPU and the oracle's own run lose orthogonality a step or two apart, from different
    rounding, so their whole-run interval logs are not compared.)"""
    n = 200
    h, S = _handle()
    N = S.ntotal
    path = str(tmp_path / "nadvibs.34.0")
    with h:
        h.set_archive(2, n, path)
        h.set_reorthog(2, 100)
        h.seed()
        first, prev, events, checked = True, [], 0, 0
        for it in range(1, n + 1):
            h.lanczos(1)
            if it < 2:
                continue
            _, _, w = h.reorth_omega(it)
            steps = [tuple(int(v) for v in r[1:]) for r in h.reorth_log() if r[0] == it]
            ranges = reorth.choose_intervals(w, it) if first else prev
            assert steps == [tuple(r) for r in ranges], f"iteration {it}"
            if ranges:
                events += 1
                first = not first
                prev = ranges
            else:
                ptr, _ = h.lanczos_vectors()[0]  # the residual r_it, unnormalised
                r = torch.as_tensor(_DevArray(ptr, N), device="cuda").cpu().numpy().copy()
                V = np.fromfile(path, dtype=np.float64, count=it * N).reshape(it, N)
                assert np.abs(V @ r - w[1:it + 1]).max() <= 1e-13 * np.linalg.norm(r)
                checked += 1
    assert events >= 4 and checked >= 150


def test_file_archive_holds_the_reference_layout(tmp_path):
    """After k iterations the file holds v_1..v_k, each as nstates records of dimen FP64 values
    (the reference's nadvibs.34): v_1 is the seed, and the records are orthonormal."""
    n = 30
    h, S = _handle()
    path = str(tmp_path / "nadvibs.34.0")
    with h:
        h.set_archive(2, n, path)
        h.seed()
        h.lanczos(n)
    V = np.fromfile(path, dtype=np.float64)
    assert V.size == n * S.ntotal
    V = V.reshape(n, S.ntotal)
    seed = np.zeros(S.ntotal)
    for s in range(S.nstates):
        seed[s * S.dimen] = 1.0
    seed /= np.linalg.norm(seed)
    assert np.abs(V[0] - seed).max() < 1e-15
    G = V @ V.T
    assert np.abs(np.diag(G) - 1).max() < 1e-12
    assert np.abs(G[np.triu_indices(10, 1)]).max() < 1e-8  # early vectors, before ghosts form


def test_reorthogonalisation_resumes_from_the_file_archive(tmp_path):
    """reorthog=2 for n1 iterations with a file archive, restart files written, a new handle
    loads them with the same archive file and continues: the resumed alpha/beta equal an
    uninterrupted run (1e-12 relative).  The restart point is chosen after a completed pair of
    Gram-Schmidt steps (the pair toggle is not part of the restart state, as in the
    reference)."""
    n = 160
    h, _ = _handle()
    with h:
        h.set_archive(1, n)
        h.set_reorthog(2, 100)
        h.seed()
        a_full, b_full = h.lanczos(n)
        log = h.reorth_log()
    steps = sorted(set(int(r[0]) for r in log))
    cands = [i for i in range(40, 120) if sum(1 for s in steps if s <= i) % 2 == 0 and i not in steps
             and (i + 1) not in steps]
    assert cands
    n1 = cands[0]
    path = str(tmp_path / "nadvibs.34.0")
    h, _ = _handle()
    with h:
        h.set_archive(2, n, path)
        h.set_reorthog(2, 100)
        h.seed()
        h.lanczos(n1)
        h.save_restart(str(tmp_path))
    h, _ = _handle()
    with h:
        h.set_archive(2, n, path)
        h.set_reorthog(2, 100)
        h.load_restart(str(tmp_path))
        a, b = h.lanczos(n - n1)
    assert np.abs(a - a_full).max() <= 1e-12 * np.abs(a_full).max()
    assert np.abs(b - b_full).max() <= 1e-12 * np.abs(b_full).max()
