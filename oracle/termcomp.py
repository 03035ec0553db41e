"""ORACLE (test infrastructure only) -- CPU restatement of the NadVibS input stage.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this module, as the
checker.  The product (``nadvibs_b200``) never imports it.

Parity status: UNPINNED against the reference.  The reference is Fortran 90 + MPI + Global
Arrays, no Fortran compiler exists in this image, and the reference ships no example input
or output for this path (its example archive is missing).  This module is a line-by-line
restatement of the reference's semantics, checked by known-answer tests instead.

Restates:
* ``get_keywords``  Source/secondary.f90:826-870   (namelist keys, defaults, derived flags)
* ``read_basis``    Source/top.f90:32-86           (cpindx, noterms)
* ``read_constants`` Source/top.f90:88-246         (list-directed reads, monomial enumeration
  Source/top.f90:153-168, cross-block merge :170-197, 1/prod(omega^(p/2)) scaling :216,
  both (a,b) and (b,a) pairs :218-231)
* ``union``         Source/secondary.f90:1034-1054
* ``compute_allIndex`` step enumeration Source/secondary.f90:27-64,98-124 (smax, shift order)
"""
from __future__ import annotations

import math
import re

import numpy as np


# ---------------------------------------------------------------- list-directed reading
def _split_tokens(line: str) -> list[str]:
    line = line.split("!")[0] if "!" in line else line
    return [t for t in re.split(r"[\s,]+", line.strip()) if t]


def _to_float(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "E"))


class ListDirected:
    """Fortran list-directed ``read(unit,*)`` over the lines of a file.

    ``skip()`` is ``read(unit,*)`` with no items (one record consumed).  ``values(n)`` reads
    n items, continuing onto following records when a record runs out, and discards the
    remainder of the last record read, as list-directed input does.  ``r*c`` repeat counts
    are honoured.
    """

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0

    def skip(self) -> None:
        if self.pos >= len(self.lines):
            raise EOFError("end of file while skipping a record")
        self.pos += 1

    def values(self, n: int) -> list[float]:
        out: list[float] = []
        while len(out) < n:
            if self.pos >= len(self.lines):
                raise EOFError(f"end of file: wanted {n} values, got {len(out)}")
            toks = _split_tokens(self.lines[self.pos])
            self.pos += 1
            for t in toks:
                if t.startswith("/"):
                    return out + [0.0] * 0  # slash ends the read, remaining items unchanged
                if "*" in t:
                    r, c = t.split("*", 1)
                    out.extend([_to_float(c)] * int(r))
                else:
                    out.append(_to_float(t))
                if len(out) >= n:
                    break
        return out[:n]


# ---------------------------------------------------------------- namelist (basis.in)
NAMELIST_DEFAULTS = dict(
    niter=1, natoms=2, nmodes=1, nstates=1, basis=[1] * 100, restart=0, bconv=0, idroots=0,
    soroots=0, reorthog=0, chkorthog=100, nseg=1, ztoler=1e-20, maxdisk=1000.0,
    weights=[1.0] * 10, shiftref=0, nirreps=1, npirr=None, ordr=2, initstate=[0] * 100,
)
_INT_KEYS = {"niter", "natoms", "nmodes", "nstates", "restart", "bconv", "idroots", "soroots",
             "reorthog", "chkorthog", "nseg", "shiftref", "nirreps", "ordr"}
_ARR_KEYS = {"basis": 100, "initstate": 100, "npirr": 10, "weights": 10}


def read_namelist(text: str) -> dict:
    """Parse the ``&NADVIBS ... /`` group (Source/secondary.f90:844-846) with its defaults
    (:835-843) and derived quantities (:847-869)."""
    m = re.search(r"&nadvibs(.*?)(/|&end)", text, flags=re.S | re.I)
    if not m:
        raise ValueError("no &NADVIBS namelist group")
    body = "\n".join(l.split("!")[0] for l in m.group(1).splitlines())
    kv = dict(NAMELIST_DEFAULTS)
    kv["basis"] = [1] * 100
    kv["initstate"] = [0] * 100
    kv["weights"] = [1.0] * 10
    npirr = [0] * 10
    npirr[0] = 1  # npirr(1)=nmodes is evaluated with the default nmodes=1 (secondary.f90:838)
    # tokens: name(idx)? = values
    parts = re.split(r"([A-Za-z_][A-Za-z_0-9]*\s*(?:\(\s*\d+\s*\))?)\s*=", body)
    for i in range(1, len(parts), 2):
        key = parts[i].strip().lower()
        vals = []
        for t in re.split(r"[\s,]+", parts[i + 1].strip()):
            if not t:
                continue
            if "*" in t:
                r, c = t.split("*", 1)
                vals.extend([c] * int(r))
            else:
                vals.append(t)
        idx = 1
        mm = re.match(r"([a-z_0-9]+)\s*\(\s*(\d+)\s*\)", key)
        if mm:
            key, idx = mm.group(1), int(mm.group(2))
        if key in _ARR_KEYS:
            conv = float if key == "weights" else (lambda s: int(float(s.replace("d", "e"))))
            if key == "npirr":
                arr = npirr
            else:
                arr = kv[key]
            for o, v in enumerate(vals):
                arr[idx - 1 + o] = conv(v.replace("d", "e").replace("D", "E")) if key == "weights" else conv(v)
        elif key in _INT_KEYS:
            kv[key] = int(float(vals[0].replace("d", "e").replace("D", "E")))
        elif key in ("ztoler", "maxdisk"):
            kv[key] = _to_float(vals[0])
        else:
            raise ValueError(f"unknown namelist key {key}")
    # a conflict between sum(npirr) and nmodes disables symmetry (secondary.f90:847-851)
    if sum(npirr) != kv["nmodes"]:
        kv["nirreps"] = 1
        npirr = [0] * 10
        npirr[0] = kv["nmodes"]
    kv["npirr"] = npirr
    kv["orthog"] = kv["reorthog"] > 0
    kv["orthogexact"] = kv["reorthog"] > 1
    kv["idroots"] = abs(kv["idroots"])
    kv["soroots"] = abs(kv["soroots"])
    kv["neworigin"] = kv["shiftref"] != 0
    kv["savevecs"] = kv["orthog"] or kv["idroots"] > 0 or kv["soroots"] > 0
    kv["bjiconv"] = 10.0 ** (-kv["bconv"])
    kv["nfunc"] = kv["basis"][: kv["nmodes"]]
    kv["statew"] = kv["weights"][: kv["nstates"]]
    kv["istate"] = kv["initstate"][: kv["nmodes"]]
    kv["dimen"] = int(np.prod(kv["nfunc"], dtype=np.int64))
    return kv


# ---------------------------------------------------------------- term compiler
def numut(n: int, d: int) -> int:
    """C(n+d-1, d) -- Source/function.f90:253-258."""
    return math.comb(n + d - 1, d)


def cpindx(nstates: int) -> list[tuple[int, int]]:
    """Block k (1-based) <-> (i, j), i >= j, k = i(i-1)/2 + j  (Source/top.f90:79-85)."""
    out = [None] * (nstates * (nstates + 1) // 2)
    for i in range(1, nstates + 1):
        for j in range(1, i + 1):
            out[i * (i - 1) // 2 + j - 1] = (i, j)
    return out


def union(lst: list[int]) -> list[int]:
    """Unique elements in order of first appearance (Source/secondary.f90:1034-1054)."""
    u: list[int] = []
    for v in lst:
        if v not in u:
            u.append(v)
    return u


def otab_sequence(nmodes: int, order: int):
    """Monomial digits in file order (Source/top.f90:153-168)."""
    otab = [1] * order
    otab[0] = 0
    for _ in range(numut(nmodes, order)):
        otab[0] += 1
        for l in range(order - 1):
            if otab[l] > nmodes:
                otab[l] = 1
                otab[l + 1] += 1
        for l in range(order - 2, -1, -1):
            if otab[l] < otab[l + 1]:
                otab[l] = otab[l + 1]
        yield list(otab)


def read_nadvibs(text: str, nmodes: int, nstates: int, ordr: int, neworigin: bool = False):
    """The list-directed reads of Source/top.f90:122-135.  Returns
    (omega[M], concoef[nstblks], pot[nstblks][ordr] arrays, extras)."""
    rd = ListDirected(text)
    nstblks = nstates * (nstates + 1) // 2
    rd.skip()
    omega = np.array(rd.values(nmodes))
    concoef = np.zeros(nstblks)
    pot = []
    for i in range(nstblks):
        rd.skip()
        concoef[i] = rd.values(1)[0]
        per = []
        for j in range(1, ordr + 1):
            rd.skip()
            per.append(np.array(rd.values(numut(nmodes, j))))
        pot.append(per)
    extra = {}
    if neworigin:
        rd.skip(); extra["bomega"] = np.array(rd.values(nmodes))
        rd.skip(); extra["dvec"] = np.array(rd.values(nmodes))
        rd.skip(); extra["tmat"] = np.array(rd.values(nmodes * nmodes))
    return omega, concoef, pot, extra


class TermTable:
    """The reference's nzindx / nzblks / nzcoef arrays (Source/progdata.f90:52-53,59)."""

    def __init__(self):
        self.nztrms: list[int] = []          # per cnt = 1..ordr
        self.modes: list[list[int]] = []     # 1-based, decreasing
        self.pows: list[list[int]] = []
        self.pairs: list[list[tuple[int, int]]] = []   # (row state, column state), 1-based
        self.coefs: list[list[float]] = []

    @property
    def nterms(self) -> int:
        return len(self.modes)


def compile_terms(nmodes, nstates, ordr, omega, concoef, pot, ztoler=1e-20) -> TermTable:
    """Restates the merge and scaling of Source/top.f90:153-231."""
    cp = cpindx(nstates)
    nstblks = len(cp)
    temp = {c: [] for c in range(1, ordr + 1)}  # cnt -> [modes, pows, blocks, coefs]
    for i in range(1, nstblks + 1):
        for j in range(1, ordr + 1):
            for k, otab in enumerate(otab_sequence(nmodes, j)):
                uniq = union(otab)
                cnt = len(uniq)
                val = float(pot[i - 1][j - 1][k])
                if abs(val) >= ztoler:
                    counts = [otab.count(u) for u in uniq]
                    loc = None
                    for n, ent in enumerate(temp[cnt]):
                        if ent[0] == uniq and ent[1] == counts:
                            loc = n
                            break
                    if loc is None:
                        temp[cnt].append([list(uniq), counts, [i], [val]])
                    else:
                        temp[cnt][loc][2].append(i)
                        temp[cnt][loc][3].append(val)
    tt = TermTable()
    for cnt in range(1, ordr + 1):
        tt.nztrms.append(len(temp[cnt]))
        for modes, counts, blocks, vals in temp[cnt]:
            dval = 1.0
            for m, p in zip(modes, counts):
                dval = dval / math.sqrt(omega[m - 1] ** p)
            prs, cfs = [], []
            for b, v in zip(blocks, vals):
                r, c = cp[b - 1]
                prs.append((r, c)); cfs.append(v * dval)
                if r != c:
                    prs.append((c, r)); cfs.append(v * dval)
            tt.modes.append(modes); tt.pows.append(counts); tt.pairs.append(prs); tt.coefs.append(cfs)
    return tt


def smax_of(pw: int, nf: int) -> int:
    """Largest usable shift for power ``pw`` in a mode of ``nf`` functions
    (Source/secondary.f90:33-37)."""
    s = pw
    while s > nf - 1:
        s -= 2
    return s


def term_steps(modes: list[int], pows: list[int], nfunc: list[int]) -> list[list[int]]:
    """Shift vectors of one term in the order of Source/secondary.f90:98-124 (last digit
    fastest, steps of 2), including the all-zero shift, which the reference skips."""
    sm = [smax_of(p, nfunc[m - 1]) for m, p in zip(modes, pows)]
    if any(s < 0 for s in sm):
        return []
    i = len(modes)
    sdir = [-s for s in sm]
    sdir[i - 1] -= 2
    out = []
    nsteps = 1
    for s in sm:
        nsteps *= s + 1
    for _ in range(nsteps):
        l = i - 1
        while sdir[l] >= sm[l]:
            sdir[l] = -sm[l]
            l -= 1
        sdir[l] += 2
        out.append(list(sdir))
    return out


def is_diag_term(pows: list[int], modes: list[int], nfunc: list[int]) -> bool:
    """All (reduced) powers even (Source/secondary.f90:49-61)."""
    return all(smax_of(p, nfunc[m - 1]) % 2 == 0 for m, p in zip(modes, pows))


def dblks(tt: TermTable, concoef, nstates: int, nfunc: list[int]) -> list[tuple[int, int]]:
    """Off-diagonal state pairs (i>j only) that receive a diagonal coupling
    (Source/top.f90:528-553)."""
    cp = cpindx(nstates)
    chk = np.zeros((nstates + 1, nstates + 1), dtype=int)
    for k, c in enumerate(concoef):
        if abs(c) > 1e-16:
            i, j = cp[k]
            chk[i, j] = chk[j, i] = 1
    for t in range(tt.nterms):
        if is_diag_term(tt.pows[t], tt.modes[t], nfunc):
            for (a, b) in tt.pairs[t]:
                chk[a, b] = 1
    out = []
    for i in range(1, nstates + 1):
        for j in range(1, i):
            if chk[i, j]:
                out.append((i, j))
    return out
