"""Packed observables, FP64 oracle (TEST INFRASTRUCTURE ONLY, see ``oracle/__init__.py``).

Restates the estimators of ``code/measure/transverse_spin.py:44-119`` and
``code/measure/dwave_packed.py:24-103`` from explicit fermion operators on each configuration:
for a term O_t the connected configuration is s' = O_t^dag s (up to its coefficient c), so
<s|O_t|s'> = c and the local value is c psi(s') / psi(s).  The sample mean of the local values,
term by term, is the estimate of <O_t>; the diagonal term of each family comes from the
occupations.  Mode m of a configuration is bit m of an integer (up modes first, site
x Ly + y), and an operator on mode m carries (-1)^(occupied modes below m).
"""

from __future__ import annotations

import numpy as np

from .hubbard import _apply_annihilate, _apply_create


def _bits(s) -> int:
    b = 0
    for m in np.flatnonzero(np.asarray(s) > 0):
        b |= 1 << int(m)
    return b


def _config(bits: int, M2: int) -> np.ndarray:
    return np.array([1 if (bits >> m) & 1 else -1 for m in range(M2)], np.int8)


def _apply(bits: int, ops):
    """ops applied left to right: [(mode, create), ...] -> (bits, coefficient) or (None, 0)."""
    c = 1
    for m, create in ops:
        bits, sg = (_apply_create if create else _apply_annihilate)(bits, m)
        if bits is None:
            return None, 0
        c *= sg
    return bits, c


def bond_pairs(Lx: int, Ly: int):
    """(c, d) of the terms t = 4 site + 2 axis + o: the bond from site along +x (axis 0) or +y
    (axis 1), (c, d) = (site, neighbour) for o = 0 and swapped for o = 1."""
    out = []
    for site in range(Lx * Ly):
        x, y = divmod(site, Ly)
        for axis in range(2):
            hi = ((x + 1) % Lx) * Ly + y if axis == 0 else x * Ly + (y + 1) % Ly
            out += [(site, hi), (hi, site)]
    return out


def terms(kind: str, Lx: int, Ly: int, a0: int, a1: int = 0):
    """[(bin, ops of O_t^dag applied to s, diagonal)] of a family.  O_t^dag's operators are
    listed in the order they act on s."""
    N = Lx * Ly
    out = []
    if kind == "transverse":
        a = a0
        xa, ya = divmod(a, Ly)
        for chan in range(2):
            for j in range(N):
                xj, yj = divmod(j, Ly)
                r = ((xj - xa) % Lx) * Ly + (yj - ya) % Ly
                if j == a:
                    out.append((chan * N + r, None, "up_not_dn" if chan == 0 else "dn_not_up"))
                    continue
                # O = S+_a S-_j = c+(a up) c(a dn) c+(j dn) c(j up); chan 1 swaps the spins.
                au, ad, ju, jd = (a, N + a, j, N + j) if chan == 0 else (N + a, a, N + j, j)
                out.append((chan * N + r, [(au, False), (ad, True), (jd, False), (ju, True)],
                            None))
    elif kind == "pair":
        a, b = a0, a1
        for t, (c, d) in enumerate(bond_pairs(Lx, Ly)):
            if (c, d) == (a, b):
                out.append((t, None, "pair"))
                continue
            # O = c+(a up) c+(b dn) c(d dn) c(c up)
            out.append((t, [(a, False), (N + b, False), (N + d, True), (c, True)], None))
    else:  # "hop": O = c+(i s) c(j s)
        i, sg = a0, a1
        for j in range(N):
            if j == i:
                out.append((j, None, "n"))
                continue
            out.append((j, [(sg * N + i, False), (sg * N + j, True)], None))
    return out


def packed_mean(s: np.ndarray, amp_fn, kind: str, Lx: int, Ly: int, a0: int, a1: int = 0,
                psi=None) -> np.ndarray:
    """Sample means of every term of the family (``amp_fn(configs) -> (sign, logabs)``)."""
    s = np.asarray(s)
    N = Lx * Ly
    M2 = 2 * N
    if psi is None:
        psi = amp_fn(s)
    sg0, la0 = psi
    tl = terms(kind, Lx, Ly, a0, a1)
    out = np.zeros(len(tl))
    for b in range(s.shape[0]):
        bits = _bits(s[b])
        conns, coef, bins = [], [], []
        for k, ops, diag in tl:
            if diag is not None:
                occ = lambda m: (bits >> m) & 1  # noqa: E731
                if diag == "up_not_dn":
                    out[k] += occ(a0) and not occ(N + a0)
                elif diag == "dn_not_up":
                    out[k] += occ(N + a0) and not occ(a0)
                elif diag == "pair":
                    out[k] += occ(a0) and occ(N + a1)
                else:
                    out[k] += occ(a1 * N + a0)
                continue
            nb, c = _apply(bits, ops)
            if nb is None:
                continue
            conns.append(_config(nb, M2))
            coef.append(c)
            bins.append(k)
        if conns:
            sg, la = amp_fn(np.array(conns))
            vals = np.array(coef) * sg * sg0[b] * np.exp(la - la0[b])
            np.add.at(out, np.array(bins), vals)
    return out / s.shape[0]
