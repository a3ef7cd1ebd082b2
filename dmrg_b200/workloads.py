"""Synthetic matvec inputs of the shapes the benchmark and tests run.

The H_eff microbench: a two-site wavefunction [m_l, n1, n2, m_r] with physical
dimension d=2 per site (charges n in {0, 1}), left and right bond dimension
m = 1024 split into nine U(1) sectors q = -4..4 with sizes proportional to
exp(-q^2/8) (largest-remainder rounding, symmetric, odd remainder to q=0), and an
MPO bond of D=5 channels with charges {0, +1, -1, 0, 0} (I, S+, S-, Sz, I), i.e.
channel-sector sizes {0: 3, +1: 1, -1: 1}.

Environments use the reference's leg orders (reference src/core.cpp:188-192):
  L~ = [m_bra, d_bra, D, m_ket, d_ket],  R~ = [d_bra, m_bra, D, d_ket, m_ket].
Block existence (charge conservation):
  L~ block (q_b, n_b, c, q_k, n_k) exists iff q_b + n_b = q_k + n_k - c
  R~ block (n_b, q_b, c, n_k, q_k) exists iff n_b - q_b = n_k - q_k + c
U(1) labels are embedded in Z_32 (all charges here lie in [-10, 10]); left bond
legs carry label q mod 32, right bond legs carry -q mod 32 (the reference's
rule is that all legs of psi add up to the sector, src/useful.cpp:172-181), so
psi sits in sector 1 (q_r = q_l + n1 + n2 - 1).
Blocks are listed in lexicographic order of their label tuples; entries are iid
N(0,1) FP64 from numpy's default_rng(seed), filled block by block in that order.

Metadata uses the flat int layout of include/dmrgx.h ("meta").
"""
from __future__ import annotations

import numpy as np

GROUP_N = 32
PSI_SECTOR = 1


def sector_sizes(m: int, qmax: int = 4, width: float = 8.0):
    """Sizes of the U(1) sectors q=-qmax..qmax proportional to exp(-q^2/width),
    summing to m: floor of the exact shares, then the remainder handed out by
    largest fractional part in symmetric +-q pairs, with an odd remainder to q=0."""
    qs = np.arange(-qmax, qmax + 1)
    w = np.exp(-qs.astype(float) ** 2 / width)
    exact = m * w / w.sum()
    base = np.floor(exact).astype(int)
    rem = m - int(base.sum())
    frac = exact - base
    # pairs (q, -q) for q>0 in decreasing fractional part
    order = sorted(range(1, qmax + 1), key=lambda q: -frac[q + qmax])
    sizes = base.copy()
    i = 0
    while rem >= 2 and i < len(order):
        q = order[i]
        sizes[qmax + q] += 1
        sizes[qmax - q] += 1
        rem -= 2
        i += 1
    if rem:
        sizes[qmax] += rem
    return {int(q): int(s) for q, s in zip(qs, sizes)}


def _meta(dims, dirs, syms):
    out = [len(dims), len(syms)] + [len(d) for d in dims]
    for d in dims:
        out += list(d)
    out += list(dirs)
    for s in syms:
        out += list(s)
    return np.array(out, np.int32)


def microbench(m: int = 1024, seed: int = 20261203, qmax: int = 4, width: float = 8.0):
    """Synthetic (L~, R~) for one two-site H_eff matvec (l_num=3, r_num=2, sector 1).

    Returns dict(lenv=(meta, vals), renv=(meta, vals), l_num, r_num, sector, group_n,
    sizes).  ``m`` smaller than 1024 gives a scaled-down instance of the same
    structure for quick parity tests."""
    N = GROUP_N
    sizes = sector_sizes(m, qmax, width)
    mdim_left = [0] * N
    mdim_right = [0] * N
    for q, s in sizes.items():
        mdim_left[q % N] = s
        mdim_right[(-q) % N] = s
    ddim = [1, 1] + [0] * (N - 2)
    # D channels: charge 0 -> 3 channels, +1 -> 1, -1 -> 1
    Ddim = [0] * N
    Ddim[0] = 3
    Ddim[1] = 1
    Ddim[N - 1] = 1
    charges_D = {0: 0, 1: 1, N - 1: -1}
    qlab = {q % N: q for q in sizes}          # left label -> charge
    qlab_r = {(-q) % N: q for q in sizes}     # right label -> charge

    rng = np.random.default_rng(seed)

    # L~ = [m_bra, d_bra, D, m_ket, d_ket]
    lsyms = []
    for a in range(N):
        if a not in qlab:
            continue
        for nb in (0, 1):
            for c in range(N):
                if c not in charges_D:
                    continue
                for k in range(N):
                    if k not in qlab:
                        continue
                    for nk in (0, 1):
                        if qlab[a] + nb == qlab[k] + nk - charges_D[c]:
                            lsyms.append((a, nb, c, k, nk))
    ldims = [mdim_left, ddim, Ddim, mdim_left, ddim]
    lvals = []
    for s in lsyms:
        shp = [ldims[i][s[i]] for i in range(5)]
        lvals.append(rng.standard_normal(int(np.prod(shp))))
    # R~ = [d_bra, m_bra, D, d_ket, m_ket]
    rsyms = []
    for nb in (0, 1):
        for a in range(N):
            if a not in qlab_r:
                continue
            for c in range(N):
                if c not in charges_D:
                    continue
                for nk in (0, 1):
                    for k in range(N):
                        if k not in qlab_r:
                            continue
                        if nb - qlab_r[a] == nk - qlab_r[k] + charges_D[c]:
                            rsyms.append((nb, a, c, nk, k))
    rdims = [ddim, mdim_right, Ddim, ddim, mdim_right]
    rvals = []
    for s in rsyms:
        shp = [rdims[i][s[i]] for i in range(5)]
        rvals.append(rng.standard_normal(int(np.prod(shp))))
    dirs = [0] * 5
    return dict(
        lenv=(_meta(ldims, dirs, lsyms), np.concatenate(lvals)),
        renv=(_meta(rdims, dirs, rsyms), np.concatenate(rvals)),
        l_num=3, r_num=2, sector=PSI_SECTOR, group_n=N, fermion=0, sizes=sizes)


def random_z2cubed(seed: int = 3, complex_: bool = False, keep: float = 0.7, msize: int = 4):
    """Random (L~, R~) pair under the Z2 x Z2 x Z2 fusion rule (labels 0..7 fusing
    by XOR, group_n -8), with fermion directions, for l_num=3, r_num=2, sector 5.

    Leg orders follow the reference's two-site environments (src/core.cpp:188-192):
    L~ = [m_bra, d_bra, D, m_ket, d_ket], R~ = [d_bra, m_bra, D, d_ket, m_ket].
    Bond legs: every label present with 1..msize states; physical legs: labels
    {0, 3, 5, 6} with one state each; MPO leg: labels {0, 1, 2, 4} with 1..2 states.
    A block exists where the XOR of its labels is 0, and is kept with probability
    ``keep`` (missing blocks exercise the task-list matching).  Directions
    L~ (+1, +1, 0, -1, -1), R~ (+1, +1, 0, -1, -1) make every parity sign of the
    task list (src/qtensor.cpp:1078-1085) appear."""
    rng = np.random.default_rng(seed)
    N = 8
    mdim = [int(v) for v in rng.integers(1, msize + 1, N)]
    ddim = [1 if a in (0, 3, 5, 6) else 0 for a in range(N)]
    Ddim = [int(rng.integers(1, 3)) if a in (0, 1, 2, 4) else 0 for a in range(N)]

    def blocks(dims):
        syms = []
        for t in np.ndindex(*(N,) * len(dims)):
            if any(dims[i][t[i]] == 0 for i in range(len(dims))):
                continue
            x = 0
            for a in t:
                x ^= a
            if x == 0 and rng.random() < keep:
                syms.append(tuple(int(a) for a in t))
        return syms

    def values(dims, syms):
        out = []
        for sy in syms:
            k = int(np.prod([dims[i][sy[i]] for i in range(len(dims))]))
            v = rng.standard_normal(k)
            if complex_:
                v = v + 1j * rng.standard_normal(k)
            out.append(v)
        return np.concatenate(out)

    ldims = [mdim, ddim, Ddim, mdim, ddim]
    rdims = [ddim, mdim, Ddim, ddim, mdim]
    lsyms, rsyms = blocks(ldims), blocks(rdims)
    dirs = [1, 1, 0, -1, -1]
    return dict(
        lenv=(_meta(ldims, dirs, lsyms), values(ldims, lsyms)),
        renv=(_meta(rdims, dirs, rsyms), values(rdims, rsyms)),
        l_num=3, r_num=2, sector=5, group_n=-8, fermion=1)


def random_psi(n: int, seed: int = 7, complex_: bool = False):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(n)
    if complex_:
        x = x + 1j * rng.standard_normal(n)
    return x
