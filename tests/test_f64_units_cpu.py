"""Work-unit assignment of the FP64 grouped kernel, on the host (no GPU).

Every 64 x 64 tile of every output block must be covered exactly once along its
K range (k-tiles of 16), the parts of a split tile must own consecutive workspace
slots, and the layout must put unit j on CTA j % grid.  A numpy restatement of
what the kernel does with a unit list (each unit's K range walked through the
block's segments, parts summed in slot order) must equal the plain block GEMMs,
so the unit semantics are pinned independently of the GPU."""
import numpy as np
import pytest

from dmrg_b200 import native, workloads
from oracle import restate

BM = BN = 64
BK = 16


def random_stage(rng, n_outs, kmax):
    desc, seg_k = [], []
    for _ in range(n_outs):
        ns = int(rng.integers(0, 7))
        desc.append((int(rng.integers(1, 300)), int(rng.integers(1, 300)), ns))
        seg_k += [int(rng.integers(1, kmax)) for _ in range(ns)]
    return desc, seg_k


def tile_kts(desc, seg_k):
    out, at = {}, 0
    for o, (m, n, ns) in enumerate(desc):
        kt = sum((k + BK - 1) // BK for k in seg_k[at:at + ns])
        at += ns
        for a in range(-(-m // BM)):
            for b in range(-(-n // BN)):
                out[(o, a, b)] = kt
    return out


def check_units(desc, seg_k, grid, mode, units, nslots):
    kts = tile_kts(desc, seg_k)
    cover, slots = {}, set()
    for u in units:
        out, tm, tn, kt0, kt1, slot, part, nparts = (int(x) for x in u)
        if out < 0:
            continue
        cover.setdefault((out, tm, tn), []).append((kt0, kt1, slot, part, nparts))
        if nparts > 1:
            assert 0 <= slot < nslots and slot not in slots
            slots.add(slot)
        else:
            assert slot == -1 and part == 0
    assert set(cover) == set(kts)
    assert len(slots) == nslots
    for key, parts in cover.items():
        parts.sort()
        at = 0
        for kt0, kt1, slot, part, nparts in parts:
            assert kt0 == at and kt1 >= kt0
            at = kt1
            assert nparts == len(parts)
            assert slot - part == parts[0][2] - parts[0][3]  # one slot base per tile
        assert at == kts[key]
    if mode >= 0 and len(units) > grid:
        assert len(units) % grid == 0


@pytest.mark.parametrize("mode", [-1, 0, 1, 2])
def test_units_cover_every_tile_once(mode):
    rng = np.random.default_rng(7 + mode)
    for trial in range(60):
        desc, seg_k = random_stage(rng, int(rng.integers(1, 50)), 3000 if trial % 2 else 40)
        grid = int(rng.integers(1, 500))
        units, nslots = native.f64_units(desc, seg_k, grid, mode)
        check_units(desc, seg_k, grid, mode, units, nslots)
        if mode <= 0:
            assert nslots == 0


def microbench_stages():
    """(out_desc, seg_k) of both matvec stages of the m=1024 U(1) microbench."""
    w = workloads.microbench(1024)
    le = restate.QT.from_ibuf(*w["lenv"])
    re_ = restate.QT.from_ibuf(*w["renv"])
    ctx = restate.build_context(restate.Group(32), le, re_, 3, 2, w["sector"])
    stages = []
    for T, rows in ((re_, ctx.rmap), (le, ctx.lmap)):
        outs = {}
        for r in rows:
            blk, out_beg, n, k = int(r[0]), int(r[2]), int(r[3]), int(r[4])
            o = outs.setdefault(out_beg, [T.blocks[blk].size // k, n, []])
            o[2].append(k)
        desc = [(m, n, len(ks)) for m, n, ks in outs.values()]
        seg_k = [k for _, _, ks in outs.values() for k in ks]
        stages.append((desc, seg_k))
    return stages


def cta_loads(units, grid):
    load = np.zeros(grid)
    for j, u in enumerate(units):
        if u[0] >= 0:
            load[j % grid] += u[4] - u[3]
    return load


def test_microbench_assignment():
    """Stage 1 (914 tiles of ~21 k-tiles) keeps whole tiles; stage 2 (200 tiles of
    up to 121 k-tiles for 444 CTAs) takes equal shares: the longest CTA drops to
    within a few k-tiles of the mean."""
    (d1, k1), (d2, k2) = microbench_stages()
    grid = 444
    u1, s1 = native.f64_units(d1, k1, grid, 1)
    check_units(d1, k1, grid, 1, u1, s1)
    assert s1 == 0
    u2, s2 = native.f64_units(d2, k2, grid, 1)
    check_units(d2, k2, grid, 1, u2, s2)
    assert s2 > 0
    whole, _ = native.f64_units(d2, k2, grid, 0)
    l_whole, l_share = cta_loads(whole, grid).max(), cta_loads(u2, grid)
    assert l_whole >= 120
    assert l_share.max() <= l_share.mean() + 8


def kernel_semantics(desc, seg_k, units, rng):
    """What the kernel computes from a unit list: C_o = sum_s A_s B_s^T, each unit
    over its k-tiles of the block's segments in order, parts summed in slot order."""
    A, B, C_ref, seg_at = [], [], [], []
    at = 0
    for m, n, ns in desc:
        seg_at.append(at)
        As = [rng.standard_normal((m, k)) for k in seg_k[at:at + ns]]
        Bs = [rng.standard_normal((n, k)) for k in seg_k[at:at + ns]]
        A.append(As)
        B.append(Bs)
        C_ref.append(sum((a @ b.T for a, b in zip(As, Bs)), np.zeros((m, n))))
        at += ns
    C = [np.full((m, n), np.nan) for m, n, _ in desc]
    partial = {}
    for u in units:
        out, tm, tn, kt0, kt1, slot, part, nparts = (int(x) for x in u)
        if out < 0:
            continue
        m, n, ns = desc[out]
        r0, c0 = tm * BM, tn * BN
        acc = np.zeros((min(BM, m - r0), min(BN, n - c0)))
        kt = 0
        for s in range(ns):
            k = seg_k[seg_at[out] + s]
            for t in range(-(-k // BK)):
                if kt0 <= kt < kt1:
                    a = A[out][s][r0:r0 + BM, t * BK:(t + 1) * BK]
                    b = B[out][s][c0:c0 + BN, t * BK:(t + 1) * BK]
                    acc += a @ b.T
                kt += 1
        if nparts == 1:
            C[out][r0:r0 + BM, c0:c0 + BN] = acc
        else:
            partial[slot] = acc
            base = slot - part
            if all(base + p in partial for p in range(nparts)):
                tot = np.zeros_like(acc)
                for p in range(nparts):
                    tot = tot + partial[base + p]
                C[out][r0:r0 + BM, c0:c0 + BN] = tot
    return C, C_ref


@pytest.mark.parametrize("mode", [0, 2])
def test_unit_semantics_reproduce_block_gemms(mode):
    rng = np.random.default_rng(11)
    desc = [(70, 130, 3), (64, 64, 1), (5, 200, 2), (129, 9, 4), (33, 70, 0)]
    seg_k = [40, 17, 100, 64, 3, 250, 1, 31, 48, 16]
    units, nslots = native.f64_units(desc, seg_k, 7, mode)
    assert (nslots > 0) == (mode == 2)  # the split path is exercised
    C, C_ref = kernel_semantics(desc, seg_k, units, rng)
    for c, r in zip(C, C_ref):
        assert np.allclose(c, r, rtol=1e-12, atol=1e-12)


def test_bad_arguments_are_refused():
    with pytest.raises(native.DmrgxError):
        native.f64_units([(10, 10, 1)], [-1], 4, 0)
    with pytest.raises(native.DmrgxError):
        native.f64_units([(10, 10, 1)], [5], 0, 0)
    with pytest.raises(native.DmrgxError):
        native.f64_units([(10, 10, 1)], [5], 4, 3)
