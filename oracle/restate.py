"""CPU restatement (numpy) of the reference's H_eff hot path.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import it.

Parity pin: every function here is checked against the reference itself, built
from its own sources into ``oracle/_ref`` (``tests/test_oracle.py``), and
against the golden fixtures committed under ``tests/golden/`` that were made
from that build (``tests/golden/make_golden.py``).

Block-sparse tensor convention (reference include/qtensor.h:26-31): ``dims[leg][sector]``
sizes, ``syms[block][leg]`` sector labels, ``dirs[leg]`` fermion directions,
``blocks[b]`` dense row-major (last index fastest, include/tensor.h:36-45).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from itertools import product

import numpy as np


# ----------------------------------------------------------------------------- fusion rule
@dataclass(frozen=True)
class Group:
    """Z_N fusion rule ``ss`` and parity ``ff`` (src/useful.cpp:28-39), or with
    ``N = -8`` the Z2 x Z2 x Z2 rule of the reference's S4E build
    (src/useful.cpp:4-27): labels 0..7 fuse by bitwise XOR (a negative label -b
    stands for b) and the parity is odd exactly for labels 2, 3, 4, 5.

    ``fermion=False`` gives parity 0 everywhere: the bosonic models with the
    reference's direction signs compiled out (the reference applies them to every
    model, src/qtensor.cpp:1084, which makes bosonic H_eff non-Hermitian)."""
    N: int
    fermion: bool = False

    @property
    def order(self) -> int:
        return 8 if self.N == -8 else self.N

    def ss(self, a: int, b: int) -> int:
        if self.N == -8:
            return a ^ (-b if b < 0 else b)
        return (a + b + self.N) % self.N

    def ff(self, a: int) -> int:
        if not self.fermion:
            return 0
        if self.N == -8:
            return 1 if a in (2, 3, 4, 5) else 0
        return a % 2

    def sign(self, x: int, y: int) -> int:
        # 1 - 2*((ff(x)*ff(y)) % 2), the reference's sign form
        return 1 - 2 * ((self.ff(x) * self.ff(y)) % 2)


# ----------------------------------------------------------------------------- tensor type
@dataclass
class QT:
    dims: list                      # dims[leg] = list of sector sizes
    syms: list                      # list of tuples, one per block
    blocks: list                    # list of ndarrays
    dirs: list = field(default_factory=list)

    @property
    def nleg(self):
        return len(self.dims)

    def block_shape(self, sym):
        return tuple(self.dims[l][s] for l, s in enumerate(sym))

    def packed(self):
        if not self.blocks:
            return np.zeros(0)
        return np.concatenate([b.reshape(-1) for b in self.blocks])

    # serialised form shared with oracle/ref_hooks.cpp
    def to_ibuf(self):
        nl = self.nleg
        out = [nl, len(self.syms)] + [len(d) for d in self.dims]
        for d in self.dims:
            out += list(d)
        dirs = self.dirs if self.dirs else [0] * nl
        out += list(dirs)
        for s in self.syms:
            out += list(s)
        return np.array(out, np.int32)

    @staticmethod
    def from_ibuf(ib, vals):
        ib = [int(x) for x in ib]
        k = 0
        nl, nb = ib[0], ib[1]
        k = 2
        nsec = ib[k:k + nl]
        k += nl
        dims = []
        for l in range(nl):
            dims.append(ib[k:k + nsec[l]])
            k += nsec[l]
        dirs = ib[k:k + nl]
        k += nl
        syms, blocks = [], []
        v = 0
        for b in range(nb):
            s = tuple(ib[k:k + nl])
            k += nl
            shp = tuple(dims[l][s[l]] for l in range(nl))
            sz = int(np.prod(shp)) if shp else 1
            syms.append(s)
            blocks.append(np.array(vals[v:v + sz]).reshape(shp))
            v += sz
        return QT(dims, syms, blocks, dirs)


def generate_map(index):
    """All label tuples in lexicographic order (src/useful.cpp:105-134)."""
    return [tuple(t) for t in product(*[range(n) for n in index])]


def get_dimension(dim, sym):
    """Total size of a packed block list (src/useful.cpp:137-148)."""
    return int(sum(np.prod([dim[j][s[j]] for j in range(len(dim))]) for s in sym))


def generate_dim_sym(G: Group, ldims, lnum, rdims, rnum, sector):
    """Sector list and ORDER of the packed wavefunction (src/useful.cpp:151-194).

    dim = last ``lnum`` legs of the left env + last ``rnum`` legs of the right env.
    Blocks ordered by left charge s = 0..N-1, then left label tuple, then right label
    tuple (each lexicographic); kept where ss(lsym, rsym) == sector."""
    dim = [list(d) for d in ldims[len(ldims) - lnum:]] + [list(d) for d in rdims[len(rdims) - rnum:]]
    lmap = generate_map([len(d) for d in dim[:lnum]])
    rmap = generate_map([len(d) for d in dim[lnum:]])
    sym = []
    if sector != -1:
        for s in range(G.order):
            t = G.ss(sector, -s)
            for lt in lmap:
                lsym = 0
                for x in lt:
                    lsym = G.ss(lsym, x)
                for rt in rmap:
                    rsym = 0
                    for x in rt:
                        rsym = G.ss(rsym, x)
                    if lsym == s and rsym == t:
                        sym.append(tuple(lt) + tuple(rt))
    else:
        sym = [tuple([0] * len(dim))]
    return dim, sym


def get_map(G: Group, T: QT, dim, sym, ta="N", tb="T", num=1, beta=0, back=False,
            dim_ret=None, sym_ret=None):
    """Task list of the block-sparse matvec (src/qtensor.cpp:997-1119).

    Each row is [block, in_beg, out_beg, rows, cols, beta, alpha]; one GEMM
    out[rows?] = alpha*T[block] x in^T per row.  With ``back=False`` the output
    layout (dim_ret, sym_ret) is created in first-appearance order and alpha is
    the fermionic sign; with ``back=True`` the given output layout is used, beta=0
    on the first write to each output block and 1 afterwards, alpha = 1.
    Returns (rows, dim_ret, sym_ret)."""
    nT = T.nleg
    indexa = nT - num if ta in "Nn" else 0
    indexb = 0 if tb in "Nn" else len(dim) - num
    for i in range(num):
        if list(T.dims[indexa + i]) != list(dim[indexb + i]):
            raise ValueError("get_map: dimensions differ")
    new_dim_ret = [list(T.dims[i]) for i in range(nT) if i < indexa or i >= indexa + num] + \
                  [list(dim[i]) for i in range(len(dim)) if i < indexb or i >= indexb + num]
    # per input block: total size, "row" size, begin offset
    sdim = []
    beg = 0
    for s in sym:
        tot = int(np.prod([dim[k][s[k]] for k in range(len(dim))]))
        if indexb:
            row = int(np.prod([dim[k][s[k]] for k in range(indexb)]))
        else:
            row = int(np.prod([dim[k][s[k]] for k in range(num)]))
        sdim.append((tot, row, beg))
        beg += tot
    rows = []
    if back:
        dim_ret = [list(d) for d in dim_ret]
        keys = [_loc(s, dim_ret) for s in sym_ret]
        offs = [0]
        for s in sym_ret[:-1]:
            offs.append(offs[-1] + int(np.prod([dim_ret[j][s[j]] for j in range(len(dim_ret))])))
        first = [True] * len(keys)
        sym_ret = list(sym_ret)
    else:
        dim_ret = new_dim_ret
        keys, offs, sym_ret = [], [0], []
        first = []
    for i, ts in enumerate(T.syms):
        for j, s in enumerate(sym):
            if any(ts[indexa + k] != s[indexb + k] for k in range(num)):
                continue
            if sdim[j][0] == 0:
                continue
            row = [i, sdim[j][2], offs[-1], sdim[j][1], sdim[j][0] // sdim[j][1], beta, 1]
            if not back:
                d_b = 0
                dirs = T.dirs if T.dirs else [0] * nT
                for k in range(nT):
                    d_b = G.ss(d_b, ts[k] * dirs[k])
                a_p = 0
                for k in range(len(dim) - num):
                    a_p = G.ss(a_p, s[k])
                row[6] = G.sign(d_b, a_p)
            st = [ts[k] for k in range(nT) if k < indexa or k >= indexa + num] + \
                 [s[k] for k in range(len(dim)) if k < indexb or k >= indexb + num]
            loc = _loc(st, dim_ret)
            same = False
            for t, key in enumerate(keys):
                if key == loc:
                    row[2] = offs[t]
                    if back and first[t]:
                        first[t] = False
                    else:
                        row[5] = 1
                    rows.append(list(row))
                    same = True
            if not same and not back:
                d = int(np.prod([dim_ret[q][st[q]] for q in range(len(dim_ret))]))
                offs.append(offs[-1] + d)
                keys.append(loc)
                sym_ret.append(tuple(st))
                rows.append(list(row))
    return np.array(rows, np.int64).reshape(-1, 7), dim_ret, sym_ret


def _loc(st, dim_ret):
    loc = 0
    for q in range(len(dim_ret)):
        loc = loc * len(dim_ret[q]) + st[q]
    return loc


def contract_map(T: QT, out, x, rows, num):
    """Apply a task list (src/qtensor.cpp:986-994 -> src/tensor.cpp:698-718, 'N','T'):
    out[ob : ob+M*N] = alpha * A[M x K] . X[N x K]^T + beta * out, row-major."""
    for r in rows:
        blk, ib, ob, nrow, ncol, beta, alpha = (int(v) for v in r)
        A = T.blocks[blk]
        K = int(np.prod(A.shape[A.ndim - num:]))
        M = A.size // K
        N, Kx = nrow, ncol
        assert Kx == K
        Am = A.reshape(M, K)
        X = x[ib: ib + N * K].reshape(N, K)
        C = alpha * (Am @ X.T)
        if beta:
            out[ob: ob + M * N] += C.reshape(-1)
        else:
            out[ob: ob + M * N] = C.reshape(-1)


@dataclass
class MatvecContext:
    """The reference's ``lanczos<T>`` matvec context (include/val_for_lanczos.h:7-24)."""
    lenv: QT
    renv: QT
    l_num: int
    r_num: int
    rmap: np.ndarray
    lmap: np.ndarray
    dim: list
    sym: list
    dim_ret: list
    sym_ret: list
    n: int
    d_store: int
    # periodic chains (PBC build, include/val_for_lanczos.h:18-23): the edge pair
    ledge: QT | None = None
    redge: QT | None = None
    remap: np.ndarray | None = None
    lemap: np.ndarray | None = None
    e_store: int = 0


def build_context(G: Group, lenv: QT, renv: QT, l_num: int, r_num: int, sector: int,
                  ledge: QT | None = None, redge: QT | None = None):
    """What a reference step function does before the eigensolve
    (src/core.cpp:201-202 and :236-247 for update_two); with ledge/redge the
    edge pair of a periodic chain (:241-247): remap against the same psi layout
    with its own store layout, lemap with beta = 1 into psi."""
    dim, sym = generate_dim_sym(G, lenv.dims, l_num - 1, renv.dims, r_num, sector)
    n = get_dimension(dim, sym)
    rmap, dim_ret, sym_ret = get_map(G, renv, dim, sym, "N", "T", r_num, 0)
    d_store = get_dimension(dim_ret, sym_ret)
    # input = the store layout, output = the fixed wavefunction layout (back=True)
    lmap, _, _ = get_map(G, lenv, dim_ret, sym_ret, "N", "T", l_num, 0, True, dim, sym)
    ctx = MatvecContext(lenv, renv, l_num, r_num, rmap, lmap, dim, sym, dim_ret, sym_ret,
                        n, d_store)
    if ledge is not None:
        remap, edim, esym = get_map(G, redge, dim, sym, "N", "T", r_num, 0)
        ctx.e_store = get_dimension(edim, esym)
        ctx.lemap, _, _ = get_map(G, ledge, edim, esym, "N", "T", l_num, 1, True, dim, sym)
        ctx.remap, ctx.ledge, ctx.redge = remap, ledge, redge
    return ctx


def av(ctx: MatvecContext, x):
    """out = lenv (x)_{l_num} (renv (x)_{r_num} x)   (src/core.cpp:22-31), plus
    ledge (x) (redge (x) x) on a periodic chain (:27-30).

    Output sectors that no task writes are zero here (the reference leaves them
    untouched)."""
    store = np.zeros(ctx.d_store, np.result_type(x, ctx.renv.blocks[0]))
    contract_map(ctx.renv, store, x, ctx.rmap, ctx.r_num)
    out = np.zeros(ctx.n, store.dtype)
    contract_map(ctx.lenv, out, store, ctx.lmap, ctx.l_num)
    if ctx.ledge is not None:
        est = np.zeros(ctx.e_store, store.dtype)
        contract_map(ctx.redge, est, x, ctx.remap, ctx.r_num)
        contract_map(ctx.ledge, out, est, ctx.lemap, ctx.l_num)
    return out


# ----------------------------------------------------------------------------- text files
def _value(tok: str, is_complex: bool):
    if is_complex:
        re_, im = tok.strip("()").split(",")
        return complex(float(re_), float(im))
    return float(tok)


def read_tensor_text(tokens, pos: int, is_complex: bool):
    """tensor<T>::read_file (src/tensor.cpp:260-271) on a token stream: the number
    of indices, the extents, then prod(extents) values (std::complex's stream
    form "(re,im)" for complex).  Returns (extents, values, next position)."""
    n = int(tokens[pos])
    ext = [int(t) for t in tokens[pos + 1: pos + 1 + n]]
    pos += 1 + n
    cnt = int(np.prod(ext)) if ext else 1
    vals = np.array([_value(t, is_complex) for t in tokens[pos: pos + cnt]],
                    np.complex128 if is_complex else np.float64)
    return ext, vals, pos + cnt


def format_tensor_text(ext, vals, is_complex: bool) -> str:
    """tensor<T>::write_file (src/tensor.cpp:249-257): the same fields, values at 32
    significant digits."""
    def fmt(x):
        return f"{x:.32g}"
    parts = [str(len(ext))] + [str(e) for e in ext]
    for v in np.ravel(vals):
        parts.append(f"({fmt(v.real)},{fmt(v.imag)})" if is_complex else fmt(float(v)))
    return " ".join(parts)


def read_state(path: str):
    """Parse a dmrgx state file (dmrgx_save_state): header fields, parameters, and
    every tensor as (QT, per-block extents)."""
    tok = open(path).read().split()
    assert tok[0] == "dmrgx-mps" and tok[1] == "1", "not a dmrgx state file"
    head = {tok[i]: tok[i + 1] for i in range(2, 16, 2)}  # model L sector m center f energy
    f = int(head["f"])
    i = 16
    assert tok[i] == "params"
    npar = int(tok[i + 1])
    params = [float(t) for t in tok[i + 2: i + 2 + npar]]
    i += 2 + npar
    tensors = {}
    while tok[i] != "end":
        if tok[i] == "site":
            name, i = f"site{int(tok[i + 1])}", i + 2
        else:
            name, i = "centre", i + 1
        nleg, nblk = int(tok[i]), int(tok[i + 1])
        i += 2
        dims = []
        for _ in range(nleg):
            ns = int(tok[i])
            dims.append([int(t) for t in tok[i + 1: i + 1 + ns]])
            i += 1 + ns
        dirs = [int(t) for t in tok[i: i + nleg]]
        i += nleg
        syms = []
        for _ in range(nblk):
            syms.append(tuple(int(t) for t in tok[i: i + nleg]))
            i += nleg
        blocks = []
        for b in range(nblk):
            ext, vals, i = read_tensor_text(tok, i, f == 2)
            assert ext == [dims[l][syms[b][l]] for l in range(nleg)]
            blocks.append(vals.reshape(ext))
        tensors[name] = QT(dims=dims, dirs=dirs, syms=syms, blocks=blocks)
    return dict(header={k: (float(v) if k == "energy" else int(v)) for k, v in head.items()},
                params=params, tensors=tensors)

