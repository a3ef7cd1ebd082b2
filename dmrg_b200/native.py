"""ctypes binding of libdmrgx.so (the C ABI declared in include/dmrgx.h).

This module is plumbing: it loads the in-tree CUDA library and converts numpy
arrays to pointers.  There is no fallback: if the library is missing the import
of a context fails with an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libdmrgx.so")

F64, C128 = 0, 1
PREC_FP64, PREC_BF16X3, PREC_TF32X3 = 0, 1, 2
SCHED_GROUPED, SCHED_PER_BLOCK = 0, 1
GROUP_Z2CUBED = -8  # group_n of the Z2 x Z2 x Z2 (S4E) fusion rule
MEM_HOST, MEM_DEVICE = 0, 1
BOUNDARY_OPEN, BOUNDARY_PERIODIC = 0, 1

# every entry point declared in include/dmrgx.h, with (restype, argtypes)
_vp, _ip, _i, _i64 = C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_int64
_i64p, _dp = C.POINTER(C.c_int64), C.POINTER(C.c_double)
SIGNATURES = {
    "dmrgx_last_error": (C.c_char_p, []),
    "dmrgx_version": (C.c_char_p, []),
    "dmrgx_ctx_create": (_i, [C.POINTER(_vp), _i, _i]),
    "dmrgx_ctx_destroy": (None, [_vp]),
    "dmrgx_set_precision": (_i, [_vp, _i]),
    "dmrgx_plan_build": (_i, [_vp, _ip, _vp, _ip, _vp, _i, _i, _i, _i, _i]),
    "dmrgx_build_maps": (_i, [_ip, _ip, _i, _i, _i, _i, _i, _i64p, _ip, _i64, _ip, _i64]),
    "dmrgx_plan_from_maps": (_i, [_vp, _i64, _i64, _ip, _i, _vp, _i64p, _i, _ip, _i, _vp,
                                  _i64p, _i]),
    "dmrgx_plan_build_pbc": (_i, [_vp, _ip, _vp, _ip, _vp, _ip, _vp, _ip, _vp, _i, _i, _i, _i,
                                  _i]),
    "dmrgx_build_maps_pbc": (_i, [_ip, _ip, _ip, _ip, _i, _i, _i, _i, _i, _i64p, _ip, _i64, _ip,
                                  _i64, _ip, _i64, _ip, _i64]),
    "dmrgx_plan_from_maps_pbc": (_i, [_vp, _i64, _i64, _ip, _i, _vp, _i64p, _i, _ip, _i, _vp,
                                      _i64p, _i, _i64, _ip, _i, _vp, _i64p, _i, _ip, _i, _vp,
                                      _i64p, _i]),
    "dmrgx_plan_info": (_i, [_vp, _i64p]),
    "dmrgx_plan_edge_info": (_i, [_vp, _i64p]),
    "dmrgx_plan_maps": (_i, [_vp, _ip, _ip]),
    "dmrgx_plan_edge_maps": (_i, [_vp, _ip, _ip]),
    "dmrgx_set_boundary": (_i, [_vp, _i]),
    "dmrgx_set_solver": (_i, [_vp, _i, _i, _i]),
    "dmrgx_save_state": (_i, [_vp, C.c_char_p]),
    "dmrgx_load_state": (_i, [_vp, C.c_char_p]),
    "dmrgx_plan_psi_layout": (_i, [_vp, _ip, _i64]),
    "dmrgx_av": (_i, [_vp, _vp, _vp, _i]),
    "dmrgx_av_noalloc": (_i, [_i, _i64, _i64, _ip, _i, _vp, _i64p, _i, _ip, _i, _vp, _i64p, _i,
                              _vp, _vp, _vp]),
    "dmrgx_eigsolve": (_i, [_vp, _i, _i, C.c_double, _i, _vp, _dp, _vp, _i64p]),
    "dmrgx_dmrg": (_i, [_vp, _i, _i, _i, _i, _i, _dp, _i, _dp, _dp, _ip, _i64p, _i64, _i64p,
                        _dp]),
    "dmrgx_set_schedule": (_i, [_vp, _i]),
    "dmrgx_split_tuning": (_i, [_vp, _ip, _i]),
    "dmrgx_f64_units": (_i, [_i, _ip, _ip, _i, _i, _ip, _i64, _i64p, _i64p]),
    "dmrgx_matvec_launches": (_i, [_vp, _ip]),
    "dmrgx_step_seconds": (_i, [_vp, _dp, _i64, _i64p]),
    "dmrgx_singular": (_i, [_vp, _dp, _dp, _ip, _i64, _i64p]),
    "dmrgx_step_split": (_i, [_vp, _dp, _i64, _i64p]),
    "dmrgx_svd": (_i, [_vp, _ip, _vp, _i, _i, _i, _i, _i64p]),
    "dmrgx_group_create": (_i, [C.POINTER(_vp), _i]),
    "dmrgx_group_destroy": (None, [_vp]),
    "dmrgx_set_group": (_i, [_vp, _vp]),
    "dmrgx_group_stats": (_i, [_vp, _i64p]),
    "dmrgx_svd_result": (_i, [_vp, _ip, _vp, _ip, _vp, _dp]),
    "dmrgx_run_seconds": (_i, [_vp, _dp, _i]),
    "dmrgx_adjoint": (_i, [_vp, _i, _dp, _i, _dp, _i64, _i64p, _dp, _dp]),
    "dmrgx_expect": (_i, [_vp, _dp, _i, _dp]),
    "dmrgx_profile": (_i, [_vp, _i]),
    "dmrgx_profile_read": (_i, [_vp, _dp, _i]),
    "dmrgx_stream": (_vp, [_vp]),
    "dmrgx_sync": (_i, [_vp]),
}

_lib = None


class DmrgxError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DmrgxError(f"{LIB_PATH} is not built; run `python -m dmrg_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise DmrgxError(f"dmrgx error {rc}: {lib().dmrgx_last_error().decode()}")


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _i64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def build_maps(lenv_meta, renv_meta, l_num, r_num, sector, group_n, fermion):
    """Host-only sector bookkeeping: (n, d_store, rmap, lmap) in the reference row format."""
    lm = np.ascontiguousarray(lenv_meta, np.int32)
    rm = np.ascontiguousarray(renv_meta, np.int32)
    info = np.zeros(4, np.int64)
    _check(lib().dmrgx_build_maps(_ip(lm), _ip(rm), l_num, r_num, sector, group_n, fermion,
                                  _i64p(info), None, 0, None, 0))
    rmap = np.zeros((max(1, info[2]), 7), np.int32)
    lmap = np.zeros((max(1, info[3]), 7), np.int32)
    _check(lib().dmrgx_build_maps(_ip(lm), _ip(rm), l_num, r_num, sector, group_n, fermion,
                                  _i64p(info), _ip(rmap), rmap.shape[0], _ip(lmap),
                                  lmap.shape[0]))
    return int(info[0]), int(info[1]), rmap[: info[2]], lmap[: info[3]]


def f64_units(out_desc, seg_k, grid, mode):
    """Host-only work units of the FP64 grouped kernel for one stage: out_desc rows
    (rows, real columns, segment count) per output block, seg_k the segments' K
    extents block by block.  Returns (units as an (n, 8) int array: out, tm, tn, kt0,
    kt1, slot, part, nparts; workspace slots)."""
    od = np.ascontiguousarray(np.asarray(out_desc, np.int32).reshape(-1))
    sk = np.ascontiguousarray(np.asarray(seg_k, np.int32).reshape(-1))
    if sk.size == 0:
        sk = np.zeros(1, np.int32)
    cnt = np.zeros(1, np.int64)
    slots = np.zeros(1, np.int64)
    _check(lib().dmrgx_f64_units(od.size // 3, _ip(od), _ip(sk), grid, mode, None, 0,
                                 _i64p(cnt), _i64p(slots)))
    units = np.zeros((max(1, int(cnt[0])), 8), np.int32)
    _check(lib().dmrgx_f64_units(od.size // 3, _ip(od), _ip(sk), grid, mode, _ip(units),
                                 int(cnt[0]), _i64p(cnt), _i64p(slots)))
    return units[: int(cnt[0])], int(slots[0])


def build_maps_pbc(lenv_meta, renv_meta, ledge_meta, redge_meta, l_num, r_num, sector, group_n,
                   fermion):
    """build_maps with the periodic edge pair: (n, d_store, rmap, lmap, e_store, remap, lemap)."""
    m = [np.ascontiguousarray(x, np.int32) for x in (lenv_meta, renv_meta, ledge_meta, redge_meta)]
    info = np.zeros(7, np.int64)
    _check(lib().dmrgx_build_maps_pbc(*[_ip(x) for x in m], l_num, r_num, sector, group_n,
                                      fermion, _i64p(info), None, 0, None, 0, None, 0, None, 0))
    maps = [np.zeros((max(1, int(info[k])), 7), np.int32) for k in (2, 3, 5, 6)]
    args = []
    for a in maps:
        args += [_ip(a), a.shape[0]]
    _check(lib().dmrgx_build_maps_pbc(*[_ip(x) for x in m], l_num, r_num, sector, group_n,
                                      fermion, _i64p(info), *args))
    rmap, lmap, remap, lemap = (a[: int(info[k])] for a, k in zip(maps, (2, 3, 5, 6)))
    return int(info[0]), int(info[1]), rmap, lmap, int(info[4]), remap, lemap


def av_noalloc(dtype, n, d_store, rmap, renv_dev, renv_sizes, lmap, lenv_dev, lenv_sizes,
               in_dev, out_dev, stream=0):
    """dmrgx_av_noalloc: device pointers for values and vectors, host task lists.

    The work is queued on ``stream`` (0 = legacy default stream); nothing is
    allocated on the device."""
    rmap = np.ascontiguousarray(rmap, np.int32).reshape(-1, 7)
    lmap = np.ascontiguousarray(lmap, np.int32).reshape(-1, 7)
    rs = np.ascontiguousarray(renv_sizes, np.int64)
    ls = np.ascontiguousarray(lenv_sizes, np.int64)
    _check(lib().dmrgx_av_noalloc(dtype, n, d_store, _ip(rmap), rmap.shape[0],
                                  C.c_void_p(renv_dev), _i64p(rs), rs.size, _ip(lmap),
                                  lmap.shape[0], C.c_void_p(lenv_dev), _i64p(ls), ls.size,
                                  C.c_void_p(in_dev), C.c_void_p(out_dev), C.c_void_p(stream)))


class Group:
    """A solve group (dmrgx_group_create): contexts that join it and run dmrg()
    from their own threads meet at every site step's eigensolve, which runs as
    one lock-step Lanczos with one grouped matvec launch per stage for all."""

    def __init__(self, members):
        p = C.c_void_p()
        _check(lib().dmrgx_group_create(C.byref(p), int(members)))
        self.ptr = p

    def stats(self):
        """(Krylov rounds, grouped launches, member matvecs served)."""
        out = np.zeros(3, np.int64)
        _check(lib().dmrgx_group_stats(self.ptr, _i64p(out)))
        return tuple(int(v) for v in out)

    def close(self):
        if self.ptr:
            lib().dmrgx_group_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """A dmrgx context (one GPU stream, device environments, a matvec plan)."""

    def __init__(self, dtype=F64, device=0):
        self.dtype = dtype
        self._np = np.complex128 if dtype == C128 else np.float64
        p = C.c_void_p()
        _check(lib().dmrgx_ctx_create(C.byref(p), dtype, device))
        self.ptr = p
        self.n = self.d_store = 0

    def close(self):
        if self.ptr:
            lib().dmrgx_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, prec):
        _check(lib().dmrgx_set_precision(self.ptr, prec))

    def matvec_launches(self) -> int:
        """Kernel launches of one matvec with the current plan and settings."""
        out = np.zeros(1, np.int32)
        _check(lib().dmrgx_matvec_launches(self.ptr, _ip(out)))
        return int(out[0])

    def split_tuning(self):
        """Autotuner choice per split stage: list of (cfg, halve, cap_scale, tuned);
        cap_scale -1 means no K-split."""
        out = np.zeros(8, np.int32)
        _check(lib().dmrgx_split_tuning(self.ptr, _ip(out), 8))
        return [(int(out[4 * i]), bool(out[4 * i + 1]), out[4 * i + 2] / 100.0, bool(out[4 * i + 3]))
                for i in range(2)]

    def set_schedule(self, schedule):
        """SCHED_GROUPED (default) or SCHED_PER_BLOCK (one cuBLAS GEMM per task row)."""
        _check(lib().dmrgx_set_schedule(self.ptr, schedule))

    def plan_build(self, lenv, renv, l_num, r_num, sector, group_n, fermion=0):
        """lenv/renv: (meta int array, packed values) pairs."""
        lm = np.ascontiguousarray(lenv[0], np.int32)
        rm = np.ascontiguousarray(renv[0], np.int32)
        lv = np.ascontiguousarray(lenv[1], self._np)
        rv = np.ascontiguousarray(renv[1], self._np)
        _check(lib().dmrgx_plan_build(self.ptr, _ip(lm), lv.ctypes.data, _ip(rm), rv.ctypes.data,
                                      l_num, r_num, sector, group_n, fermion))
        self._refresh()

    def plan_build_pbc(self, lenv, renv, ledge, redge, l_num, r_num, sector, group_n,
                       fermion=0):
        """Periodic chain: (meta, values) of lenv, renv and the edge pair ledge, redge."""
        ms = [np.ascontiguousarray(t[0], np.int32) for t in (lenv, renv, ledge, redge)]
        vs = [np.ascontiguousarray(t[1], self._np) for t in (lenv, renv, ledge, redge)]
        args = []
        for m, v in zip(ms, vs):
            args += [_ip(m), v.ctypes.data]
        _check(lib().dmrgx_plan_build_pbc(self.ptr, *args, l_num, r_num, sector, group_n,
                                          fermion))
        self._refresh()

    def plan_from_maps_pbc(self, n, d_store, rmap, renv_vals, renv_sizes, lmap, lenv_vals,
                           lenv_sizes, e_store, remap, redge_vals, redge_sizes, lemap,
                           ledge_vals, ledge_sizes):
        """The drop-in for a PBC build's lanczos<T>: both pairs' task lists and blocks."""
        keep = []

        def m7(a):
            a = np.ascontiguousarray(a, np.int32).reshape(-1, 7)
            keep.append(a)
            return _ip(a), a.shape[0]

        def vals(v, sz):
            v = np.ascontiguousarray(v, self._np)
            sz = np.ascontiguousarray(sz, np.int64)
            keep.extend([v, sz])
            return v.ctypes.data, _i64p(sz), sz.size

        _check(lib().dmrgx_plan_from_maps_pbc(
            self.ptr, n, d_store, *m7(rmap), *vals(renv_vals, renv_sizes), *m7(lmap),
            *vals(lenv_vals, lenv_sizes), e_store, *m7(remap), *vals(redge_vals, redge_sizes),
            *m7(lemap), *vals(ledge_vals, ledge_sizes)))
        self._refresh()

    def edge_maps(self):
        """(e_store, remap, lemap) of the current plan's edge pair."""
        info = np.zeros(3, np.int64)
        _check(lib().dmrgx_plan_edge_info(self.ptr, _i64p(info)))
        r = np.zeros((max(1, int(info[1])), 7), np.int32)
        l = np.zeros((max(1, int(info[2])), 7), np.int32)
        _check(lib().dmrgx_plan_edge_maps(self.ptr, _ip(r), _ip(l)))
        return int(info[0]), r[: int(info[1])], l[: int(info[2])]

    def save_state(self, path):
        """Write the state of the last dmrg() (site tensors, centre) to a text file."""
        _check(lib().dmrgx_save_state(self.ptr, os.fsencode(path)))

    def load_state(self, path):
        """Read a state written by save_state; adjoint() and expect() then apply to it."""
        _check(lib().dmrgx_load_state(self.ptr, os.fsencode(path)))

    def set_solver(self, nev=6, ncv=0, predict=False):
        """Site-step eigensolver of the next dmrg(): eigenvalues per step, Krylov basis
        (0: the reference's), White's wavefunction prediction."""
        _check(lib().dmrgx_set_solver(self.ptr, nev, ncv, int(bool(predict))))

    def set_group(self, group):
        """Join a solve group (None: leave it)."""
        _check(lib().dmrgx_set_group(self.ptr, group.ptr if group is not None else None))

    def set_boundary(self, boundary):
        """BOUNDARY_OPEN (default) or BOUNDARY_PERIODIC for the next dmrg()."""
        _check(lib().dmrgx_set_boundary(self.ptr, boundary))

    def plan_from_maps(self, n, d_store, rmap, renv_vals, renv_sizes, lmap, lenv_vals,
                       lenv_sizes):
        rmap = np.ascontiguousarray(rmap, np.int32).reshape(-1, 7)
        lmap = np.ascontiguousarray(lmap, np.int32).reshape(-1, 7)
        rv = np.ascontiguousarray(renv_vals, self._np)
        lv = np.ascontiguousarray(lenv_vals, self._np)
        rs = np.ascontiguousarray(renv_sizes, np.int64)
        ls = np.ascontiguousarray(lenv_sizes, np.int64)
        _check(lib().dmrgx_plan_from_maps(self.ptr, n, d_store, _ip(rmap), rmap.shape[0],
                                          rv.ctypes.data, _i64p(rs), rs.size, _ip(lmap),
                                          lmap.shape[0], lv.ctypes.data, _i64p(ls), ls.size))
        self._refresh()

    def _refresh(self):
        info = np.zeros(8, np.int64)
        _check(lib().dmrgx_plan_info(self.ptr, _i64p(info)))
        self.n, self.d_store = int(info[0]), int(info[1])
        self.n_rmap, self.n_lmap = int(info[2]), int(info[3])
        self.flops = int(info[4])

    def maps(self):
        r = np.zeros((max(1, self.n_rmap), 7), np.int32)
        l = np.zeros((max(1, self.n_lmap), 7), np.int32)
        _check(lib().dmrgx_plan_maps(self.ptr, _ip(r), _ip(l)))
        return r[: self.n_rmap], l[: self.n_lmap]

    def av(self, x, out=None):
        """Host arrays in/out (the reference-facing call); ``out``: a host array of n
        elements to write (e.g. page-locked), else a new one."""
        x = np.ascontiguousarray(x, self._np)
        assert x.size == self.n
        y = np.empty(self.n, self._np) if out is None else out
        assert y.dtype == self._np and y.size == self.n and y.flags.c_contiguous
        _check(lib().dmrgx_av(self.ptr, x.ctypes.data, y.ctypes.data, MEM_HOST))
        return y

    def av_device(self, x_ptr: int, y_ptr: int):
        """Device pointers (e.g. torch tensors' data_ptr()) on this context's stream."""
        _check(lib().dmrgx_av(self.ptr, C.c_void_p(x_ptr), C.c_void_p(y_ptr), MEM_DEVICE))

    def eigsolve(self, nev=6, ncv=0, tol=1e-10, maxiter=0, v0=None):
        """Lowest nev eigenvalues and the lowest eigenvector (device Lanczos).

        Returns (evals, evec, info dict)."""
        ev = np.zeros(max(nev, 1))
        vec = np.zeros(self.n, self._np)
        info = np.zeros(6, np.int64)
        p0 = None
        if v0 is not None:
            v0 = np.ascontiguousarray(v0, self._np)
            p0 = v0.ctypes.data
        _check(lib().dmrgx_eigsolve(self.ptr, nev, ncv, tol, maxiter, p0,
                                    ev.ctypes.data_as(_dp), vec.ctypes.data, _i64p(info)))
        d = dict(matvecs=int(info[0]), matvecs_fp64=int(info[1]), cycles=int(info[2]),
                 corrections=int(info[3]), converged=int(info[4]),
                 residual=float(info[5:6].view(np.float64)[0]))
        return ev[:nev], vec, d

    def dmrg(self, model, L, m, sweeps, params, sector=0, cap=100000):
        """Run the reference dmrg() schedule on the GPU.  model: 'kitaev' (F64
        context), 'xyz' or 'potts' (C128 context).  Returns a dict of per-step
        arrays (lr, energies[:, 6], trunc, entropy, s20[:, 20], nsv, matvecs) and
        timings: the rows of the reference's energy and singular-value files
        (src/useful.cpp:54-102) in full precision."""
        code = {"kitaev": 0, "xyz": 1, "potts": 2, "xyz_real": 3}[model]
        par = np.ascontiguousarray(params, np.float64)
        en = np.zeros((cap, 6))
        tr = np.zeros(cap)
        lr = np.zeros((cap, 2), np.int32)
        mv = np.zeros(cap, np.int64)
        ns = np.zeros(1, np.int64)
        sec = np.zeros(5)
        _check(lib().dmrgx_dmrg(self.ptr, code, L, m, sweeps, sector, par.ctypes.data_as(_dp),
                                par.size, en.ctypes.data_as(_dp), tr.ctypes.data_as(_dp),
                                _ip(lr), _i64p(mv), cap, _i64p(ns), sec.ctypes.data_as(_dp)))
        k = int(ns[0])
        self._L = L
        self._nparams = 3 if code == 0 else min(4, max(3, par.size))
        ent = np.zeros(max(k, 1))
        s20 = np.zeros((max(k, 1), 20))
        nsv = np.zeros(max(k, 1), np.int32)
        _check(lib().dmrgx_singular(self.ptr, ent.ctypes.data_as(_dp), s20.ctypes.data_as(_dp),
                                    _ip(nsv), k, _i64p(ns)))
        return dict(lr=lr[:k], energies=en[:k], trunc=tr[:k], entropy=ent[:k], s20=s20[:k],
                    nsv=nsv[:k], matvecs=mv[:k],
                    seconds=dict(total=sec[0], eig=sec[1], svd=sec[2], env=sec[3], fuse=sec[4]))

    def run_seconds(self):
        """Time split of the last dmrg() run: steps, eig, svd, env, fuse, plan (seconds)."""
        out = np.zeros(10)
        _check(lib().dmrgx_run_seconds(self.ptr, out.ctypes.data_as(_dp), 10))
        return dict(zip(("steps", "eig", "svd", "env", "fuse", "plan", "plan_maps",
                         "plan_images", "plan_split", "plan_tune"), out.tolist()))

    def step_seconds(self):
        """Wall seconds of every site step of the last dmrg() run."""
        ns = np.zeros(1, np.int64)
        _check(lib().dmrgx_step_seconds(self.ptr, None, 0, _i64p(ns)))
        out = np.zeros(max(1, int(ns[0])))
        _check(lib().dmrgx_step_seconds(self.ptr, out.ctypes.data_as(_dp), out.size, _i64p(ns)))
        return out[:int(ns[0])]

    def svd(self, meta, vals, num, cutoff, group_n, fermion):
        """Block SVD with truncation (the reference's qtensor::svd): returns
        ((U meta, U values), (V meta, V values), singular values)."""
        m = np.ascontiguousarray(meta, np.int32)
        dt = np.complex128 if self.dtype == C128 else np.float64
        v = np.ascontiguousarray(vals, dt)
        sz = np.zeros(5, np.int64)
        _check(lib().dmrgx_svd(self.ptr, _ip(m), v.ctypes.data, num, cutoff, group_n, fermion,
                               _i64p(sz)))
        um = np.zeros(max(1, sz[0]), np.int32)
        uv = np.zeros(max(1, sz[1]), dt)
        vm = np.zeros(max(1, sz[2]), np.int32)
        vv = np.zeros(max(1, sz[3]), dt)
        sv = np.zeros(max(1, sz[4]))
        _check(lib().dmrgx_svd_result(self.ptr, _ip(um), uv.ctypes.data, _ip(vm), vv.ctypes.data,
                                      sv.ctypes.data_as(_dp)))
        return (um[:sz[0]], uv[:sz[1]]), (vm[:sz[2]], vv[:sz[3]]), sv[:sz[4]]

    def step_split(self):
        """Per-step split of the last dmrg() run: rows (eig, svd, env, fuse, plan) seconds."""
        ns = np.zeros(1, np.int64)
        _check(lib().dmrgx_step_split(self.ptr, None, 0, _i64p(ns)))
        out = np.zeros((max(1, int(ns[0])), 5))
        _check(lib().dmrgx_step_split(self.ptr, out.ctypes.data_as(_dp), out.shape[0], _i64p(ns)))
        return out[:int(ns[0])]

    def adjoint(self, nparams=None, recompute=False, want_w=False):
        """Gradient of the last dmrg() ground-state energy: dict with dE_dparams
        (model parameter order), checks (E0, centre energy spread, max
        |<dE/dW_k, W_k> - E0|, dropped weight), seconds and, with want_w, the
        per-site dE/dW_k (L x w_len doubles, bulk MPO block layout)."""
        npar = nparams if nparams is not None else self._nparams
        g = np.zeros(max(1, npar))
        chk = np.zeros(4)
        sec = np.zeros(1)
        wl = np.zeros(1, np.int64)
        _check(lib().dmrgx_adjoint(self.ptr, 1 if recompute else 0, g.ctypes.data_as(_dp), npar,
                                   None, 0, _i64p(wl), chk.ctypes.data_as(_dp),
                                   sec.ctypes.data_as(_dp)))
        out = dict(dE_dparams=g[:npar].copy(), checks=chk, seconds=float(sec[0]))
        if want_w:
            # a second sweep with the tensor output (the centre ends at the right edge)
            w = np.zeros((self._L, int(wl[0])))
            _check(lib().dmrgx_adjoint(self.ptr, 0, g.ctypes.data_as(_dp), npar,
                                       w.ctypes.data_as(_dp), w.size, _i64p(wl), None, None))
            out["dE_dW"] = w
        return out

    def expect(self, params):
        """<Psi|H(params)|Psi> of the last dmrg() state for the same model."""
        par = np.ascontiguousarray(params, np.float64)
        v = np.zeros(1)
        _check(lib().dmrgx_expect(self.ptr, par.ctypes.data_as(_dp), par.size,
                                  v.ctypes.data_as(_dp)))
        return float(v[0])

    def profile(self, enable: bool):
        _check(lib().dmrgx_profile(self.ptr, 1 if enable else 0))

    def profile_read(self):
        """(matvecs, ms per slot [split, stage 1, stage 2]) since profile(True)."""
        out = np.zeros(4)
        _check(lib().dmrgx_profile_read(self.ptr, out.ctypes.data_as(_dp), 4))
        return int(out[0]), out[1:4].copy()

    def stream(self) -> int:
        return int(lib().dmrgx_stream(self.ptr) or 0)

    def sync(self):
        _check(lib().dmrgx_sync(self.ptr))
