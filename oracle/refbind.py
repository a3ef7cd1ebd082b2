"""ctypes binding to the oracle build of the reference DMRG code (oracle/_ref).

TEST INFRASTRUCTURE ONLY.  Tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use this as the checker; the product never imports
it.

The reference solves each site step with ARPACK reverse communication
(src/dsaupd.cpp:65-155 real: dsaupd 'SA', ncv=4*nev, tol=1e-10, maxiter=3n;
src/znaupd.cpp:78-197 complex: znaupd 'SR', ncv=6*nev, eigenvalues sorted by
real part).  ARPACK is not installed as a library here, so ``ref_hooks.cpp``
forwards each ``znaupd`` call to the callback registered below, which runs the
ARPACK bundled with SciPy with those same settings, applying the reference's own
``av()`` as the operator.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFDIR = os.path.join(HERE, "_ref")
VARIANTS = ("kitaev", "xyz", "potts", "u1", "s4e", "kitaev_pbc", "xyz_pbc", "potts_pbc",
            "kitaev_dropin", "xyz_dropin", "potts_dropin")
MODEL = {"kitaev": 0, "xyz": 1, "potts": 2}

_EIG_CB = C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                      C.c_void_p, C.c_void_p)
_libs: dict = {}
_keep = []


def available(variant: str = "xyz") -> bool:
    return os.path.exists(os.path.join(REFDIR, f"liboref_{variant}.so"))


def build(ref: str | None = None) -> None:
    """Compile oracle/_ref from the reference sources.

    ref: the reference checkout (the directory holding include/ and src/), else
    the DMRG_REFERENCE environment variable.  No-op when neither names an
    existing directory (the prebuilt libraries are used as they are)."""
    ref = ref or os.environ.get("DMRG_REFERENCE")
    if not ref or not os.path.isdir(ref):
        return
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref}", "-j8"], check=True)


class StepCapture:
    """Collects per-step data from inside the reference eigensolver hook."""

    def __init__(self, want=None):
        self.want = want          # predicate(step_index, info) -> bool
        self.steps = []           # list of dicts for captured steps
        self.count = 0
        self.nmatvec = 0


class Ref:
    """One oracle variant (symmetry / fermion configuration)."""

    def __init__(self, variant: str):
        if variant not in _libs:
            path = os.path.join(REFDIR, f"liboref_{variant}.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
            lib = C.CDLL(path)
            self._declare(lib)
            _libs[variant] = lib
        self.lib = _libs[variant]
        self.variant = variant
        self.N = self.lib.oref_symmetry()
        self.fermion = bool(self.lib.oref_fermion())
        self.pbc = bool(self.lib.oref_pbc())
        self.capture: StepCapture | None = None
        self._cb = _EIG_CB(self._eig_cb)
        _keep.append(self._cb)
        self.lib.oref_set_eig_callback(self._cb)
        self.energies_by_step = []
        self.evals_by_step = []

    @staticmethod
    def _declare(lib):
        vp, ip, dp, i, l = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int, C.c_long
        lib.oref_set_eig_callback.argtypes = [_EIG_CB]
        lib.oref_quiet.argtypes = [i]
        lib.oref_av.argtypes = [i, vp, vp, vp]
        lib.oref_pv_info.argtypes = [i, vp, ip]
        lib.oref_pv_maps.argtypes = [i, vp, ip, ip]
        lib.oref_pv_edge_maps.argtypes = [i, vp, ip, ip]
        lib.oref_pv_build_pbc.argtypes = [i, vp, vp, vp, vp, i, i, i, ip]
        lib.oref_pv_build_pbc.restype = vp
        lib.oref_pv_env.argtypes = [i, vp, i]
        lib.oref_pv_env.restype = vp
        lib.oref_qt_serialize.argtypes = [i, vp, ip, l, vp, l]
        lib.oref_qt_serialize.restype = l
        lib.oref_qt_new.argtypes = [i, ip, vp]
        lib.oref_qt_new.restype = vp
        lib.oref_qt_free.argtypes = [i, vp]
        lib.oref_gen_dim_sym.argtypes = [i, vp, i, vp, i, i, ip, l]
        lib.oref_gen_dim_sym.restype = l
        lib.oref_pv_build.argtypes = [i, vp, vp, i, i, i, ip]
        lib.oref_pv_build.restype = vp
        lib.oref_pv_store_layout.argtypes = [i, vp, ip, l]
        lib.oref_pv_store_layout.restype = l
        lib.oref_pv_free.argtypes = [i, vp]
        lib.oref_svd.argtypes = [i, vp, i, i, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), dp, i]
        lib.oref_env_update.argtypes = [i, vp, vp, i, i]
        lib.oref_env_update.restype = vp
        lib.oref_fuse.argtypes = [i, vp, vp, i]
        lib.oref_fuse.restype = vp
        lib.oref_mpo_tensor.argtypes = [i, dp, i, ip]
        lib.oref_mpo_tensor.restype = vp
        lib.oref_run.argtypes = [i, i, i, i, i, dp, C.c_char_p, i]
        lib.oref_tensor_read.argtypes = [i, C.c_char_p, ip, i, vp, l]
        lib.oref_tensor_read.restype = l
        lib.oref_sv_count.restype = l
        lib.oref_sv_row.argtypes = [l, ip, dp, dp, l]
        lib.oref_sv_row.restype = l
        lib.oref_en_count.restype = l
        lib.oref_en_row.argtypes = [l, ip, dp]
        lib.oref_en_row.restype = l

    # ------------------------------------------------------------------ eigensolver hook
    def _eig_cb(self, n, nev, is_complex, evals_p, evecs_p, pv):
        try:
            dt = np.complex128 if is_complex else np.float64
            cap = self.capture
            if cap is not None:
                cap.count += 1
            xin = np.zeros(n, dt)
            xout = np.zeros(n, dt)

            def mv(x):
                xin[:] = np.asarray(x).reshape(-1)
                self.lib.oref_av(is_complex, pv, xin.ctypes.data, xout.ctypes.data)
                if cap is not None:
                    cap.nmatvec += 1
                return xout.copy()

            w, v = arpack_lowest(mv, n, nev, bool(is_complex))
            for k in range(nev):
                evals_p[k] = float(w[k]) if k < len(w) else 0.0
            dst = np.ctypeslib.as_array(C.cast(evecs_p, C.POINTER(C.c_double)),
                                        shape=(n * (2 if is_complex else 1),))
            dst[:] = v.view(np.float64) if is_complex else v
            self.energies_by_step.append(float(w[0]))
            self.evals_by_step.append([float(x) for x in w[:nev]])
            if cap is not None and cap.want is not None:
                info = self.pv_info(is_complex, pv)
                if cap.want(cap.count - 1, info):
                    cap.steps.append(self.snapshot(is_complex, pv, v, w, info))
            return 0
        except Exception as exc:  # never let an exception unwind through C
            import traceback
            traceback.print_exc()
            print("oracle eigensolver callback failed:", exc)
            return 1

    # ------------------------------------------------------------------ helpers
    def pv_info(self, is_complex, pv):
        out = (C.c_int * 6)()
        self.lib.oref_pv_info(is_complex, pv, out)
        return dict(l_num=out[0], r_num=out[1], n_rmap=out[2], n_lmap=out[3], n_remap=out[4],
                    n_lemap=out[5])

    def pv_edge_maps(self, is_complex, pv, info):
        r = np.zeros((max(info["n_remap"], 1), 7), np.int32)
        lm = np.zeros((max(info["n_lemap"], 1), 7), np.int32)
        self.lib.oref_pv_edge_maps(is_complex, pv, r.ctypes.data_as(C.POINTER(C.c_int)),
                                   lm.ctypes.data_as(C.POINTER(C.c_int)))
        return r[: info["n_remap"]], lm[: info["n_lemap"]]

    def pv_maps(self, is_complex, pv, info):
        r = np.zeros((max(info["n_rmap"], 1), 7), np.int32)
        lm = np.zeros((max(info["n_lmap"], 1), 7), np.int32)
        self.lib.oref_pv_maps(is_complex, pv, r.ctypes.data_as(C.POINTER(C.c_int)),
                              lm.ctypes.data_as(C.POINTER(C.c_int)))
        return r[: info["n_rmap"]], lm[: info["n_lmap"]]

    def qt_to_py(self, is_complex, qt):
        li = self.lib.oref_qt_serialize(is_complex, qt, None, 0, None, 0)
        lv = self.lib.oref_qt_serialize(is_complex, qt, (C.c_int * 1)(), 0, None, -1)
        ib = np.zeros(li, np.int32)
        vb = np.zeros(max(lv, 1), np.complex128 if is_complex else np.float64)
        rc = self.lib.oref_qt_serialize(is_complex, qt, ib.ctypes.data_as(C.POINTER(C.c_int)),
                                        li, vb.ctypes.data, lv)
        assert rc == 0
        return ib, vb[:lv]

    def py_to_qt(self, is_complex, ibuf, vals):
        ib = np.ascontiguousarray(ibuf, np.int32)
        vb = np.ascontiguousarray(vals, np.complex128 if is_complex else np.float64)
        _keep.append((ib, vb))
        return self.lib.oref_qt_new(is_complex, ib.ctypes.data_as(C.POINTER(C.c_int)),
                                    vb.ctypes.data)

    def snapshot(self, is_complex, pv, v, w, info):
        rmap, lmap = self.pv_maps(is_complex, pv, info)
        le = self.qt_to_py(is_complex, self.lib.oref_pv_env(is_complex, pv, 0))
        re = self.qt_to_py(is_complex, self.lib.oref_pv_env(is_complex, pv, 1))
        n = v.shape[0]
        rng = np.random.default_rng(1234 + n)
        x = rng.standard_normal(n)
        if is_complex:
            x = x + 1j * rng.standard_normal(n)
        y = np.zeros(n, x.dtype)
        self.lib.oref_av(is_complex, pv, x.ctypes.data, y.ctypes.data)
        snap = dict(info=info, rmap=rmap, lmap=lmap, lenv=le, renv=re, evec=v.copy(),
                    evals=np.array(w), x=x, ax=y)
        if self.pbc:
            snap["remap"], snap["lemap"] = self.pv_edge_maps(is_complex, pv, info)
            snap["ledge"] = self.qt_to_py(is_complex, self.lib.oref_pv_env(is_complex, pv, 2))
            snap["redge"] = self.qt_to_py(is_complex, self.lib.oref_pv_env(is_complex, pv, 3))
        return snap

    # ------------------------------------------------------------------ runs
    def run(self, model: str, L: int, m: int, n: int, sector: int, params, schedule=0,
            capture: StepCapture | None = None, quiet=True):
        """Run a shipped driver's set-up and the reference schedule.

        Returns dict with 'energy' rows (l, r, E0..E5) and 'singular' rows
        (l, r, S, s0..s19, trunc_err) parsed from the reference's own output files
        (src/useful.cpp:54-102), and in full double precision: 'step_e0' /
        'step_evals' (the eigensolver's values of every step, taken in the znaupd
        hook), 'en' (every energy row at its print_energy call) and 'sv' (per step: l, r, cutoff, entropy, truncation error and the
        whole spectrum the reference's svd returned, recorded at its
        print_singular call)."""
        par = (C.c_double * 8)(*([float(p) for p in params] + [0.0] * (8 - len(params))))
        self.capture = capture
        self.energies_by_step = []
        self.evals_by_step = []
        self.lib.oref_sv_clear()
        cwd = os.getcwd()
        with tempfile.TemporaryDirectory() as td:
            os.chdir(td)
            try:
                if quiet:
                    self.lib.oref_quiet(1)
                rc = self.lib.oref_run(MODEL[model], L, m, n, sector, par, b"_oracle_.txt",
                                       schedule)
            finally:
                if quiet:
                    self.lib.oref_quiet(0)
                os.chdir(cwd)
            if rc != 0:
                raise RuntimeError(f"oref_run({model}) returned {rc} in variant {self.variant}")
            en = np.loadtxt(os.path.join(td, "energy_oracle_.txt"), ndmin=2)
            sg = np.loadtxt(os.path.join(td, "singular_oracle_.txt"), ndmin=2)
        self.capture = None
        return dict(energy=en, singular=sg, step_e0=list(self.energies_by_step),
                    step_evals=list(self.evals_by_step), sv=self.sv_rows(),
                    en=self.en_rows())

    def en_rows(self):
        """The energy rows recorded since the last run, full precision: (l, r, values)."""
        rows = []
        lr = (C.c_int * 2)()
        val = (C.c_double * 6)()
        for i in range(self.lib.oref_en_count()):
            n = self.lib.oref_en_row(i, lr, val)
            rows.append(dict(l=lr[0], r=lr[1], evals=[val[k] for k in range(max(n, 0))]))
        return rows

    def sv_rows(self):
        """The full-precision singular-value rows recorded since the last run."""
        rows = []
        head = (C.c_int * 3)()
        se = (C.c_double * 2)()
        for i in range(self.lib.oref_sv_count()):
            n = self.lib.oref_sv_row(i, head, se, None, 0)
            s = np.zeros(max(n, 1))
            self.lib.oref_sv_row(i, head, se, s.ctypes.data_as(C.POINTER(C.c_double)), n)
            rows.append(dict(l=head[0], r=head[1], cutoff=head[2], entropy=se[0],
                             trunc=se[1], s=s[:n]))
        return rows

    def tensor_read(self, is_complex, path, icap=8, vcap=1 << 20):
        """The first dense tensor of a text file, read by the reference's
        tensor<T>::read_file: (extents, values)."""
        idx = np.zeros(icap, np.int32)
        vals = np.zeros(vcap, np.complex128 if is_complex else np.float64)
        n = self.lib.oref_tensor_read(is_complex, os.fsencode(path),
                                      idx.ctypes.data_as(C.POINTER(C.c_int)), icap,
                                      vals.ctypes.data, vcap)
        if n < 0:
            raise RuntimeError(f"reference read_file failed on {path}")
        return idx, vals[:n]

    def mpo_tensor(self, model: str, params, part=0):
        par = (C.c_double * 8)(*([float(p) for p in params] + [0.0] * (8 - len(params))))
        isc = C.c_int(0)
        qt = self.lib.oref_mpo_tensor(MODEL[model], par, part, C.byref(isc))
        if not qt:
            raise RuntimeError("model not available in this oracle variant")
        out = self.qt_to_py(isc.value, qt)
        self.lib.oref_qt_free(isc.value, qt)
        return isc.value, out


def arpack_lowest(mv, n, nev, is_complex):
    """The reference's eigensolver settings on SciPy's ARPACK.

    Real: dsaupd 'SA', ncv=min(4*nev, n), tol=1e-10, maxiter=3n (src/dsaupd.cpp:68-85).
    Complex: znaupd 'SR', ncv=min(6*nev, n), same tol/maxiter, eigenvalues sorted by
    real part (src/znaupd.cpp:92-110, :180-188).  Returns (eigenvalues ascending,
    eigenvector of the lowest)."""
    from scipy.sparse.linalg import LinearOperator, eigs, eigsh, ArpackNoConvergence
    dt = np.complex128 if is_complex else np.float64
    op = LinearOperator((n, n), matvec=mv, dtype=dt)
    if n <= nev + 1:
        H = np.column_stack([mv(np.eye(n, dtype=dt)[:, k]) for k in range(n)])
        w, V = np.linalg.eigh(0.5 * (H + H.conj().T))
        return w, V[:, 0]
    try:
        if not is_complex:
            w, V = eigsh(op, k=nev, which="SA", ncv=min(4 * nev, n), tol=1e-10, maxiter=3 * n)
        else:
            w, V = eigs(op, k=nev, which="SR", ncv=min(6 * nev, n), tol=1e-10, maxiter=3 * n)
    except ArpackNoConvergence as e:
        w, V = e.eigenvalues, e.eigenvectors
    order = np.argsort(np.real(w))
    w = np.real(w[order])
    V = V[:, order]
    return w, V[:, 0].astype(dt)
