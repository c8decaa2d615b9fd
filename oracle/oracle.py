"""ctypes front end to the CPU references the tests compare against. TEST INFRASTRUCTURE ONLY.

Only the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only to check or time against it.

Two CPU references live here:

* ``liboracle.so`` -- the C restatement of the HPCG 3.1 reference path
  (``hpcg_oracle.c``; each routine cites the reference file:line it follows).
* ``_ref/libhpcg_ref.so`` -- the reference itself, compiled from its own sources
  with ``ref_bridge.cpp`` (present only where the reference tree was available
  at build time). It pins the restatement.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SLOTS = 27

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


class _Level(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("n", C.c_int),
        ("nnz", C.c_void_p), ("cols", C.c_void_p), ("vals", C.c_void_p),
        ("diag", C.c_void_p), ("f2c", C.c_void_p),
    ]


class _Level32(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("nnz", C.c_void_p), ("cols", C.c_void_p), ("vals", C.c_void_p),
        ("diag", C.c_void_p), ("f2c", C.c_void_p),
    ]


def _load_oracle():
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
    lib = C.CDLL(path)
    lib.ora_generate.restype = C.c_int64
    lib.ora_generate.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ora_f2c.argtypes = [C.c_int, C.c_int, C.c_int, _i32p]
    lib.ora_spmv.argtypes = [C.POINTER(_Level), _f64p, _f64p]
    lib.ora_symgs.argtypes = [C.POINTER(_Level), _f64p, _f64p]
    lib.ora_gs_forward.argtypes = [C.POINTER(_Level), _f64p, _f64p]
    lib.ora_gs_backward.argtypes = [C.POINTER(_Level), _f64p, _f64p]
    lib.ora_restriction.argtypes = [C.c_int, _i32p, _f64p, _f64p, _f64p]
    lib.ora_prolongation.argtypes = [C.c_int, _i32p, _f64p, _f64p]
    lib.ora_mg.restype = C.c_int
    lib.ora_mg.argtypes = [C.POINTER(_Level), C.c_int, C.c_int, _f64p, _f64p]
    lib.ora_dot.restype = C.c_double
    lib.ora_dot.argtypes = [C.c_int, _f64p, _f64p]
    lib.ora_waxpby.argtypes = [C.c_int, C.c_double, _f64p, C.c_double, _f64p, _f64p]
    lib.ora_residual.restype = C.c_double
    lib.ora_residual.argtypes = [C.c_int, _f64p, _f64p]
    lib.ora_cg.restype = C.c_int
    lib.ora_cg.argtypes = [C.POINTER(_Level), C.c_int, _f64p, _f64p, C.c_int, C.c_double, C.c_int,
                           C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double), _f64p]
    lib.ora_symgs_skip.argtypes = [C.POINTER(_Level), _f64p, _f64p, C.c_int]
    lib.ora_mg_skip.restype = C.c_int
    lib.ora_mg_skip.argtypes = [C.POINTER(_Level), C.c_int, C.c_int, _f64p, _f64p, C.c_void_p]
    lib.ora_cg_skip.restype = C.c_int
    lib.ora_cg_skip.argtypes = [C.POINTER(_Level), C.c_int, _f64p, _f64p, C.c_int, C.c_double, C.c_int,
                                C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double), _f64p,
                                C.c_void_p]
    lib.ora_permute_level.argtypes = [C.c_int, _i32p, _i32p, _i32p, _i32p, _f64p, _i32p,
                                      _i32p, _i32p, _f64p, _i32p]
    lib.ora_permute_f2c.argtypes = [C.c_int, _i32p, _i32p, _i32p, _i32p]
    lib.ora_mg_f32.restype = C.c_int
    lib.ora_mg_f32.argtypes = [C.POINTER(_Level32), C.c_int, C.c_int, _f32p, _f32p]
    lib.ora_mg_f32_skip.restype = C.c_int
    lib.ora_mg_f32_skip.argtypes = [C.POINTER(_Level32), C.c_int, C.c_int, _f32p, _f32p, _i32p]
    lib.ora_cg_mixed.restype = C.c_int
    lib.ora_cg_mixed.argtypes = [C.POINTER(_Level), C.POINTER(_Level32), C.c_int, _f64p, _f64p, C.c_int,
                                 C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double), _f64p]
    lib.ora_cg_mixed_skip.restype = C.c_int
    lib.ora_cg_mixed_skip.argtypes = [C.POINTER(_Level), C.POINTER(_Level32), C.c_int, _f64p, _f64p, C.c_int,
                                      C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), _f64p, C.c_void_p]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load_oracle()
    return _lib


@dataclass
class Level:
    """One grid level in the oracle's row-major 27-slot layout."""
    nx: int
    ny: int
    nz: int
    nnz: np.ndarray    # int32 [n]
    cols: np.ndarray   # int32 [n*27]
    vals: np.ndarray   # float64 [n*27]
    diag: np.ndarray   # int32 [n]
    f2c: np.ndarray | None = None  # int32 [n of next level]
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n(self) -> int:
        return int(self.nnz.shape[0])

    @property
    def total_nnz(self) -> int:
        return int(self.nnz.sum())

    def c(self) -> _Level:
        return _Level(self.nx, self.ny, self.nz, self.n, self.nnz.ctypes.data, self.cols.ctypes.data,
                      self.vals.ctypes.data, self.diag.ctypes.data,
                      self.f2c.ctypes.data if self.f2c is not None else None)

    def dense_rows(self):
        """(cols, vals) as [n, 27] views."""
        return self.cols.reshape(-1, SLOTS), self.vals.reshape(-1, SLOTS)


def _levels_c(levels):
    arr = (_Level * len(levels))()
    for i, L in enumerate(levels):
        arr[i] = L.c()
    return arr


@dataclass
class Problem:
    levels: list
    b: np.ndarray
    x: np.ndarray
    xexact: np.ndarray


def generate_level(nx, ny, nz, want_vectors=False):
    n = nx * ny * nz
    nnz = np.zeros(n, np.int32)
    cols = np.zeros(n * SLOTS, np.int32)
    vals = np.zeros(n * SLOTS, np.float64)
    diag = np.zeros(n, np.int32)
    if want_vectors:
        b, x, xe = np.zeros(n), np.zeros(n), np.zeros(n)
        lib().ora_generate(nx, ny, nz, nnz, cols, vals, diag, b.ctypes.data, x.ctypes.data, xe.ctypes.data)
        return Level(nx, ny, nz, nnz, cols, vals, diag), b, x, xe
    lib().ora_generate(nx, ny, nz, nnz, cols, vals, diag, None, None, None)
    return Level(nx, ny, nz, nnz, cols, vals, diag)


def generate(nx, ny=None, nz=None, nlevels=4) -> Problem:
    """GenerateProblem_ref + 3x GenerateCoarseProblem (main.cpp:137-144)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    L0, b, x, xe = generate_level(nx, ny, nz, want_vectors=True)
    levels = [L0]
    for _ in range(1, nlevels):
        f = levels[-1]
        f2c = np.zeros((f.nx // 2) * (f.ny // 2) * (f.nz // 2), np.int32)
        lib().ora_f2c(f.nx, f.ny, f.nz, f2c)
        f.f2c = f2c
        levels.append(generate_level(f.nx // 2, f.ny // 2, f.nz // 2))
    return Problem(levels, b, x, xe)


def spmv(L: Level, x):
    y = np.zeros(L.n)
    lib().ora_spmv(C.byref(L.c()), np.ascontiguousarray(x, np.float64), y)
    return y


def symgs(L: Level, r, x):
    x = np.array(x, np.float64, copy=True)
    lib().ora_symgs(C.byref(L.c()), np.ascontiguousarray(r, np.float64), x)
    return x


def gs_forward(L: Level, r, x):
    x = np.array(x, np.float64, copy=True)
    lib().ora_gs_forward(C.byref(L.c()), np.ascontiguousarray(r, np.float64), x)
    return x


def mg(levels, r, lev=0, skip=None):
    """ComputeMG_ref; skip[l] = trailing rows of level l whose backward GS update is
    left out (see ora_symgs_skip), None for the reference's V-cycle."""
    x = np.zeros(levels[lev].n)
    sk = None if skip is None else np.ascontiguousarray(skip, np.int32)
    err = lib().ora_mg_skip(_levels_c(levels), len(levels), lev, np.ascontiguousarray(r, np.float64), x,
                            sk.ctypes.data if sk is not None else None)
    assert err == 0
    return x


def symgs_skip(L: Level, r, x, skip):
    x = np.array(x, np.float64, copy=True)
    lib().ora_symgs_skip(C.byref(L.c()), np.ascontiguousarray(r, np.float64), x, int(skip))
    return x


def restriction(f2c, rf, Axf):
    rc = np.zeros(f2c.shape[0])
    lib().ora_restriction(f2c.shape[0], f2c, rf, Axf, rc)
    return rc


def prolongation(f2c, xc, xf):
    xf = np.array(xf, np.float64, copy=True)
    lib().ora_prolongation(f2c.shape[0], f2c, np.ascontiguousarray(xc, np.float64), xf)
    return xf


def dot(x, y):
    x = np.ascontiguousarray(x, np.float64)
    y = x if y is x else np.ascontiguousarray(y, np.float64)
    return lib().ora_dot(x.shape[0], x, y)


def waxpby(alpha, x, beta, y):
    w = np.zeros(x.shape[0])
    lib().ora_waxpby(x.shape[0], alpha, np.ascontiguousarray(x, np.float64), beta,
                     np.ascontiguousarray(y, np.float64), w)
    return w


def residual(v1, v2):
    return lib().ora_residual(v1.shape[0], np.ascontiguousarray(v1, np.float64),
                              np.ascontiguousarray(v2, np.float64))


def cg(levels, b, x0, max_iter, tolerance, do_prec=True, skip=None):
    """CG_ref (with the V-cycle of mg(skip=...)). Returns (x, niters, normr, normr0, hist[0..niters])."""
    x = np.array(x0, np.float64, copy=True)
    hist = np.zeros(max_iter + 1)
    ni, nr, nr0 = C.c_int(0), C.c_double(0), C.c_double(0)
    sk = None if skip is None else np.ascontiguousarray(skip, np.int32)
    err = lib().ora_cg_skip(_levels_c(levels), len(levels), np.ascontiguousarray(b, np.float64), x, max_iter,
                            tolerance, int(do_prec), C.byref(ni), C.byref(nr), C.byref(nr0), hist,
                            sk.ctypes.data if sk is not None else None)
    assert err == 0
    return x, ni.value, nr.value, nr0.value, hist[: ni.value + 1].copy()


def to_f32(levels):
    """FP32 copies of the level values for the mixed-precision form."""
    out = []
    for L in levels:
        out.append(dict(n=L.n, nnz=L.nnz, cols=L.cols, vals=L.vals.astype(np.float32), diag=L.diag, f2c=L.f2c))
    return out


def _levels32_c(l32):
    arr = (_Level32 * len(l32))()
    for i, L in enumerate(l32):
        arr[i] = _Level32(L["n"], L["nnz"].ctypes.data, L["cols"].ctypes.data, L["vals"].ctypes.data,
                          L["diag"].ctypes.data, L["f2c"].ctypes.data if L["f2c"] is not None else None)
    return arr


def mg_f32(l32, r, skip=None):
    """FP32 V-cycle (ComputeMG_ref.cpp:39-63 in float); skip: per-level rows not
    repeated at the turn of each symmetric sweep (None: the reference's sweep)."""
    x = np.zeros(l32[0]["n"], np.float32)
    if skip is None:
        err = lib().ora_mg_f32(_levels32_c(l32), len(l32), 0, np.ascontiguousarray(r, np.float32), x)
    else:
        sk = np.ascontiguousarray(skip, np.int32)
        err = lib().ora_mg_f32_skip(_levels32_c(l32), len(l32), 0, np.ascontiguousarray(r, np.float32), x, sk)
    assert err == 0
    return x


def cg_mixed(levels, b, x0, max_iter, tolerance, skip=None):
    """FP64 flexible PCG around the FP32 V-cycle (mg_f32 with `skip`). Returns
    (x, niters, normr, normr0, hist[0..niters])."""
    l32 = to_f32(levels)
    x = np.array(x0, np.float64, copy=True)
    hist = np.zeros(max_iter + 1)
    ni, nr, nr0 = C.c_int(0), C.c_double(0), C.c_double(0)
    sk = None if skip is None else np.ascontiguousarray(skip, np.int32)
    err = lib().ora_cg_mixed_skip(_levels_c(levels), _levels32_c(l32), len(levels),
                                  np.ascontiguousarray(b, np.float64), x, max_iter, tolerance,
                                  C.byref(ni), C.byref(nr), C.byref(nr0), hist,
                                  sk.ctypes.data if sk is not None else None)
    assert err == 0
    return x, ni.value, nr.value, nr0.value, hist[: ni.value + 1].copy()


# ---------------------------------------------------------------------------
# orderings
# ---------------------------------------------------------------------------

def parity_colour(nx, ny, nz):
    """Colour of every natural row: (ix&1) | (iy&1)<<1 | (iz&1)<<2."""
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return ((ix & 1) | ((iy & 1) << 1) | ((iz & 1) << 2)).reshape(-1).astype(np.int32)


def colour_new2old(nx, ny, nz, sweep):
    """Rows grouped by colour in the order `sweep` (a permutation of 0..7 giving the
    parity colour swept first, second, ...); inside one colour, natural order."""
    col = parity_colour(nx, ny, nz)
    rank = np.empty(8, np.int64)
    rank[np.asarray(sweep)] = np.arange(8)
    key = rank[col] * (nx * ny * nz) + np.arange(nx * ny * nz)
    return np.argsort(key, kind="stable").astype(np.int32)


def permute(levels, new2old_per_level):
    """The same hierarchy renumbered: new row q of level l = old row new2old[l][q]."""
    out = []
    o2n = []
    for n2o in new2old_per_level:
        inv = np.empty_like(n2o)
        inv[n2o] = np.arange(n2o.shape[0], dtype=np.int32)
        o2n.append(inv)
    for l, L in enumerate(levels):
        n = L.n
        pn = np.zeros(n, np.int32); pc = np.zeros(n * SLOTS, np.int32)
        pv = np.zeros(n * SLOTS); pd = np.zeros(n, np.int32)
        lib().ora_permute_level(n, new2old_per_level[l], o2n[l], L.nnz, L.cols, L.vals, L.diag, pn, pc, pv, pd)
        P = Level(L.nx, L.ny, L.nz, pn, pc, pv, pd)
        if L.f2c is not None:
            pf = np.zeros(L.f2c.shape[0], np.int32)
            lib().ora_permute_f2c(L.f2c.shape[0], L.f2c, new2old_per_level[l + 1], o2n[l], pf)
            P.f2c = pf
        out.append(P)
    return out


# ---------------------------------------------------------------------------
# the reference itself (present where oracle/_ref was built)
# ---------------------------------------------------------------------------

REF_LIB = os.path.join(HERE, "_ref", "libhpcg_ref.so")


def have_reference() -> bool:
    return os.path.exists(REF_LIB)


class Reference:
    """The HPCG 3.1 reference routines over a problem set up as main.cpp does."""

    _lib = None

    @classmethod
    def _load(cls):
        if cls._lib is None:
            l = C.CDLL(REF_LIB)
            l.ref_create.restype = C.c_void_p
            l.ref_create.argtypes = [C.c_int, C.c_int, C.c_int]
            l.ref_destroy.argtypes = [C.c_void_p]
            l.ref_level_rows.restype = C.c_int
            l.ref_level_rows.argtypes = [C.c_void_p, C.c_int]
            l.ref_level_nnz.restype = C.c_longlong
            l.ref_level_nnz.argtypes = [C.c_void_p, C.c_int]
            l.ref_export_level.argtypes = [C.c_void_p, C.c_int, _i32p, _i32p, _f64p, _i32p, C.c_void_p]
            l.ref_get_vectors.argtypes = [C.c_void_p, _f64p, _f64p, _f64p]
            l.ref_set_b.argtypes = [C.c_void_p, _f64p]
            l.ref_set_values.argtypes = [C.c_void_p, C.c_int, _f64p]
            for f in (l.ref_spmv, l.ref_symgs, l.ref_mg):
                f.restype = C.c_int
                f.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p]
            l.ref_dot.restype = C.c_double
            l.ref_dot.argtypes = [C.c_int, _f64p, _f64p]
            l.ref_waxpby.argtypes = [C.c_int, C.c_double, _f64p, C.c_double, _f64p, _f64p]
            l.ref_residual.restype = C.c_double
            l.ref_residual.argtypes = [C.c_int, _f64p, _f64p]
            l.ref_cg.restype = C.c_int
            l.ref_cg.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]
            l.ref_permute.argtypes = [C.c_void_p, C.POINTER(C.POINTER(C.c_int))]
            l.ref_test_cg.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4
            l.ref_test_symmetry.argtypes = [C.c_void_p, C.c_uint, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double), C.POINTER(C.c_int)]
            cls._lib = l
        return cls._lib

    def __init__(self, nx, ny=None, nz=None):
        self.l = self._load()
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.h = self.l.ref_create(nx, ny, nz)
        self.dims = (nx, ny, nz)

    def close(self):
        if self.h:
            self.l.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rows(self, lev=0):
        return self.l.ref_level_rows(self.h, lev)

    def export_level(self, lev):
        n = self.rows(lev)
        nnz = np.zeros(n, np.int32); cols = np.zeros(n * SLOTS, np.int32)
        vals = np.zeros(n * SLOTS); diag = np.zeros(n, np.int32)
        nc = self.rows(lev + 1) if lev < 3 else 0
        f2c = np.zeros(max(nc, 1), np.int32)
        self.l.ref_export_level(self.h, lev, nnz, cols, vals, diag, f2c.ctypes.data if nc else None)
        d = (self.dims[0] >> lev, self.dims[1] >> lev, self.dims[2] >> lev)
        return Level(*d, nnz, cols, vals, diag, f2c[:nc].copy() if nc else None)

    def levels(self):
        return [self.export_level(l) for l in range(4)]

    def vectors(self):
        n = self.rows(0)
        b, x, xe = np.zeros(n), np.zeros(n), np.zeros(n)
        self.l.ref_get_vectors(self.h, b, x, xe)
        return b, x, xe

    def set_b(self, b):
        self.l.ref_set_b(self.h, np.ascontiguousarray(b, np.float64))

    def set_values(self, lev, vals):
        self.l.ref_set_values(self.h, lev, np.ascontiguousarray(vals, np.float64))

    def spmv(self, x, lev=0):
        y = np.zeros(self.rows(lev))
        assert self.l.ref_spmv(self.h, lev, np.ascontiguousarray(x, np.float64), y) == 0
        return y

    def symgs(self, r, x, lev=0):
        x = np.array(x, np.float64, copy=True)
        assert self.l.ref_symgs(self.h, lev, np.ascontiguousarray(r, np.float64), x) == 0
        return x

    def mg(self, r, lev=0):
        x = np.zeros(self.rows(lev))
        assert self.l.ref_mg(self.h, lev, np.ascontiguousarray(r, np.float64), x) == 0
        return x

    def dot(self, x, y):
        return self.l.ref_dot(x.shape[0], np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64))

    def waxpby(self, alpha, x, beta, y):
        w = np.zeros(x.shape[0])
        self.l.ref_waxpby(x.shape[0], alpha, np.ascontiguousarray(x, np.float64), beta,
                          np.ascontiguousarray(y, np.float64), w)
        return w

    def residual(self, v1, v2):
        return self.l.ref_residual(v1.shape[0], np.ascontiguousarray(v1, np.float64),
                                   np.ascontiguousarray(v2, np.float64))

    def cg(self, max_iter, tol, do_prec=True, x0=None):
        x = np.zeros(self.rows(0)) if x0 is None else np.array(x0, np.float64, copy=True)
        ni, nr, nr0 = C.c_int(0), C.c_double(0), C.c_double(0)
        assert self.l.ref_cg(self.h, x, max_iter, tol, int(do_prec), C.byref(ni), C.byref(nr), C.byref(nr0)) == 0
        return x, ni.value, nr.value, nr0.value

    def permute(self, new2old_per_level):
        keep = [np.ascontiguousarray(a, np.int32) for a in new2old_per_level]
        arr = (C.POINTER(C.c_int) * len(keep))(*[a.ctypes.data_as(C.POINTER(C.c_int)) for a in keep])
        self.l.ref_permute(self.h, arr)

    def test_cg(self):
        v = [C.c_int(0) for _ in range(4)]
        self.l.ref_test_cg(self.h, *[C.byref(t) for t in v])
        return dict(count_pass=v[0].value, count_fail=v[1].value, niters_no_prec=v[2].value,
                    niters_prec=v[3].value)

    def test_symmetry(self, seed=1):
        a, b, c = C.c_double(0), C.c_double(0), C.c_int(0)
        self.l.ref_test_symmetry(self.h, seed, C.byref(a), C.byref(b), C.byref(c))
        return dict(depsym_spmv=a.value, depsym_mg=b.value, count_fail=c.value)


REF_MPI_LIB = os.path.join(HERE, "_ref", "libhpcg_ref_mpi.so")


def have_reference_ranks() -> bool:
    return os.path.exists(REF_MPI_LIB)


class ReferenceRanks:
    """The reference run as npx*npy*npz MPI ranks (its MPI branch, compiled
    against the thread-based MPI stand-in in mpi_shim/): every call runs the
    reference routine on all ranks at once. Vectors are lists with one array per
    rank, in the rank's local row order."""

    _lib = None

    @classmethod
    def _load(cls):
        if cls._lib is None:
            l = C.CDLL(REF_MPI_LIB)
            vp, i = C.c_void_p, C.c_int
            pp = C.POINTER(C.POINTER(C.c_double))
            l.refmpi_create.restype = vp
            l.refmpi_create.argtypes = [i] * 6
            l.refmpi_destroy.argtypes = [vp]
            l.refmpi_level_sizes.argtypes = [vp, i, i, _i32p]
            l.refmpi_export_level.argtypes = [vp, i, i] + [vp] * 10
            l.refmpi_get_b.argtypes = [vp, i, _f64p]
            l.refmpi_set_b.argtypes = [vp, i, _f64p]
            for f in (l.refmpi_spmv, l.refmpi_symgs, l.refmpi_mg):
                f.restype = i
                f.argtypes = [vp, i, pp, pp]
            l.refmpi_dot.restype = C.c_double
            l.refmpi_dot.argtypes = [vp, pp, pp]
            l.refmpi_cg.restype = i
            l.refmpi_cg.argtypes = [vp, pp, i, C.c_double, i, C.POINTER(i), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]
            l.refmpi_permute.argtypes = [vp, i, C.POINTER(C.POINTER(C.c_int))]
            l.refmpi_optimal_shape.argtypes = [i, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
            cls._lib = l
        return cls._lib

    @classmethod
    def optimal_shape(cls, size):
        """ComputeOptimalShapeXYZ(size) of the reference."""
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        cls._load().refmpi_optimal_shape(size, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def __init__(self, npx, npy, npz, nx, ny=None, nz=None):
        self.l = self._load()
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.grid = (npx, npy, npz)
        self.dims = (nx, ny, nz)
        self.nranks = npx * npy * npz
        self.h = self.l.refmpi_create(npx, npy, npz, nx, ny, nz)

    def close(self):
        if self.h:
            self.l.refmpi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sizes(self, rank, lev=0):
        """(nrow, ncol, neighbours, entries sent) of one rank's level."""
        s = np.zeros(4, np.int32)
        self.l.refmpi_level_sizes(self.h, rank, lev, s)
        return tuple(int(v) for v in s)

    def export(self, rank, lev=0):
        n, ncol, nnb, nsend = self.sizes(rank, lev)
        nc = self.sizes(rank, lev + 1)[0] if lev < 3 else 0
        out = dict(nnz=np.zeros(n, np.int32), cols=np.zeros(n * SLOTS, np.int32), vals=np.zeros(n * SLOTS),
                   f2c=np.zeros(max(nc, 1), np.int32), neighbors=np.zeros(max(nnb, 1), np.int32),
                   recv_len=np.zeros(max(nnb, 1), np.int32), send_len=np.zeros(max(nnb, 1), np.int32),
                   send_rows=np.zeros(max(nsend, 1), np.int32), ext_global=np.zeros(max(ncol - n, 1), np.int64),
                   l2g=np.zeros(n, np.int64))
        keys = ("nnz", "cols", "vals", "f2c", "neighbors", "recv_len", "send_len", "send_rows", "ext_global", "l2g")
        self.l.refmpi_export_level(self.h, rank, lev, *[out[k].ctypes.data for k in keys])
        out["f2c"] = out["f2c"][:nc] if nc else None
        for k, m in (("neighbors", nnb), ("recv_len", nnb), ("send_len", nnb), ("send_rows", nsend),
                     ("ext_global", ncol - n)):
            out[k] = out[k][:m]
        out.update(n=n, ncol=ncol)
        return out

    def get_b(self, rank):
        b = np.zeros(self.sizes(rank)[0])
        self.l.refmpi_get_b(self.h, rank, b)
        return b

    def set_b(self, rank, b):
        self.l.refmpi_set_b(self.h, rank, np.ascontiguousarray(b, np.float64))

    def _cols(self, vecs, lev):
        """Per-rank copies with ncol entries (externals zero), and their pointer array."""
        full = []
        for r, v in enumerate(vecs):
            n, ncol = self.sizes(r, lev)[:2]
            f = np.zeros(ncol)
            f[:n] = v[:n]
            full.append(f)
        return full, self._ptrs(full)

    @staticmethod
    def _ptrs(arrs):
        return (C.POINTER(C.c_double) * len(arrs))(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])

    def spmv(self, xs, lev=0):
        xf, xp = self._cols(xs, lev)
        ys = [np.zeros(self.sizes(r, lev)[0]) for r in range(self.nranks)]
        assert self.l.refmpi_spmv(self.h, lev, xp, self._ptrs(ys)) == 0
        return ys

    def symgs(self, rs, xs, lev=0):
        rs = [np.ascontiguousarray(r, np.float64) for r in rs]
        xf, xp = self._cols(xs, lev)
        assert self.l.refmpi_symgs(self.h, lev, self._ptrs(rs), xp) == 0
        return [x[: self.sizes(r, lev)[0]].copy() for r, x in enumerate(xf)]

    def mg(self, rs, lev=0):
        rs = [np.ascontiguousarray(r, np.float64) for r in rs]
        xf, xp = self._cols([np.zeros(self.sizes(r, lev)[0]) for r in range(self.nranks)], lev)
        assert self.l.refmpi_mg(self.h, lev, self._ptrs(rs), xp) == 0
        return [x[: self.sizes(r, lev)[0]].copy() for r, x in enumerate(xf)]

    def dot(self, xs, ys):
        xs = [np.ascontiguousarray(v, np.float64) for v in xs]
        ys = [np.ascontiguousarray(v, np.float64) for v in ys]
        return self.l.refmpi_dot(self.h, self._ptrs(xs), self._ptrs(ys))

    def cg(self, max_iter, tol, do_prec=True):
        xf, xp = self._cols([np.zeros(self.sizes(r)[0]) for r in range(self.nranks)], 0)
        ni, nr, nr0 = C.c_int(0), C.c_double(0), C.c_double(0)
        assert self.l.refmpi_cg(self.h, xp, max_iter, tol, int(do_prec), C.byref(ni), C.byref(nr),
                                C.byref(nr0)) == 0
        return [x[: self.sizes(r)[0]].copy() for r, x in enumerate(xf)], ni.value, nr.value, nr0.value

    def permute(self, rank, new2old_per_level):
        keep = [np.ascontiguousarray(a, np.int32) for a in new2old_per_level]
        arr = (C.POINTER(C.c_int) * len(keep))(*[a.ctypes.data_as(C.POINTER(C.c_int)) for a in keep])
        self.l.refmpi_permute(self.h, rank, arr)
