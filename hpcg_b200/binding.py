"""Python binding of the hpcg_b200 C ABI (include/hpcg_b200.h).

The entry points keep the reference's names and argument meaning
(src/ComputeSPMV.hpp:20, ComputeSYMGS.hpp:20, ComputeMG.hpp:20, CG.hpp:22-24,
ComputeDotProduct.hpp:18-19, ComputeWAXPBY.hpp:18-19, ComputeResidual.hpp:18,
OptimizeProblem.hpp:22-28). Where the reference returns a non-zero int, these
raise ``HpcgError`` carrying that status.

Vectors are float64 and contiguous: numpy arrays (host) or torch tensors (host
or CUDA), in the reference's natural row order. The library is loaded from this
package directory; there is no fallback if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhpcg_b200.so")

OK = 0
ERR_CUDA = 1
ERR_ARG = 2
ERR_UNSUPPORTED = 3
ERR_NOMEM = 4
ERR_HANDLE = 5
ERR_TIMEOUT = 6
SYMGS_COLOUR = 0
SYMGS_NATURAL = 1

EXPORTS = (
    "hpcg_b200_optimize", "hpcg_b200_generate", "hpcg_b200_get_rhs", "hpcg_b200_free",
    "hpcg_b200_memory_use", "hpcg_b200_set_diagonal", "hpcg_b200_set_values", "hpcg_b200_set_symgs_mode",
    "hpcg_b200_spmv", "hpcg_b200_symgs", "hpcg_b200_mg", "hpcg_b200_dot", "hpcg_b200_waxpby",
    "hpcg_b200_residual", "hpcg_b200_cg", "hpcg_b200_cg_mixed", "hpcg_b200_level_info",
    "hpcg_b200_export_level", "hpcg_b200_colour_permutation", "hpcg_b200_stream", "hpcg_b200_profile",
    "hpcg_b200_profile_read", "hpcg_b200_dot_noalloc", "hpcg_b200_adjoint", "hpcg_b200_cg_multi", "hpcg_b200_mg_multi",
    "hpcg_b200_level_config", "hpcg_b200_batch_create", "hpcg_b200_batch_problem", "hpcg_b200_batch_cg_mixed", "hpcg_b200_batch_free",
    "hpcg_b200_batch_form", "hpcg_b200_grid_wait_selftest", "hpcg_b200_level_first_config",
    "hpcg_b200_set_host_reuse", "hpcg_b200_level_wavefront", "hpcg_b200_wave_wait_selftest",
    "hpcg_b200_stream_probe",
    "hpcg_b200_process_grid", "hpcg_b200_generate_rank", "hpcg_b200_halo_plan", "hpcg_b200_rank_info",
    "hpcg_b200_comm_unique_id", "hpcg_b200_comm_nccl", "hpcg_b200_comm_local", "hpcg_b200_comm_free",
    "hpcg_b200_shard_spmv", "hpcg_b200_shard_symgs", "hpcg_b200_shard_mg", "hpcg_b200_shard_dot", "hpcg_b200_shard_cg",
    "hpcg_b200_mg_f32", "hpcg_b200_wait_selftest", "hpcg_b200_level_packed", "hpcg_b200_last_error",
)


class HpcgError(RuntimeError):
    def __init__(self, what, status, detail=""):
        super().__init__(f"{what} failed with status {status}" + (f": {detail}" if detail else ""))
        self.status = status


class LevelDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nrow", C.c_int), ("ncol", C.c_int),
        ("nonzeros_in_row", C.c_void_p), ("mtx_ind_l", C.c_void_p), ("matrix_values", C.c_void_p),
        ("f2c", C.c_void_p),
    ]


_lib = None


def lib():
    """The loaded libhpcg_b200.so (raises if the extension was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C hpcg_b200` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        l = C.CDLL(LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        l.hpcg_b200_optimize.argtypes = [C.POINTER(LevelDesc), i, i, C.POINTER(vp)]
        l.hpcg_b200_generate.argtypes = [i, i, i, i, i, C.POINTER(vp)]
        l.hpcg_b200_get_rhs.argtypes = [vp, vp]
        l.hpcg_b200_free.argtypes = [vp]
        l.hpcg_b200_memory_use.argtypes = [vp]
        l.hpcg_b200_memory_use.restype = d
        l.hpcg_b200_set_diagonal.argtypes = [vp, vp]
        l.hpcg_b200_set_values.argtypes = [vp, i, vp]
        l.hpcg_b200_set_symgs_mode.argtypes = [vp, i]
        l.hpcg_b200_spmv.argtypes = [vp, vp, vp]
        l.hpcg_b200_symgs.argtypes = [vp, vp, vp]
        l.hpcg_b200_mg.argtypes = [vp, vp, vp]
        l.hpcg_b200_dot.argtypes = [i, vp, vp, C.POINTER(d)]
        l.hpcg_b200_waxpby.argtypes = [i, d, vp, d, vp, vp]
        l.hpcg_b200_residual.argtypes = [i, vp, vp, C.POINTER(d)]
        l.hpcg_b200_cg.argtypes = [vp, vp, vp, i, d, i, C.POINTER(i), C.POINTER(d), C.POINTER(d), vp]
        l.hpcg_b200_cg_mixed.argtypes = [vp, vp, vp, i, d, C.POINTER(i), C.POINTER(d), C.POINTER(d)]
        l.hpcg_b200_level_info.argtypes = [vp, i, C.POINTER(i), C.POINTER(C.c_int64), vp]
        l.hpcg_b200_level_packed.argtypes = [vp, i, C.POINTER(C.c_int64)]
        l.hpcg_b200_export_level.argtypes = [vp, i, vp, vp, vp, vp]
        l.hpcg_b200_colour_permutation.argtypes = [i, i, i, vp, vp]
        l.hpcg_b200_stream.argtypes = [i]
        l.hpcg_b200_stream.restype = vp
        l.hpcg_b200_profile.argtypes = [i, i]
        l.hpcg_b200_profile_read.argtypes = [i, i, C.POINTER(d), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        l.hpcg_b200_dot_noalloc.argtypes = [i, vp, vp, vp, vp]
        l.hpcg_b200_adjoint.argtypes = [vp, vp, vp, i, d, vp, vp, C.POINTER(i)]
        l.hpcg_b200_cg_multi.argtypes = [vp, i, vp, vp, i, d, vp, vp, vp]
        l.hpcg_b200_mg_multi.argtypes = [vp, i, vp, vp]
        l.hpcg_b200_level_config.argtypes = [vp, i, vp]
        l.hpcg_b200_batch_create.argtypes = [i, vp, vp, vp, i, C.POINTER(vp)]
        l.hpcg_b200_batch_problem.argtypes = [vp, i, C.POINTER(vp)]
        l.hpcg_b200_batch_cg_mixed.argtypes = [vp, vp, vp, i, d, vp, vp, vp]
        l.hpcg_b200_batch_free.argtypes = [vp]
        l.hpcg_b200_batch_form.argtypes = [vp, C.POINTER(i)]
        l.hpcg_b200_grid_wait_selftest.argtypes = [i, d]
        l.hpcg_b200_level_first_config.argtypes = [vp, i, vp, vp]
        l.hpcg_b200_set_host_reuse.argtypes = [vp, i]
        l.hpcg_b200_level_wavefront.argtypes = [vp, i, C.POINTER(i)]
        l.hpcg_b200_wave_wait_selftest.argtypes = [vp, d]
        l.hpcg_b200_stream_probe.argtypes = [vp, i, C.POINTER(C.c_float), C.POINTER(d)]
        l.hpcg_b200_process_grid.argtypes = [i, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        l.hpcg_b200_generate_rank.argtypes = [i, i, i, i, i, i, i, i, i, C.POINTER(vp)]
        l.hpcg_b200_halo_plan.argtypes = [i, i, i, i, i, i, i, C.POINTER(i), vp, vp, vp, vp]
        l.hpcg_b200_rank_info.argtypes = [vp, i, vp]
        l.hpcg_b200_comm_unique_id.argtypes = [vp]
        l.hpcg_b200_comm_nccl.argtypes = [vp, i, i, vp, C.POINTER(vp)]
        l.hpcg_b200_comm_local.argtypes = [i, vp, C.POINTER(vp)]
        l.hpcg_b200_comm_free.argtypes = [vp]
        for f in (l.hpcg_b200_shard_spmv, l.hpcg_b200_shard_symgs, l.hpcg_b200_shard_mg):
            f.argtypes = [vp, vp, vp]
        l.hpcg_b200_shard_dot.argtypes = [vp, vp, vp, C.POINTER(d)]
        l.hpcg_b200_shard_cg.argtypes = [vp, vp, vp, i, d, i, C.POINTER(i), C.POINTER(d), C.POINTER(d), vp]
        l.hpcg_b200_mg_f32.argtypes = [vp, vp, vp]
        l.hpcg_b200_wait_selftest.argtypes = [i, d]
        l.hpcg_b200_last_error.restype = C.c_char_p
        for name in EXPORTS:
            f = getattr(l, name)
            if name not in ("hpcg_b200_memory_use", "hpcg_b200_last_error", "hpcg_b200_stream"):
                f.restype = C.c_int
        _lib = l
    return _lib


def last_error() -> str:
    return lib().hpcg_b200_last_error().decode()


def _check(status, what):
    if status != OK:
        raise HpcgError(what, status, last_error())


def _ptr(v, n=None):
    """Data pointer of a float64 contiguous numpy array or torch tensor."""
    if v is None:
        return None
    if isinstance(v, np.ndarray):
        if v.dtype != np.float64 or not v.flags.c_contiguous:
            raise TypeError("vectors must be contiguous float64")
        if n is not None and v.size < n:
            raise ValueError(f"vector of length {v.size} shorter than {n}")
        return v.ctypes.data
    if hasattr(v, "data_ptr"):
        import torch
        if v.dtype != torch.float64 or not v.is_contiguous():
            raise TypeError("vectors must be contiguous float64")
        if n is not None and v.numel() < n:
            raise ValueError(f"vector of length {v.numel()} shorter than {n}")
        return v.data_ptr()
    raise TypeError(f"unsupported vector type {type(v)}")


def _rowptrs(base_addr, n, row_bytes):
    return (np.uint64(base_addr) + np.arange(n, dtype=np.uint64) * np.uint64(row_bytes)).astype(np.uint64)


class Problem:
    """A device-resident HPCG hierarchy: the object OptimizeProblem hangs on
    A.optimizationData (src/OptimizeProblem.cpp:37)."""

    def __init__(self, handle, dims, nlevels):
        self._h = C.c_void_p(handle)
        self.dims = dims
        self.nlevels = nlevels

    # ---- construction ---------------------------------------------------
    @classmethod
    def optimize(cls, levels, device=0):
        """OptimizeProblem from the reference's per-level arrays. Each level is a
        mapping with nx, ny, nz, nnz [n], cols [n*27] (int32, entry j of row i at
        i*27+j), vals [n*27] float64 and f2c [n_coarse] int32 (None on the last)."""
        keep = []
        descs = (LevelDesc * len(levels))()
        for i, L in enumerate(levels):
            n = int(L["nx"] * L["ny"] * L["nz"])
            nnz8 = np.ascontiguousarray(L["nnz"], dtype=np.int8)
            cols = np.ascontiguousarray(L["cols"], dtype=np.int32)
            vals = np.ascontiguousarray(L["vals"], dtype=np.float64)
            cp = _rowptrs(cols.ctypes.data, n, 27 * 4)
            vp = _rowptrs(vals.ctypes.data, n, 27 * 8)
            f2c = L.get("f2c")
            f2c = None if f2c is None else np.ascontiguousarray(f2c, dtype=np.int32)
            keep += [nnz8, cols, vals, cp, vp, f2c]
            descs[i] = LevelDesc(L["nx"], L["ny"], L["nz"], n, n, nnz8.ctypes.data, cp.ctypes.data, vp.ctypes.data,
                                 f2c.ctypes.data if f2c is not None else None)
        h = C.c_void_p()
        _check(lib().hpcg_b200_optimize(descs, len(levels), device, C.byref(h)), "hpcg_b200_optimize")
        return cls(h.value, (levels[0]["nx"], levels[0]["ny"], levels[0]["nz"]), len(levels))

    @classmethod
    def generate(cls, nx, ny=None, nz=None, nlevels=4, device=0):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        h = C.c_void_p()
        _check(lib().hpcg_b200_generate(nx, ny, nz, nlevels, device, C.byref(h)), "hpcg_b200_generate")
        return cls(h.value, (nx, ny, nz), nlevels)

    @classmethod
    def generate_rank(cls, nx, ny, nz, npx, npy, npz, rank, nlevels=4, device=0):
        """Rank `rank`'s local nx*ny*nz block of an npx*npy*npz run, with its halo
        plan (the reference's GenerateProblem + SetupHalo on that rank)."""
        h = C.c_void_p()
        _check(lib().hpcg_b200_generate_rank(nx, ny, nz, npx, npy, npz, rank, nlevels, device, C.byref(h)),
               "hpcg_b200_generate_rank")
        return cls(h.value, (nx, ny, nz), nlevels)

    def rank_info(self, level=0):
        out = np.zeros(10, np.int32)
        _check(lib().hpcg_b200_rank_info(self._h, level, out.ctypes.data), "hpcg_b200_rank_info")
        keys = ("rank", "nranks", "npx", "npy", "npz", "ipx", "ipy", "ipz", "neighbors", "externals")
        return dict(zip(keys, (int(v) for v in out)))

    def free(self):
        if getattr(self, "_owned_by_batch", False):
            return
        if self._h and self._h.value:
            _check(lib().hpcg_b200_free(self._h), "hpcg_b200_free")
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def nrow(self):
        return self.dims[0] * self.dims[1] * self.dims[2]

    # ---- configuration ----------------------------------------------------
    def memory_use(self) -> float:
        return lib().hpcg_b200_memory_use(self._h)

    def set_symgs_mode(self, mode):
        _check(lib().hpcg_b200_set_symgs_mode(self._h, mode), "hpcg_b200_set_symgs_mode")

    def set_diagonal(self, diag):
        _check(lib().hpcg_b200_set_diagonal(self._h, _ptr(diag, self.nrow)), "hpcg_b200_set_diagonal")

    def set_values(self, level, values27):
        _check(lib().hpcg_b200_set_values(self._h, level, _ptr(values27)), "hpcg_b200_set_values")

    def get_rhs(self, out=None):
        out = np.zeros(self.nrow) if out is None else out
        _check(lib().hpcg_b200_get_rhs(self._h, _ptr(out, self.nrow)), "hpcg_b200_get_rhs")
        return out

    # ---- the reference's entry points -------------------------------------
    def ComputeSPMV(self, x, y):
        _check(lib().hpcg_b200_spmv(self._h, _ptr(x, self.nrow), _ptr(y, self.nrow)), "ComputeSPMV")
        return 0

    def ComputeSYMGS(self, r, x):
        _check(lib().hpcg_b200_symgs(self._h, _ptr(r, self.nrow), _ptr(x, self.nrow)), "ComputeSYMGS")
        return 0

    def ComputeMG(self, r, x):
        _check(lib().hpcg_b200_mg(self._h, _ptr(r, self.nrow), _ptr(x, self.nrow)), "ComputeMG")
        return 0

    def CG(self, b, x, max_iter, tolerance, do_preconditioning=True, times=None):
        """Returns (niters, normr, normr0); x is updated in place."""
        ni, nr, nr0 = C.c_int(0), C.c_double(0), C.c_double(0)
        t = None
        if times is not None:
            t = np.ascontiguousarray(times, dtype=np.float64)
        _check(lib().hpcg_b200_cg(self._h, _ptr(b, self.nrow), _ptr(x, self.nrow), max_iter, tolerance,
                                  int(bool(do_preconditioning)), C.byref(ni), C.byref(nr), C.byref(nr0),
                                  t.ctypes.data if t is not None else None), "CG")
        if times is not None:
            times[:] = t
        return ni.value, nr.value, nr0.value

    def CG_mixed(self, b, x, max_iter, tolerance):
        ni, nr, nr0 = C.c_int(0), C.c_double(0), C.c_double(0)
        _check(lib().hpcg_b200_cg_mixed(self._h, _ptr(b, self.nrow), _ptr(x, self.nrow), max_iter, tolerance,
                                        C.byref(ni), C.byref(nr), C.byref(nr0)), "CG_mixed")
        return ni.value, nr.value, nr0.value

    def ComputeMG_f32(self, r, x):
        """x = widen(MG32(narrow(r))): the FP32 V-cycle of CG_mixed alone."""
        _check(lib().hpcg_b200_mg_f32(self._h, _ptr(r, self.nrow), _ptr(x, self.nrow)), "hpcg_b200_mg_f32")
        return 0

    def CG_multi(self, b, x, max_iter, tolerance):
        """nrhs = len(b) / nrow systems (b, x: [nrhs, nrow] contiguous float64).
        Returns (niters, normr, normr0) as numpy arrays, x updated in place."""
        nrhs = (b.size if isinstance(b, np.ndarray) else b.numel()) // self.nrow
        ni = np.zeros(nrhs, np.int32)
        nr = np.zeros(nrhs)
        nr0 = np.zeros(nrhs)
        _check(lib().hpcg_b200_cg_multi(self._h, nrhs, _ptr(b, nrhs * self.nrow), _ptr(x, nrhs * self.nrow),
                                        max_iter, tolerance, ni.ctypes.data, nr.ctypes.data, nr0.ctypes.data),
               "hpcg_b200_cg_multi")
        return ni, nr, nr0

    def ComputeMG_multi(self, r, x):
        nrhs = (r.size if isinstance(r, np.ndarray) else r.numel()) // self.nrow
        _check(lib().hpcg_b200_mg_multi(self._h, nrhs, _ptr(r, nrhs * self.nrow), _ptr(x, nrhs * self.nrow)),
               "hpcg_b200_mg_multi")
        return 0

    def adjoint(self, x, g, max_iter, tolerance, grad_b, grad_values27):
        """Implicit adjoint of the solve: grad_b = lambda (A lambda = g), grad_values27
        = -lambda_i x_j per slot. Returns the adjoint solve's iteration count."""
        ni = C.c_int(0)
        _check(lib().hpcg_b200_adjoint(self._h, _ptr(x, self.nrow), _ptr(g, self.nrow), max_iter, tolerance,
                                       _ptr(grad_b, self.nrow), _ptr(grad_values27, 27 * self.nrow), C.byref(ni)),
               "hpcg_b200_adjoint")
        return ni.value

    # ---- inspection ------------------------------------------------------------
    def level_info(self, level):
        n, pitch = C.c_int(0), C.c_int64(0)
        starts = np.zeros(9, np.int32)
        _check(lib().hpcg_b200_level_info(self._h, level, C.byref(n), C.byref(pitch), starts.ctypes.data),
               "hpcg_b200_level_info")
        return n.value, pitch.value, starts

    def level_pack_width(self, level):
        """Form of the level's packed columns: 1 or 2 (offset bytes), 3 (the
        diagonal form); 0 if it keeps only its 32-bit columns."""
        b = self.level_packed(level)
        if b == 0:
            return 0
        _, pitch, _ = self.level_info(level)
        per_tile = b // (pitch // 128)
        return {28 * 4 + 27 * 128: 1, 28 * 4 + 27 * 256: 2, 28 * 4 + 27 * 16: 3}[per_tile]

    def level_packed(self, level):
        """Bytes of the level's packed column index (0: 32-bit columns only)."""
        b = C.c_int64(0)
        _check(lib().hpcg_b200_level_packed(self._h, level, C.byref(b)), "hpcg_b200_level_packed")
        return b.value

    def level_config(self, level):
        """Autotuner choices of a level: dict(gs, gs_first, gs32, spmv, spmv_order, tuned, gs32_first)."""
        out = np.zeros(7, np.int32)
        _check(lib().hpcg_b200_level_config(self._h, level, out.ctypes.data), "hpcg_b200_level_config")
        keys = ("gs", "gs_first", "gs32", "spmv", "spmv_order", "tuned", "gs32_first")
        return dict(zip(keys, (int(v) for v in out)))

    def set_host_reuse(self, enable):
        """hpcg_b200_set_host_reuse: whether CG may skip sending an unchanged
        host b and a zero host x."""
        _check(lib().hpcg_b200_set_host_reuse(self._h, int(bool(enable))), "hpcg_b200_set_host_reuse")

    def level_first_config(self, level):
        """The first sweep's configuration at each of the 8 sweep positions:
        (fp64 list, fp32 list)."""
        a = np.zeros(8, np.int32)
        b = np.zeros(8, np.int32)
        _check(lib().hpcg_b200_level_first_config(self._h, level, a.ctypes.data, b.ctypes.data),
               "hpcg_b200_level_first_config")
        return [int(v) for v in a], [int(v) for v in b]

    def level_wavefront(self, level):
        """hpcg_b200_level_wavefront: 1 if the level's sweeps from nonzero x run
        as one wavefront launch each, else 0."""
        on = C.c_int(0)
        _check(lib().hpcg_b200_level_wavefront(self._h, level, C.byref(on)), "hpcg_b200_level_wavefront")
        return int(on.value)

    def wave_wait_selftest(self, limit_seconds):
        """hpcg_b200_wave_wait_selftest: the status code (not raised)."""
        return int(lib().hpcg_b200_wave_wait_selftest(self._h, float(limit_seconds)))

    def stream_probe(self, level=0):
        """hpcg_b200_stream_probe: (milliseconds, bytes) of one launch of the
        FP64 phases' copy pipeline over the level's whole matrix with consumers
        that hand each stage straight back."""
        ms, nb = C.c_float(0.0), C.c_double(0.0)
        _check(lib().hpcg_b200_stream_probe(self._h, level, C.byref(ms), C.byref(nb)), "hpcg_b200_stream_probe")
        return float(ms.value), float(nb.value)

    def level_config_string(self):
        """HPCG_B200_LEVEL_CONFIG that repeats this problem's tuned choices (the
        first sweeps per sweep position, and the wavefront-sweep choice)."""
        parts = []
        for lv in range(self.nlevels):
            c = self.level_config(lv)
            f64, f32 = self.level_first_config(lv)
            parts.append(",".join([str(c["gs"]), "/".join(map(str, f64)), str(c["spmv"]), str(c["spmv_order"]),
                                   str(c["gs32"]), "/".join(map(str, f32)), str(self.level_wavefront(lv))]))
        return ";".join(parts)

    def export_level(self, level):
        n, pitch, starts = self.level_info(level)
        n2o = np.zeros(n, np.int32)
        cols = np.zeros(27 * pitch, np.int32)
        vals = np.zeros(27 * pitch, np.float64)
        nc = self.level_info(level + 1)[0] if level + 1 < self.nlevels else 0
        f2c = np.zeros(max(nc, 1), np.int32)
        _check(lib().hpcg_b200_export_level(self._h, level, n2o.ctypes.data, cols.ctypes.data, vals.ctypes.data,
                                            f2c.ctypes.data if nc else None), "hpcg_b200_export_level")
        return dict(n=n, pitch=pitch, starts=starts, new2old=n2o, cols=cols.reshape(27, pitch),
                    vals=vals.reshape(27, pitch), f2c=f2c[:nc] if nc else None)


def process_grid(nranks):
    """The reference's default (npx, npy, npz) for nranks (ComputeOptimalShapeXYZ.cpp)."""
    a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
    _check(lib().hpcg_b200_process_grid(nranks, C.byref(a), C.byref(b), C.byref(c)), "hpcg_b200_process_grid")
    return a.value, b.value, c.value


def halo_plan(nx, ny, nz, npx, npy, npz, rank):
    """Host-computed halo plan of one rank's level: dict(neighbors, counts,
    send_rows (local natural), ext_global), as SetupHalo_ref.cpp stores it."""
    nnb = C.c_int(0)
    _check(lib().hpcg_b200_halo_plan(nx, ny, nz, npx, npy, npz, rank, C.byref(nnb), None, None, None, None),
           "hpcg_b200_halo_plan")
    nbr = np.zeros(26, np.int32)
    cnt = np.zeros(26, np.int32)
    _check(lib().hpcg_b200_halo_plan(nx, ny, nz, npx, npy, npz, rank, C.byref(nnb), nbr.ctypes.data,
                                     cnt.ctypes.data, None, None), "hpcg_b200_halo_plan")
    total = int(cnt[: nnb.value].sum())
    send = np.zeros(max(total, 1), np.int32)
    ext = np.zeros(max(total, 1), np.int64)
    _check(lib().hpcg_b200_halo_plan(nx, ny, nz, npx, npy, npz, rank, C.byref(nnb), None, None, send.ctypes.data,
                                     ext.ctypes.data), "hpcg_b200_halo_plan")
    k = nnb.value
    return dict(neighbors=nbr[:k].copy(), counts=cnt[:k].copy(), send_rows=send[:total].copy(),
                ext_global=ext[:total].copy())


def comm_unique_id() -> bytes:
    """128-byte NCCL id for hpcg_b200_comm_nccl (make it on one rank, broadcast it)."""
    buf = (C.c_ubyte * 128)()
    _check(lib().hpcg_b200_comm_unique_id(buf), "hpcg_b200_comm_unique_id")
    return bytes(buf)


class Comm:
    """The ranks of a run this process drives: one rank over NCCL
    (Comm.nccl), or every rank on one GPU (Comm.local). The routines take one
    vector per driven rank, in the rank's local natural order."""

    def __init__(self, handle, problems):
        self._h = C.c_void_p(handle)
        self.problems = list(problems)

    @classmethod
    def local(cls, problems):
        arr = (C.c_void_p * len(problems))(*[p.handle.value for p in problems])
        h = C.c_void_p()
        _check(lib().hpcg_b200_comm_local(len(problems), arr, C.byref(h)), "hpcg_b200_comm_local")
        return cls(h.value, problems)

    @classmethod
    def nccl(cls, unique_id: bytes, nranks, rank, problem):
        buf = (C.c_ubyte * 128).from_buffer_copy(unique_id)
        h = C.c_void_p()
        _check(lib().hpcg_b200_comm_nccl(buf, nranks, rank, problem.handle, C.byref(h)), "hpcg_b200_comm_nccl")
        return cls(h.value, [problem])

    def free(self):
        if self._h and self._h.value:
            _check(lib().hpcg_b200_comm_free(self._h), "hpcg_b200_comm_free")
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def _vecs(self, vs):
        if len(vs) != len(self.problems):
            raise ValueError(f"{len(self.problems)} vectors expected, got {len(vs)}")
        return (C.c_void_p * len(vs))(*[_ptr(v, p.nrow) for v, p in zip(vs, self.problems)])

    def ComputeSPMV(self, xs, ys):
        _check(lib().hpcg_b200_shard_spmv(self._h, self._vecs(xs), self._vecs(ys)), "hpcg_b200_shard_spmv")
        return 0

    def ComputeSYMGS(self, rs, xs):
        _check(lib().hpcg_b200_shard_symgs(self._h, self._vecs(rs), self._vecs(xs)), "hpcg_b200_shard_symgs")
        return 0

    def ComputeMG(self, rs, xs):
        _check(lib().hpcg_b200_shard_mg(self._h, self._vecs(rs), self._vecs(xs)), "hpcg_b200_shard_mg")
        return 0

    def ComputeDotProduct(self, xs, ys):
        r = C.c_double(0)
        _check(lib().hpcg_b200_shard_dot(self._h, self._vecs(xs), self._vecs(ys), C.byref(r)), "hpcg_b200_shard_dot")
        return r.value

    def CG(self, bs, xs, max_iter, tolerance, do_preconditioning=True, times=None):
        ni, nr, nr0 = C.c_int(0), C.c_double(0), C.c_double(0)
        t = None if times is None else np.ascontiguousarray(times, dtype=np.float64)
        _check(lib().hpcg_b200_shard_cg(self._h, self._vecs(bs), self._vecs(xs), max_iter, tolerance,
                                        int(bool(do_preconditioning)), C.byref(ni), C.byref(nr), C.byref(nr0),
                                        t.ctypes.data if t is not None else None), "hpcg_b200_shard_cg")
        if times is not None:
            times[:] = t
        return ni.value, nr.value, nr0.value


def colour_permutation(nx, ny, nz):
    """(new2old, colour_start) of the library's colour order (host computation)."""
    n2o = np.zeros(nx * ny * nz, np.int32)
    starts = np.zeros(9, np.int32)
    _check(lib().hpcg_b200_colour_permutation(nx, ny, nz, n2o.ctypes.data, starts.ctypes.data),
           "hpcg_b200_colour_permutation")
    return n2o, starts


class Batch:
    """Independent problems of different sizes solved together
    (hpcg_b200_batch_*). Member problems are views owned by the batch."""

    def __init__(self, dims, device=0):
        m = len(dims)
        nx = np.array([d[0] for d in dims], np.int32)
        ny = np.array([d[1] for d in dims], np.int32)
        nz = np.array([d[2] for d in dims], np.int32)
        h = C.c_void_p()
        _check(lib().hpcg_b200_batch_create(m, nx.ctypes.data, ny.ctypes.data, nz.ctypes.data, device, C.byref(h)),
               "hpcg_b200_batch_create")
        self._h = h
        self.dims = [tuple(int(v) for v in d) for d in dims]
        self.problems = []
        for i, d in enumerate(self.dims):
            ph = C.c_void_p()
            _check(lib().hpcg_b200_batch_problem(self._h, i, C.byref(ph)), "hpcg_b200_batch_problem")
            p = Problem.__new__(Problem)
            p._h, p.dims, p.nlevels = ph, d, 4
            p._owned_by_batch = True
            self.problems.append(p)

    def CG_mixed(self, bs, xs, max_iter, tolerance):
        m = len(self.dims)
        bp = (C.c_void_p * m)(*[_ptr(v) for v in bs])
        xp = (C.c_void_p * m)(*[_ptr(v) for v in xs])
        ni = np.zeros(m, np.int32)
        nr = np.zeros(m)
        nr0 = np.zeros(m)
        _check(lib().hpcg_b200_batch_cg_mixed(self._h, bp, xp, max_iter, tolerance, ni.ctypes.data,
                                              nr.ctypes.data, nr0.ctypes.data), "hpcg_b200_batch_cg_mixed")
        return ni, nr, nr0

    def form(self):
        """0: one launch per step (register phases), 1: the same with bulk-copy
        phases, 2: the whole iteration in one cooperative launch."""
        f = C.c_int(-1)
        _check(lib().hpcg_b200_batch_form(self._h, C.byref(f)), "hpcg_b200_batch_form")
        return f.value

    def free(self):
        if self._h and self._h.value:
            for p in self.problems:
                p._h = C.c_void_p()  # owned by the batch
            _check(lib().hpcg_b200_batch_free(self._h), "hpcg_b200_batch_free")
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


PROF_GS_FULL, PROF_GS_FIRST, PROF_SPMV, PROF_RESTRICT, PROF_GS32_FULL, PROF_GS32_FIRST, PROF_GS_SWEEP = range(7)


def stream(device=0):
    """The library's cudaStream_t for `device` (an integer handle)."""
    return lib().hpcg_b200_stream(device)


def profile(enable, device=0):
    _check(lib().hpcg_b200_profile(device, int(bool(enable))), "hpcg_b200_profile")


def profile_read(kind, device=0):
    """(total_ms, launches, rows) of one timed kernel class."""
    ms, ln, rows = C.c_double(0), C.c_int64(0), C.c_int64(0)
    _check(lib().hpcg_b200_profile_read(device, kind, C.byref(ms), C.byref(ln), C.byref(rows)),
           "hpcg_b200_profile_read")
    return ms.value, ln.value, rows.value


def wait_selftest(seconds, device=0):
    """Status of hpcg_b200_wait_selftest: a device-side wait on a barrier that
    nothing completes, given up after `seconds` (ERR_TIMEOUT expected)."""
    return lib().hpcg_b200_wait_selftest(device, float(seconds))


def grid_wait_selftest(seconds, device=0):
    """Status of hpcg_b200_grid_wait_selftest: every block of a cooperative
    launch waits at a grid barrier for one arrival too many, and gives up after
    `seconds` (ERR_TIMEOUT expected)."""
    return lib().hpcg_b200_grid_wait_selftest(device, float(seconds))


def ComputeDotProduct(n, x, y):
    """ComputeDotProduct_ref.cpp:46-80 semantics; returns the scalar."""
    out = C.c_double(0)
    _check(lib().hpcg_b200_dot(n, _ptr(x, n), _ptr(y, n), C.byref(out)), "ComputeDotProduct")
    return out.value


def ComputeWAXPBY(n, alpha, x, beta, y, w):
    _check(lib().hpcg_b200_waxpby(n, alpha, _ptr(x, n), beta, _ptr(y, n), _ptr(w, n)), "ComputeWAXPBY")
    return 0


def ComputeResidual(n, v1, v2):
    out = C.c_double(0)
    _check(lib().hpcg_b200_residual(n, _ptr(v1, n), _ptr(v2, n), C.byref(out)), "ComputeResidual")
    return out.value
