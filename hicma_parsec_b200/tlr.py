"""Python binding of the C ABI (``include/hicma_tlr.h``) through ctypes.

The classes mirror the reference's operator surface for the factorization
path: ``STARSH_gen`` (hicma_parsec/hicma_parsec.h:187-198), ``HiCMA_dpotrf_L``
(hicma_parsec.h:38-56), ``parsec_band_size_auto_tuning`` (hicma_parsec.h:111-115),
``parsec_band_regenerate`` (hicma_parsec.h:94-100), ``parsec_rank_gather``
(hicma_parsec.h:124-127), ``HICMA_get_stat2`` (hicma_internal.c:52-71) and
``STARSH_check`` (hicma_parsec.h:162-169), plus the log-determinant / solve /
log-likelihood additions.  Every call goes to the CUDA library; there is no
CPU fallback: if the library is missing this module raises on import of the
library.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libhicma_tlr.so")
# HICMA_TLR_LIB=checked selects the bounds-checked build (every batched launch
# validated on the host first); a path selects that file.
LIB_PATH_CHECKED = os.path.join(HERE, "lib", "libhicma_tlr_checked.so")

LOWER = 122
UPPER = 121
KIND_RANDTLR, KIND_ED_SIN_2D, KIND_SQEXP_2D, KIND_SQEXP_3D, KIND_EXP_3D, KIND_ED_SIN_3D = 0, 1, 2, 3, 4, 5
KIND_MD_VIRUS, KIND_MD_CUBE = 6, 7
KIND_NDIM = {1: 2, 2: 2, 3: 3, 4: 3, 5: 3, 6: 3, 7: 3}     # point kinds; randtlr has no points
(RBF_GAUSSIAN, RBF_EXPON, RBF_INVQUAD, RBF_INVMQUAD, RBF_MATERNC1, RBF_MATERNC2, RBF_TPS, RBF_CTPS,
 RBF_WENDLAND) = range(9)
PREC_FP64, PREC_MIXED = 0, 1
ERR_ARG, ERR_CUDA, ERR_OOM, ERR_RANK_OVERFLOW, ERR_TIMEOUT, ERR_STATE, ERR_NOT_SUPPORTED = -1, -2, -3, -4, -5, -6, -7

_lib = None


class TLRError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with code {code}: {msg}")
        self.code = code


class CProblem(C.Structure):
    _fields_ = [("kind", C.c_int), ("beta", C.c_double), ("nu", C.c_double), ("noise", C.c_double),
                ("sigma", C.c_double), ("seed", C.c_ulonglong), ("wave_k", C.c_double),
                ("add_diag", C.c_double), ("rbf_kernel", C.c_int), ("radius", C.c_double),
                ("numobj", C.c_int), ("order", C.c_int), ("density", C.c_double)]


@dataclass
class Problem:
    """STARS-H problem (``starsh_ssdata_generate`` / ``starsh_eddata_generate``
    arguments, hicma_parsec/testing_dpotrf.c:300-365; defaults of the reference).
    ``wave_k`` applies to the electrodynamics kinds 1 and 5, ``add_diag`` to them
    and to randtlr (kind 0); ``add_diag <= 0`` means N
    (hicma_parsec/hicma_parsec.c:289-291).  The mesh kinds 6 (md-3d-virus) and 7
    (md-3d-cube) evaluate the radial basis function ``rbf_kernel`` of
    ``r / radius`` plus ``add_diag`` on the diagonal (testing_dpotrf.c:366-381);
    ``numobj`` and ``density`` place kind 6's mesh copies, ``order`` 1 Morton
    orders the points of both."""
    kind: int = KIND_SQEXP_2D
    beta: float = 0.1
    nu: float = 0.5
    noise: float = 0.1
    sigma: float = 1.0
    seed: int = 0
    wave_k: float = 50.0
    add_diag: float = 0.0
    rbf_kernel: int = RBF_GAUSSIAN
    radius: float = 0.0
    numobj: int = 1
    order: int = 1
    density: float = -1.0

    @property
    def ndim(self) -> int:
        return KIND_NDIM[self.kind]

    def c(self) -> CProblem:
        return CProblem(self.kind, self.beta, self.nu, self.noise, self.sigma, self.seed, self.wave_k,
                        self.add_diag, self.rbf_kernel, self.radius, self.numobj, self.order, self.density)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def load_library(path: str | None = None):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    env = os.environ.get("HICMA_TLR_LIB", "")
    path = path or (LIB_PATH_CHECKED if env == "checked" else (env or LIB_PATH))
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library not built: {path} (run python -m hicma_parsec_b200.build)")
    lib = C.CDLL(path)
    vp, i, d, ip, dp, ul = C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_ulong)
    sig = {
        "hicma_tlr_init": (i, [i, C.c_size_t, C.POINTER(vp)]),
        "hicma_tlr_fini": (i, [vp]),
        "hicma_tlr_stream": (vp, [vp]),
        "hicma_tlr_last_error": (C.c_char_p, []),
        "hicma_tlr_desc_create": (i, [vp, i, i, i, i, C.POINTER(vp)]),
        "hicma_tlr_desc_destroy": (i, [vp]),
        "hicma_tlr_desc_info": (i, [vp, ip, ip, ip, ip, ip]),
        "hicma_tlr_desc_copy": (i, [vp, vp, vp]),
        "hicma_tlr_points": (i, [C.POINTER(CProblem), i, vp]),
        "hicma_tlr_points_mesh": (i, [C.POINTER(CProblem), C.c_char_p, i, vp]),
        "hicma_tlr_generate": (i, [vp, i, vp, vp, C.POINTER(CProblem), vp, d, i, i, i, ip]),
        "hicma_tlr_rank_gather": (i, [vp, vp, vp, i]),
        "hicma_tlr_rank_stat": (i, [vp, i, i, ip, ip, dp]),
        "hicma_tlr_band_autotune": (i, [vp, i, i, i]),
        "hicma_tlr_band_regenerate": (i, [vp, i, vp, C.POINTER(CProblem), i]),
        "hicma_tlr_dpotrf_L": (i, [vp, i, vp, vp, d, i, i, ip, i, i, i, i, ip, vp, vp, vp, i]),
        "hicma_tlr_dpotrf_L_rank": (i, [vp, i, vp, vp, vp, d, i, i, ip, i, i, i, i, ip, vp, vp, vp, i]),
        "hicma_tlr_set_precision": (i, [vp, i]),
        "hicma_tlr_dpotrf_L_start": (i, [vp, vp, d, i, i]),
        "hicma_tlr_dpotrf_L_wait": (i, [vp, vp, vp]),
        "hicma_tlr_uncompress": (i, [vp, vp, vp, C.c_long]),
        "hicma_tlr_tile_get": (i, [vp, vp, i, i, vp, ip]),
        "hicma_tlr_tile_set": (i, [vp, vp, i, i, vp, i]),
        "hicma_tlr_store_bytes": (i, [vp, vp, C.POINTER(C.c_size_t)]),
        "hicma_tlr_store_get": (i, [vp, vp, vp, vp]),
        "hicma_tlr_store_set": (i, [vp, vp, vp, vp]),
        "hicma_tlr_store_stream": (i, [vp, vp, vp, C.c_size_t]),
        "hicma_tlr_logdet": (i, [vp, vp, dp]),
        "hicma_tlr_solve": (i, [vp, vp, i, vp, C.c_long]),
        "hicma_tlr_loglik": (i, [vp, vp, vp, dp, dp, vp]),
        "hicma_tlr_rank_history": (i, [vp, vp, vp, vp, vp]),
        "hicma_tlr_k_wait_probe": (i, [C.c_longlong, C.c_longlong, i, dp, vp]),
        "hicma_tlr_bounds_checked": (i, []),
        "hicma_tlr_op_counts": (C.c_ulong, [C.c_char, C.c_ulong, C.c_ulong, C.c_ulong, C.c_ulong]),
        "hicma_tlr_autotune": (i, [vp, i, i, i, vp, vp]),
        "hicma_tlr_tuning_get": (i, [vp, vp]),
        "hicma_tlr_tuning_set": (i, [vp, vp]),
        "hicma_tlr_bounds_register": (i, [vp, C.c_size_t]),
        "hicma_tlr_bounds_unregister": (i, [vp]),
        "hicma_tlr_bounds_inside": (i, [vp, C.c_size_t]),
        "hicma_tlr_serve_loglik": (i, [vp, C.POINTER(CProblem), i, i, d, i, i, vp, dp, dp, vp, ip]),
        "hicma_tlr_last_stats": (i, [vp, vp, i]),
        "hicma_tlr_check": (i, [vp, vp, C.POINTER(CProblem), vp, dp, dp]),
        "hicma_tlr_check_probe": (i, [vp, vp, C.POINTER(CProblem), i, C.c_ulonglong, dp]),
        "hicma_tlr_prof_enable": (i, [vp, i]),
        "hicma_tlr_prof_read": (i, [vp, vp, i]),
        "hicma_tlr_k_cov": (i, [C.POINTER(CProblem), vp, i, i, i, i, i, vp, i, vp]),
        "hicma_tlr_k_dgemm": (i, [i, i, i, i, i, d, vp, i, vp, i, d, vp, i, vp]),
        "hicma_tlr_k_potrf": (i, [vp, i, vp, i, vp, vp, i]),
        "hicma_tlr_k_lr_update": (i, [vp, i, vp, vp, i, vp, vp, i, vp, vp, ip, d, i, i]),
        "hicma_tlr_k_compress": (i, [vp, i, vp, vp, vp, i, d, ip]),
        "hicma_tlr_k_potrf_noalloc": (i, [i, vp, i, vp, vp, i, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load_library().hicma_tlr_last_error().decode()


def _check(code: int, where: str) -> int:
    if code < 0:
        raise TLRError(code, where, last_error())
    return code


def points(prob: Problem, n: int) -> np.ndarray:
    """Points [ndim][n] of the problem (host generator of the library)."""
    lib = load_library()
    if prob.kind not in KIND_NDIM:
        raise TLRError(ERR_ARG, "hicma_tlr_points", f"unsupported problem kind {prob.kind}")
    out = np.empty((prob.ndim, n), dtype=np.float64)
    cp = prob.c()
    _check(lib.hicma_tlr_points(C.byref(cp), n, _p(out)), "hicma_tlr_points")
    return out


def points_mesh(prob: Problem, mesh_file: str, n: int) -> np.ndarray:
    """Points [3][n] of the md-3d-virus problem: ``prob.numobj`` copies of the
    mesh read from ``mesh_file`` (x y z triples), placed by ``prob.density``
    and ordered by ``prob.order`` (``hicma_tlr_points_mesh``)."""
    lib = load_library()
    out = np.empty((3, n), dtype=np.float64)
    cp = prob.c()
    _check(lib.hicma_tlr_points_mesh(C.byref(cp), os.fsencode(mesh_file), n, _p(out)), "hicma_tlr_points_mesh")
    return out


class Context:
    """One GPU, one stream, one workspace (setup_parsec / cleanup_parsec)."""

    def __init__(self, device: int = 0, workspace_bytes: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib.hicma_tlr_init(device, workspace_bytes, C.byref(h)), "hicma_tlr_init")
        self.h = h
        self._mats = weakref.WeakSet()

    @property
    def stream(self) -> int:
        return self.lib.hicma_tlr_stream(self.h) or 0

    PROF_CLASSES = ("gemm", "qr", "qapply", "core_svd", "potrf", "cov", "copy", "other", "proj",
                    "gemm_y", "gemm_trsm", "gemm_syrk", "gemm_dense", "gemm_gen", "gram", "rcholqr")

    def prof_enable(self, on: bool = True) -> None:
        _check(self.lib.hicma_tlr_prof_enable(self.h, int(on)), "hicma_tlr_prof_enable")

    def prof_read(self) -> dict:
        nc = len(self.PROF_CLASSES)
        out = np.zeros(4 * nc)
        _check(self.lib.hicma_tlr_prof_read(self.h, _p(out), nc), "hicma_tlr_prof_read")
        o = out.reshape(nc, 4)
        return {name: {"launches": int(o[k, 0]), "seconds": float(o[k, 1]), "flops": float(o[k, 2]),
                       "bytes": float(o[k, 3])} for k, name in enumerate(self.PROF_CLASSES)}

    def set_precision(self, prec: int) -> None:
        _check(self.lib.hicma_tlr_set_precision(self.h, prec), "hicma_tlr_set_precision")

    def autotune(self, nb: int, maxrank: int, reps: int = 3) -> dict:
        """hicma_tlr_autotune: measure the kernel choices for tile size nb and keep
        the fastest; returns the table and the measured medians (ms)."""
        t = np.zeros(2, dtype=np.int32)
        ms = np.full(11, np.nan)
        _check(self.lib.hicma_tlr_autotune(self.h, nb, maxrank, reps, _p(t), _p(ms)), "hicma_tlr_autotune")
        widths = (48, 64, 96, 128)
        return {"gemm_narrow_n": int(t[0]), "potrf_grid": int(t[1]),
                "potrf_ms": [float(v) for v in ms[:3]],
                "gemm_ms": {w: {"128x32": float(ms[3 + 2 * i]), "64x64": float(ms[4 + 2 * i])}
                            for i, w in enumerate(widths)}}

    def tuning(self) -> tuple:
        t = np.zeros(2, dtype=np.int32)
        _check(self.lib.hicma_tlr_tuning_get(self.h, _p(t)), "hicma_tlr_tuning_get")
        return int(t[0]), int(t[1])

    def set_tuning(self, gemm_narrow_n: int, potrf_grid: int) -> None:
        t = np.array([gemm_narrow_n, potrf_grid], dtype=np.int32)
        _check(self.lib.hicma_tlr_tuning_set(self.h, _p(t)), "hicma_tlr_tuning_set")

    def close(self) -> None:
        if self.h:
            for m in list(self._mats):
                m.close()
            self.lib.hicma_tlr_fini(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TLRMatrix:
    """Device tile store: dense band + packed [U, V] off-band tiles + rank map
    (dcA / dcAr of hicma_parsec/testing_dpotrf.c:418-453)."""

    def __init__(self, ctx: Context, n: int, nb: int, maxrank: int, band_size: int = 1):
        self.ctx, self.lib = ctx, ctx.lib
        h = C.c_void_p()
        _check(self.lib.hicma_tlr_desc_create(ctx.h, n, nb, maxrank, band_size, C.byref(h)), "hicma_tlr_desc_create")
        self.h = h
        ctx._mats.add(self)
        self.n, self.nb, self.maxrank = n, nb, maxrank
        self.nt = n // nb

    @property
    def band_size(self) -> int:
        b = C.c_int()
        _check(self.lib.hicma_tlr_desc_info(self.h, None, None, None, None, C.byref(b)), "hicma_tlr_desc_info")
        return b.value

    def close(self):
        if self.h:
            self.lib.hicma_tlr_desc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- generation -----------------------------------------------------
    def generate(self, prob: Problem, tol: float, maxrank: int | None = None, pts: np.ndarray | None = None) -> int:
        """STARSH_gen; returns info (0, or -1 when a tile is rejected)."""
        info = C.c_int(0)
        cp = prob.c()
        if pts is not None:
            pts = np.ascontiguousarray(pts, dtype=np.float64)
        Ar = np.empty(self.nt * self.nt, dtype=np.int32)
        _check(self.lib.hicma_tlr_generate(self.ctx.h, LOWER, self.h, _p(Ar), C.byref(cp), _p(pts), tol,
                                           maxrank or self.maxrank, self.band_size, 0, C.byref(info)),
               "hicma_tlr_generate")
        self.gen_ranks = Ar    # rank map of the generation; rejected tiles are -1
        return info.value

    def rejected_tiles(self) -> list:
        """Off-band tiles the last generation rejected (rank rule), as (m, n)."""
        G = getattr(self, "gen_ranks", None)
        if G is None:
            return []
        b = self.band_size
        return [(m, n) for m in range(b, self.nt) for n in range(0, m - b + 1) if G[n * self.nt + m] < 0]

    def potrf_start(self, acc: float, maxrank: int | None = None, fixed_rank: int = 0) -> None:
        """HiCMA_dpotrf_L_2flow_New: enqueue the factorization on a background
        thread and return; potrf_wait() completes it."""
        _check(self.lib.hicma_tlr_dpotrf_L_start(self.ctx.h, self.h, acc, fixed_rank, maxrank or self.maxrank),
               "hicma_tlr_dpotrf_L_start")

    def potrf_wait(self) -> int:
        """Wait for potrf_start; returns info (errors raise)."""
        return _check(self.lib.hicma_tlr_dpotrf_L_wait(self.ctx.h, self.h, None), "hicma_tlr_dpotrf_L_wait")

    def rank_history(self) -> dict:
        """Rank history of the last factorization: NT x NT arrays [m, n]
        'initial', 'minimum', 'maximum', 'final' (-1 off the low-rank part)."""
        nt = self.nt
        out = {k: np.empty(nt * nt, dtype=np.int32) for k in ("initial", "minimum", "maximum", "final")}
        _check(self.lib.hicma_tlr_rank_history(self.h, _p(out["initial"]), _p(out["minimum"]), _p(out["maximum"]),
                                                _p(out["final"])), "hicma_tlr_rank_history")
        return {k: v.reshape(nt, nt).T.copy() for k, v in out.items()}

    def rank_map(self) -> np.ndarray:
        G = np.empty(self.nt * self.nt, dtype=np.int32)
        _check(self.lib.hicma_tlr_rank_gather(self.ctx.h, self.h, _p(G), self.band_size), "hicma_tlr_rank_gather")
        return G

    def band_regenerate(self, prob: Problem, band_size: int) -> None:
        cp = prob.c()
        _check(self.lib.hicma_tlr_band_regenerate(self.ctx.h, LOWER, self.h, C.byref(cp), band_size),
               "hicma_tlr_band_regenerate")

    # --- factorization --------------------------------------------------
    def potrf(self, acc: float, maxrank: int | None = None, fixed_rank: int = 0, lookahead: int = -1,
              want_counters: bool = False, verbose: int = 0):
        """HiCMA_dpotrf_L; returns info (and op counters when asked)."""
        la = C.c_int(lookahead)
        two = C.c_int(0)
        tiles = np.zeros(self.nt * self.nt, dtype=np.uint64) if want_counters else None
        ops = np.zeros(1, dtype=np.uint64) if want_counters else None
        cpt = np.zeros(6, dtype=np.float64)
        mr = maxrank or self.maxrank
        info = _check(self.lib.hicma_tlr_dpotrf_L(self.ctx.h, LOWER, self.h, None, acc, fixed_rank, mr,
                                                  C.byref(la), self.band_size, self.nb, mr, 0, C.byref(two),
                                                  _p(tiles), _p(ops), _p(cpt), verbose), "hicma_tlr_dpotrf_L")
        if want_counters:
            return info, tiles.reshape(self.nt, self.nt), int(ops[0]), cpt
        return info

    def stats(self) -> np.ndarray:
        s = np.zeros(16)
        _check(self.lib.hicma_tlr_last_stats(self.h, _p(s), 16), "hicma_tlr_last_stats")
        return s

    def copy_from(self, other: "TLRMatrix") -> None:
        _check(self.lib.hicma_tlr_desc_copy(self.ctx.h, other.h, self.h), "hicma_tlr_desc_copy")

    # --- results --------------------------------------------------------
    def uncompress(self) -> np.ndarray:
        D = np.empty((self.n, self.n), dtype=np.float64, order="F")
        _check(self.lib.hicma_tlr_uncompress(self.ctx.h, self.h, _p(D), self.n), "hicma_tlr_uncompress")
        return D

    def tile(self, m: int, n: int):
        r = C.c_int()
        _check(self.lib.hicma_tlr_tile_get(self.ctx.h, self.h, m, n, None, C.byref(r)), "hicma_tlr_tile_get")
        if r.value < 0:
            buf = np.empty((self.nb, self.nb), dtype=np.float64, order="F")
            _check(self.lib.hicma_tlr_tile_get(self.ctx.h, self.h, m, n, _p(buf), C.byref(r)), "hicma_tlr_tile_get")
            return buf
        buf = np.empty((self.nb, 2 * r.value), dtype=np.float64, order="F")
        _check(self.lib.hicma_tlr_tile_get(self.ctx.h, self.h, m, n, _p(buf), C.byref(r)), "hicma_tlr_tile_get")
        return buf[:, :r.value], buf[:, r.value:]

    def set_tile(self, m: int, n: int, data) -> None:
        if isinstance(data, tuple):
            U, V = data
            buf = np.asfortranarray(np.hstack([U, V]), dtype=np.float64)
            r = U.shape[1]
        else:
            buf = np.asfortranarray(data, dtype=np.float64)
            r = -1
        _check(self.lib.hicma_tlr_tile_set(self.ctx.h, self.h, m, n, _p(buf), r), "hicma_tlr_tile_set")

    def store_bytes(self) -> int:
        b = C.c_size_t()
        _check(self.lib.hicma_tlr_store_bytes(self.ctx.h, self.h, C.byref(b)), "hicma_tlr_store_bytes")
        return b.value

    def store_get(self, buf_ptr: int, ranks: np.ndarray | None = None) -> None:
        _check(self.lib.hicma_tlr_store_get(self.ctx.h, self.h, C.c_void_p(buf_ptr), _p(ranks)), "hicma_tlr_store_get")

    def store_set(self, buf_ptr: int, ranks: np.ndarray) -> None:
        _check(self.lib.hicma_tlr_store_set(self.ctx.h, self.h, C.c_void_p(buf_ptr), _p(ranks)), "hicma_tlr_store_set")

    def store_stream(self, buf_ptr: int | None, nbytes: int = 0) -> None:
        """Arm the copy-out of the next factorization into host memory at
        buf_ptr (column layout, hicma_tlr_store_stream); None disarms."""
        _check(self.lib.hicma_tlr_store_stream(self.ctx.h, self.h, C.c_void_p(buf_ptr or 0), nbytes),
               "hicma_tlr_store_stream")

    def check(self, prob: Problem, approx: "TLRMatrix | None" = None):
        """(||L L^T - A|| / ||A||, ||L - L0|| / ||L||) on the device."""
        r1, r2 = C.c_double(), C.c_double()
        cp = prob.c()
        _check(self.lib.hicma_tlr_check(self.ctx.h, self.h, C.byref(cp), approx.h if approx else None,
                                        C.byref(r1), C.byref(r2)), "hicma_tlr_check")
        return r1.value, r2.value

    def check_probe(self, prob: Problem, nprobe: int = 16, seed: int = 0) -> float:
        """||(A - L L^T) Z||_F / ||A Z||_F with nprobe Gaussian probes (any N)."""
        r = C.c_double()
        cp = prob.c()
        _check(self.lib.hicma_tlr_check_probe(self.ctx.h, self.h, C.byref(cp), nprobe, seed, C.byref(r)),
               "hicma_tlr_check_probe")
        return r.value

    def logdet(self) -> float:
        v = C.c_double()
        _check(self.lib.hicma_tlr_logdet(self.ctx.h, self.h, C.byref(v)), "hicma_tlr_logdet")
        return v.value

    def solve(self, b: np.ndarray) -> np.ndarray:
        X = np.asfortranarray(np.array(b, dtype=np.float64, copy=True).reshape(self.n, -1))
        _check(self.lib.hicma_tlr_solve(self.ctx.h, self.h, X.shape[1], _p(X), self.n), "hicma_tlr_solve")
        return X[:, 0] if np.ndim(b) == 1 else X

    def loglik(self, y: np.ndarray):
        y = np.ascontiguousarray(y, dtype=np.float64)
        ll, ld = C.c_double(), C.c_double()
        x = np.empty(self.n)
        _check(self.lib.hicma_tlr_loglik(self.ctx.h, self.h, _p(y), C.byref(ll), C.byref(ld), _p(x)), "hicma_tlr_loglik")
        return ll.value, ld.value, x


# ---------------------------------------------------------------------------
# Reference-named entry points (same argument meaning and error behaviour,
# except that argument errors raise instead of returning 0 silently).
# ---------------------------------------------------------------------------
def STARSH_gen(ctx: Context, uplo: int, A: TLRMatrix, prob: Problem, tol: float, maxrank: int,
               band_size: int, send_full_tile: int = 0) -> int:
    if uplo != LOWER:
        raise TLRError(ERR_NOT_SUPPORTED, "STARSH_gen", "only dplasmaLower")
    if band_size != A.band_size:
        raise TLRError(ERR_ARG, "STARSH_gen", "band_size differs from the descriptor")
    return A.generate(prob, tol, maxrank)


def HiCMA_dpotrf_L(ctx: Context, uplo: int, A: TLRMatrix, acc: float, fixed_rank: int, maxrank: int,
                   lookahead: int = -1, band_size: int | None = None, hmb: int = 300, compmaxrank: int = 0,
                   send_full_tile: int = 0, verbose: int = 0):
    """Returns (info, tileopcounters NT x NT, total opcount, critical_path_time[6])."""
    lib = ctx.lib
    la = C.c_int(lookahead)
    two = C.c_int(0)
    tiles = np.zeros(A.nt * A.nt, dtype=np.uint64)
    ops = np.zeros(1, dtype=np.uint64)
    cpt = np.zeros(6)
    info = _check(lib.hicma_tlr_dpotrf_L(ctx.h, uplo, A.h, None, acc, fixed_rank, maxrank, C.byref(la),
                                         A.band_size if band_size is None else band_size, hmb,
                                         compmaxrank or maxrank, send_full_tile, C.byref(two), _p(tiles), _p(ops),
                                         _p(cpt), verbose), "HiCMA_dpotrf_L")
    return info, tiles.reshape(A.nt, A.nt), int(ops[0]), cpt


def serve_loglik(ctx: Context, prob: Problem, n: int, nb: int, acc: float, y: np.ndarray, maxrank: int = 0,
                 autoband: bool = True):
    """One serving request in one library call (hicma_tlr_serve_loglik):
    returns (status, loglik, logdet, x, band); status is 0 or the positive
    factorization info; errors raise."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    if y.shape != (n,):
        raise TLRError(ERR_ARG, "hicma_tlr_serve_loglik", "y must have N entries")
    ll, ld, band = C.c_double(float("nan")), C.c_double(float("nan")), C.c_int(0)
    x = np.empty(n)
    cp = prob.c()
    st = _check(ctx.lib.hicma_tlr_serve_loglik(ctx.h, C.byref(cp), n, nb, acc, maxrank, int(autoband), _p(y),
                                               C.byref(ll), C.byref(ld), _p(x), C.byref(band)),
                "hicma_tlr_serve_loglik")
    return st, ll.value, ld.value, x, band.value


def parsec_band_size_auto_tuning(rank_array: np.ndarray, nt: int, nb: int, verbose: int = 0) -> int:
    G = np.ascontiguousarray(rank_array, dtype=np.int32)
    return _check(load_library().hicma_tlr_band_autotune(_p(G), nt, nb, verbose), "band_autotune")


def HICMA_get_stat2(rank_array: np.ndarray, nt: int, band_size: int):
    G = np.ascontiguousarray(rank_array, dtype=np.int32)
    mn, mx, av = C.c_int(), C.c_int(), C.c_double()
    _check(load_library().hicma_tlr_rank_stat(_p(G), nt, band_size, C.byref(mn), C.byref(mx), C.byref(av)),
           "HICMA_get_stat2")
    return mn.value, mx.value, av.value
