"""CPU oracle for the tile-low-rank (TLR) Cholesky path of HiCMA-PaRSEC.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library imports this module:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` use it, and only to compare results against (or as the timed CPU restatement).

PARITY UNPINNED.  The arithmetic of the reference lives in three git
submodules that are empty in the reference tree (``dplasma``, ``hcore``,
``stars-h``; ``.gitmodules:1-10``) and no commit of them is pinned.  The
reference ships no golden vectors or known-answer files either (its two CTest
entries, ``hicma_parsec/CMakeLists.txt:59-62``, only run ``--check`` against a
dense factorization at run time).  This module therefore restates:

* the task graph, case selection, rank-0 skips and association orders of
  ``hicma_parsec/HiCMA_dpotrf_L_2flow.jdf`` exactly;
* the generation graph of ``hicma_parsec/STARSH_gen.jdf`` (band tiles dense,
  off-band tiles compressed to a packed ``[U, V]`` pair plus a rank);
* the band auto-tuning rule of ``hicma_parsec/band_size_auto_tuning.jdf``;
* the flop model of ``hicma_parsec/op_counts.h`` (including its float32 casts;
  pinned bit for bit against that header compiled unchanged, the golden vectors
  in ``tests/golden/op_counts.json``);
* the checks of ``hicma_parsec/testing_dpotrf.c:111-230``;

and restates from their published mathematics the absent third-party pieces:

* STARS-H ``randtlr`` (``-D 0``, ``testing_dpotrf.c:315-321``): per tile row a
  random orthonormal basis Q_m, singular values S_k = 0.5**k, tiles
  Q_m diag(S) Q_n^T plus ``add_diag`` on the diagonal (see
  :func:`randtlr_basis`);
* STARS-H point placement (jittered grid + Morton order) and the squared
  exponential / exponential covariance kernels (call sites
  ``testing_dpotrf.c:336-358``) and the electrodynamics ``sin(k r) / r``
  kernels in 2D and 3D (call sites ``testing_dpotrf.c:325-334,359-365``);
* the mesh-deformation problems (``-D 6`` md-3d-virus, ``-D 7`` md-3d-cube,
  ``testing_dpotrf.c:366-381``): the nine radial basis functions of ``-B``
  (``hicma_parsec.c:80``, :func:`rbf_phi`) of r / radius plus ``add_diag`` on
  the diagonal; STARS-H's point generators for them are absent, so the node
  rules (:func:`cube_points`, :func:`virus_points`) are this restatement's own,
  shared with the library's host code;
* STARS-H ``starsh_dense_dlrrsdd`` rank rule: the smallest rank whose
  discarded singular values have Frobenius norm <= tol * (Frobenius norm of the
  sampled spectrum); a tile is rejected (rank -1, ``STARSH_gen.jdf:169-171``)
  when that rank is >= min(m, n)/2 or > maxrank;
* HCORE ``dgemm_qr_svd``/``dgemm_ormqr`` recompression: QR of the stacked
  ``[Cu, Au]`` and ``[Cv, -Y]``, SVD of ``R_U R_V^T`` and an absolute
  truncation sigma_i >= acc (or a fixed rank when ``fixed_rank > 0``), capped
  at the storage maxrank.

Conventions (shared with the CUDA path): a low-rank tile is A(m,n) = U V^T
with U (NB x r) having orthonormal columns and V (NB x r) carrying the
singular values.  Rank arrays are column-major NT x NT int arrays,
``G[n*NT + m]`` for tile (m, n) (``band_size_auto_tuning.jdf:48``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla

# Problem kinds (``-D``), numbering of ``testing_dpotrf.c:12``.
KIND_RANDTLR = 0
KIND_ED_SIN_2D = 1
KIND_SQEXP_2D = 2
KIND_SQEXP_3D = 3
KIND_EXP_3D = 4
KIND_ED_SIN_3D = 5
KIND_MD_VIRUS = 6
KIND_MD_CUBE = 7
KIND_NAMES = {KIND_RANDTLR: "randtlr", KIND_ED_SIN_2D: "ed-2d-sin", KIND_SQEXP_2D: "st-2d-sqexp", KIND_SQEXP_3D: "st-3d-sqexp",
              KIND_EXP_3D: "st-3d-exp", KIND_ED_SIN_3D: "ed-3d-sin", KIND_MD_VIRUS: "md-3d-virus",
              KIND_MD_CUBE: "md-3d-cube"}
KIND_NDIM = {KIND_ED_SIN_2D: 2, KIND_SQEXP_2D: 2, KIND_SQEXP_3D: 3, KIND_EXP_3D: 3, KIND_ED_SIN_3D: 3,
             KIND_MD_VIRUS: 3, KIND_MD_CUBE: 3}
# Radial basis functions of the mesh kinds (-B, hicma_parsec.c:80)
RBF_GAUSSIAN, RBF_EXPON, RBF_INVQUAD, RBF_INVMQUAD, RBF_MATERNC1, RBF_MATERNC2, RBF_TPS, RBF_CTPS, RBF_WENDLAND = range(9)
MESH_SEED_XOR = 0x4D45534856495255

RANDTLR_DECAY = 0.5               # testing_dpotrf.c:318
RANDTLR_KMAX = 64                 # singular directions kept: 0.5**64 is below FP64 resolution
RANDTLR_SEED_XOR = 0x52414E44544C5200
FLUCTUATION = 0.66666667          # hicma_parsec_internal.h:107
MORTON_BITS = 21

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


# --------------------------------------------------------------------------
# Points (STARS-H ``STARSH_PARTICLES_UNIFORM`` + Morton sort, restated)
# --------------------------------------------------------------------------
def _mix64(x):
    """splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = np.asarray(x, dtype=np.uint64) + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counters) -> np.ndarray:
    """Counter-based uniform doubles in [0, 1): 53 high bits of
    mix64(mix64(seed) + counter)."""
    base = _mix64(np.array([seed], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        z = _mix64(base + np.asarray(counters, dtype=np.uint64))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def grid_side(n: int, ndim: int) -> int:
    """Smallest s with s**ndim >= n."""
    s = max(1, int(round(n ** (1.0 / ndim))))
    while s ** ndim < n:
        s += 1
    while s > 1 and (s - 1) ** ndim >= n:
        s -= 1
    return s


def morton_codes(pts: np.ndarray) -> np.ndarray:
    ndim = pts.shape[1]
    q = np.floor(pts * float(1 << MORTON_BITS)).astype(np.int64)
    q = np.clip(q, 0, (1 << MORTON_BITS) - 1).astype(np.uint64)
    code = np.zeros(pts.shape[0], dtype=np.uint64)
    for b in range(MORTON_BITS):
        for a in range(ndim):
            code |= ((q[:, a] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * ndim + a)
    return code


def gen_points(n: int, ndim: int, seed: int = 0) -> np.ndarray:
    """n points in [0,1]^ndim: a side^ndim grid (side = ceil(n^(1/ndim))),
    each point jittered uniformly by +/-0.4 of the spacing, Morton-sorted
    (stable), first n kept.  Returns an (n, ndim) float64 array.

    Restates STARS-H's uniform particle placement called at
    ``testing_dpotrf.c:336-358`` (seeded by ``srand(0)``, ``:312``); the
    generator here is a documented counter-based one so that the CUDA host
    code reproduces it bit for bit.
    """
    side = grid_side(n, ndim)
    total = side ** ndim
    idx = np.arange(total, dtype=np.int64)
    pts = np.empty((total, ndim), dtype=np.float64)
    for a in range(ndim):
        c = (idx // (side ** a)) % side
        u = uniform01(seed, idx * ndim + a)
        pts[:, a] = ((c.astype(np.float64) + 0.1) + 0.8 * u) / float(side)
    order = np.argsort(morton_codes(pts), kind="stable")
    return np.ascontiguousarray(pts[order[:n]])


def _order_points(c: np.ndarray, order: int, n: int) -> np.ndarray:
    """First n rows of the (total, 3) point set c after a stable Morton sort
    (order 1; coordinates mapped to [0, 1) through the set's bounding box for
    the code only) or as given (order 0)."""
    if order == 1 and c.shape[0] > 0:
        lo, hi = c.min(axis=0), c.max(axis=0)
        w = hi - lo
        u = np.zeros_like(c)
        for a in range(3):
            if w[a] > 0.0:
                u[:, a] = (c[:, a] - lo[a]) / w[a] * (1.0 - 2.0 ** -30)
        c = c[np.argsort(morton_codes(u), kind="stable")]
    return np.ascontiguousarray(c[:n])


def cube_points(n: int, order: int = 1) -> np.ndarray:
    """md-3d-cube nodes (``testing_dpotrf.c:375-381``; STARS-H's
    ``starsh_generate_3d_rbf_mesh_coordinates_cube`` is absent from the
    reference tree, so this is the restatement's own rule): the cell centres
    ((i + 1/2)/s, (j + 1/2)/s, (k + 1/2)/s) of an s^3 grid on the unit cube,
    s = ceil(cbrt(n)), x fastest, Morton ordered when ``order == 1``; the
    first n.  Same arithmetic as the library's host generator."""
    s = grid_side(n, 3)
    i = np.arange(s ** 3, dtype=np.int64)
    g = np.stack([i % s, (i // s) % s, i // (s * s)], axis=1).astype(np.float64)
    return _order_points((g + 0.5) / float(s), order, n)


def read_mesh(path: str) -> np.ndarray:
    """x y z triples of a mesh file (whitespace separated, '#' comments)."""
    vals = []
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0]
            for tok in line.split():
                v = float(tok)
                if not math.isfinite(v):
                    raise ValueError("mesh file: a token that is not a finite number")
                vals.append(v)
    if not vals or len(vals) % 3:
        raise ValueError("mesh file: expected x y z triples")
    return np.array(vals, dtype=np.float64).reshape(-1, 3)


def virus_points(mesh: np.ndarray, n: int, prob: "Problem") -> np.ndarray:
    """md-3d-virus population (``testing_dpotrf.c:366-374``; STARS-H's
    ``starsh_generate_3d_rbf_mesh_coordinates_virus`` is absent from the
    reference tree, so the placement is the restatement's own rule):
    ``numobj`` copies of the mesh, each centred on its bounding-box centre
    (diameter d = the box diagonal), on a cubic lattice of side
    ceil(cbrt(numobj)) with spacing d cbrt(pi / (6 density)) (density capped
    at pi/6, where the bounding spheres touch), or, for density <= 0, at
    centres uniform in a cube of side 2 d cbrt(numobj) (seeded counter
    generator); Morton ordered when ``order == 1``; the first n nodes."""
    nobj = prob.numobj if prob.numobj > 0 else 1
    M = mesh.shape[0]
    if n > nobj * M:
        raise ValueError("N exceeds numobj times the mesh's node count")
    lo, hi = mesh.min(axis=0), mesh.max(axis=0)
    d2 = 0.0
    for a in range(3):
        d2 += (hi[a] - lo[a]) * (hi[a] - lo[a])
    d = math.sqrt(d2) if math.sqrt(d2) > 0.0 else 1.0
    side = grid_side(nobj, 3)
    o = np.arange(nobj, dtype=np.int64)
    if prob.density > 0.0:
        dens = min(prob.density, math.pi / 6.0)
        spacing = d * math.cbrt(math.pi / (6.0 * dens))
        ctr = spacing * np.stack([o % side, (o // side) % side, o // (side * side)], axis=1).astype(np.float64)
    else:
        L = 2.0 * d * math.cbrt(float(nobj))
        sd = (prob.seed ^ MESH_SEED_XOR) & 0xFFFFFFFFFFFFFFFF
        ctr = L * uniform01(sd, np.arange(3 * nobj, dtype=np.uint64)).reshape(nobj, 3)
    centred = mesh - 0.5 * (lo + hi)
    c = (ctr[:, None, :] + centred[None, :, :]).reshape(-1, 3)
    return _order_points(c, prob.order, n)


def rbf_phi(f: int, s: np.ndarray) -> np.ndarray:
    """Radial basis functions of s = r / radius (-B, ``hicma_parsec.c:80``):
    Gaussian exp(-s^2), exponential exp(-s), inverse quadratic 1/(1+s^2),
    inverse multiquadric 1/sqrt(1+s^2), Matern C1 (1+s) exp(-s), Matern C2
    (1 + s + s^2/3) exp(-s), thin-plate spline s^2 log s, compactly supported
    thin-plate (1-s)^5 and Wendland C2 (1-s)^4 (4s+1) on s < 1."""
    with np.errstate(divide="ignore", invalid="ignore"):
        if f == RBF_GAUSSIAN:
            return np.exp(-(s * s))
        if f == RBF_EXPON:
            return np.exp(-s)
        if f == RBF_INVQUAD:
            return 1.0 / (1.0 + s * s)
        if f == RBF_INVMQUAD:
            return 1.0 / np.sqrt(1.0 + s * s)
        if f == RBF_MATERNC1:
            return (1.0 + s) * np.exp(-s)
        if f == RBF_MATERNC2:
            return ((1.0 + s) + (s * s) / 3.0) * np.exp(-s)
        if f == RBF_TPS:
            return np.where(s > 0.0, (s * s) * np.log(np.where(s > 0.0, s, 1.0)), 0.0)
        t = 1.0 - s
        t2 = t * t
        if f == RBF_CTPS:
            return np.where(s < 1.0, (t2 * t2) * t, 0.0)
        if f == RBF_WENDLAND:
            return np.where(s < 1.0, (t2 * t2) * (4.0 * s + 1.0), 0.0)
    raise ValueError(f"rbf_kernel {f}")


# --------------------------------------------------------------------------
# Covariance kernels (STARS-H ssdata block kernels, restated)
# --------------------------------------------------------------------------
@dataclass
class Problem:
    kind: int = KIND_SQEXP_2D
    beta: float = 0.1          # testing_dpotrf.c:303
    nu: float = 0.5            # testing_dpotrf.c:304 (unused by sqexp/exp)
    noise: float = 0.1         # testing_dpotrf.c:305 (the reference's nugget)
    sigma: float = 1.0         # testing_dpotrf.c:306
    seed: int = 0
    wave_k: float = 50.0       # electrodynamics wave number (hicma_parsec.c:188, flag -w)
    add_diag: float = 0.0      # electrodynamics / mesh diagonal; <= 0 means N (hicma_parsec.c:289-291, flag -j)
    rbf_kernel: int = RBF_GAUSSIAN   # mesh kinds: basis function (flag -B)
    radius: float = 0.0        # mesh kinds: shape radius (flag -R)
    numobj: int = 1            # md-3d-virus: copies of the mesh (flag -K)
    order: int = 1             # mesh kinds: 0 no reordering, 1 Morton (flag -O)
    density: float = -1.0      # md-3d-virus: packing density, <= 0 random (flag -S)

    @property
    def ndim(self) -> int:
        return KIND_NDIM[self.kind]


def gaussian_counter(seed: int, rows: int, cols: int) -> np.ndarray:
    """rows x cols standard normals, column-major counter i = r + c * rows:
    Box-Muller on u1 = (53 high bits of mix64(mix64(seed) + 2i) + 1) 2**-53 and
    u2 = (53 high bits of mix64(mix64(seed) + 2i + 1)) 2**-53, g = sqrt(-2 ln u1)
    cos(2 pi u2).  The same generator fills the device's sketch matrices."""
    i = np.arange(rows * cols, dtype=np.uint64)
    base = _mix64(np.array([seed], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        z1 = _mix64(base + np.uint64(2) * i)
        z2 = _mix64(base + np.uint64(2) * i + np.uint64(1))
    u1 = ((z1 >> np.uint64(11)).astype(np.float64) + 1.0) * (2.0 ** -53)
    u2 = (z2 >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)
    g = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    return g.reshape(cols, rows).T


def randtlr_basis(n: int, nb: int, seed: int = 0) -> np.ndarray:
    """STARS-H ``starsh_randtlr_generate(data, N, NB, decay=0.5, add_diag)``
    (``testing_dpotrf.c:315-321``), restated: every block row m gets an
    orthonormal NB x NB basis Q_m from the QR of a Gaussian matrix, and the
    singular values are S_0 = 1, S_k = S_{k-1} * decay, so every off-diagonal
    tile Q_m diag(S) Q_n^T has the same spectrum (the "equal ranks" problem).

    Only the first K = min(NB, 64) columns of each Q_m are formed (the first K
    columns of a QR depend only on the first K columns of its input, and
    0.5**64 is far below the FP64 resolution of the tile entries).  The
    Gaussian input of block m comes from :func:`gaussian_counter` with seed
    ``(seed ^ RANDTLR_SEED_XOR) + m``; column signs are fixed so that R has a
    positive diagonal (the unique thin QR).  Returns the (n, 2K) array
    [Q | Q diag(S)], which plays the part of the points array."""
    if n % nb != 0:
        raise ValueError("N must be a multiple of NB")
    K = min(nb, RANDTLR_KMAX)
    S = RANDTLR_DECAY ** np.arange(K, dtype=np.float64)
    out = np.empty((n, 2 * K))
    for m in range(n // nb):
        sd = ((seed ^ RANDTLR_SEED_XOR) + m) & 0xFFFFFFFFFFFFFFFF
        Q, R = np.linalg.qr(gaussian_counter(sd, nb, K))
        Q = Q * np.where(np.diag(R) < 0.0, -1.0, 1.0)
        out[m * nb:(m + 1) * nb, :K] = Q
        out[m * nb:(m + 1) * nb, K:] = Q * S
    return out


def problem_points(prob: "Problem", n: int, nb: int) -> np.ndarray:
    """The per-row data a problem's kernel reads: points (n, ndim) for the
    point kernels, the (n, 2K) basis for randtlr."""
    if prob.kind == KIND_RANDTLR:
        return randtlr_basis(n, nb, prob.seed)
    if prob.kind == KIND_MD_CUBE:
        return cube_points(n, prob.order)
    if prob.kind == KIND_MD_VIRUS:
        raise ValueError("md-3d-virus points come from a mesh (virus_points)")
    return gen_points(n, prob.ndim, prob.seed)


def cov_block(prob: Problem, pts: np.ndarray, r0: int, nr: int, c0: int, nc: int) -> np.ndarray:
    """Column-major covariance block A[r0:r0+nr, c0:c0+nc]; the nugget is
    added where the global row and column indices coincide.  Same call shape
    as ``kernel(nrows, ncols, irow, icol, data, data, out, ld)``
    (``STARSH_gen.jdf:70-72``).

    Electrodynamics kinds (``-D 1``, ``-D 5``): ``sin(k r) / r`` with ``k`` the
    wave number, and ``add_diag`` (N when not positive) where ``r == 0``; no
    nugget, no variance.  randtlr (``-D 0``): ``pts`` is the basis of
    :func:`randtlr_basis` and the block is Q[rows] (Q diag(S))[cols]^T with
    ``add_diag`` where the global indices coincide."""
    X = pts[r0:r0 + nr]
    Y = pts[c0:c0 + nc]
    if prob.kind == KIND_RANDTLR:
        K = pts.shape[1] // 2
        A = X[:, :K] @ Y[:, K:].T
        lo, hi = max(r0, c0), min(r0 + nr, c0 + nc)
        if lo < hi:
            i = np.arange(lo, hi)
            A[i - r0, i - c0] += prob.add_diag if prob.add_diag > 0.0 else float(pts.shape[0])
        return A
    r2 = np.zeros((nr, nc))
    for a in range(pts.shape[1]):
        d = X[:, a][:, None] - Y[:, a][None, :]
        r2 = r2 + d * d
    if prob.kind in (KIND_MD_VIRUS, KIND_MD_CUBE):
        A = rbf_phi(prob.rbf_kernel, np.sqrt(r2) * (1.0 / prob.radius))
        lo, hi = max(r0, c0), min(r0 + nr, c0 + nc)
        if lo < hi:
            i = np.arange(lo, hi)
            A[i - r0, i - c0] += prob.add_diag if prob.add_diag > 0.0 else float(pts.shape[0])
        return A
    if prob.kind in (KIND_ED_SIN_2D, KIND_ED_SIN_3D):
        r = np.sqrt(r2)
        diag = prob.add_diag if prob.add_diag > 0.0 else float(pts.shape[0])
        with np.errstate(divide="ignore", invalid="ignore"):
            A = np.sin(prob.wave_k * r) / r
        A[r2 == 0.0] = diag
        return A
    if prob.kind == KIND_EXP_3D:
        A = prob.sigma * np.exp(-np.sqrt(r2) / prob.beta)
    else:
        A = prob.sigma * np.exp(-r2 / (2.0 * prob.beta * prob.beta))
    lo, hi = max(r0, c0), min(r0 + nr, c0 + nc)
    if lo < hi:
        i = np.arange(lo, hi)
        A[i - r0, i - c0] += prob.noise
    return A


def dense_matrix(prob: Problem, pts: np.ndarray) -> np.ndarray:
    n = pts.shape[0]
    return cov_block(prob, pts, 0, n, 0, n)


# --------------------------------------------------------------------------
# op_counts.h restated (integer/float quirks kept)
# --------------------------------------------------------------------------
_U64 = (1 << 64) - 1


def _f32(x) -> float:
    return float(np.float32(x))


def op_counts(op: str, a: int, b: int, c: int, d: int) -> int:
    """``op_counts`` of ``hicma_parsec/op_counts.h:10-72`` with unsigned long
    wrap-around and its float32 casts in the geqrf branch."""
    if op == "q":
        m, n = a, b
        t1 = (2 * m * n * n) & _U64
        t2 = int(_f32(_f32((2 * n * n * n) & _U64) / np.float32(3.0)))
        t3 = (2 * m * n) & _U64
        t4 = int(_f32(_f32((17 * n) & _U64) / np.float32(3.0)))
        return (t1 - t2 + t3 + t4) & _U64
    if op == "c":
        n = a
        v = float(((n * n * n) & _U64) // 3) - float((n * n) & _U64) / 2.0 + float(n // 6)
        return int(v) & _U64
    if op == "t":
        m, n, side = a, b, c
        return (n * m * m) & _U64 if side == 1 else (m * n * n) & _U64
    if op == "m":
        return (a * b * c * 2) & _U64
    if op == "s":
        return (22 * a * a * a) & _U64
    if op == "o":
        m, n, k, side = a, b, c, d
        if side == 1:
            return (4 * n * m * k - 2 * n * k * k + 3 * n * k) & _U64
        return (4 * n * m * k - 2 * m * k * k + 2 * m * k + n * k - (k * k) // 2 + k // 2) & _U64
    if op == "r":
        m, n, side = a, b, c
        return (m * m * n) & _U64 if side == 1 else (m * n * n) & _U64
    raise ValueError(op)


def flops_dpotrf(n: float) -> float:
    """FLOPS_DPOTRF of ``flops.h:86-87,272`` (dense-equivalent flop count)."""
    n = float(n)
    fmuls = n * (((1.0 / 6.0) * n + 0.5) * n + (1.0 / 3.0))
    fadds = n * (((1.0 / 6.0) * n) * n - (1.0 / 6.0))
    return fmuls + fadds


def gemm_lr_opcount(nb: int, ra: int, rb: int, rc_old: int, rc_new: int, b_dense: bool) -> int:
    """Op count of a low-rank-C GEMM task, ``HiCMA_dpotrf_L_2flow.jdf:909-924``
    (B dense) and ``:1076-1092`` (B low rank)."""
    ka = rc_old + ra
    qra = op_counts("q", nb, ka, 0, 0)
    if b_dense:
        qrb = op_counts("q", nb, ka, 0, 0) + op_counts("m", ra, nb, nb, 0)
    else:
        qrb = op_counts("m", ra, rb, nb, 0) + op_counts("m", ra, nb, rb, 0) + op_counts("q", nb, ka, 0, 0)
    svd = op_counts("r", ka, ka, 2, 0) + op_counts("s", ka, 0, 0, 0) + ka * rc_new
    newu = op_counts("o", nb, rc_new, ka, 1)
    newv = op_counts("o", rc_new, nb, ka, 2)
    return (qra + qrb + svd + newu + newv) & _U64


# --------------------------------------------------------------------------
# TLR matrix
# --------------------------------------------------------------------------
@dataclass
class TLRMatrix:
    n: int
    nb: int
    band: int
    maxrank: int
    dense: dict = field(default_factory=dict)   # (m, n) -> NB x NB array
    U: dict = field(default_factory=dict)       # (m, n) -> NB x r
    V: dict = field(default_factory=dict)       # (m, n) -> NB x r

    @property
    def nt(self) -> int:
        return self.n // self.nb

    def is_dense(self, m: int, n: int) -> bool:
        return m - n < self.band

    def rank(self, m: int, n: int) -> int:
        return -1 if self.is_dense(m, n) else self.U[(m, n)].shape[1]

    def rank_array(self) -> np.ndarray:
        """Column-major NT x NT map, -1 on the band and the upper triangle
        (``testing_dpotrf.c:450-453``)."""
        nt = self.nt
        G = -np.ones(nt * nt, dtype=np.int32)
        for (m, n), u in self.U.items():
            G[n * nt + m] = u.shape[1]
        return G

    def copy(self) -> "TLRMatrix":
        return TLRMatrix(self.n, self.nb, self.band, self.maxrank,
                         {k: v.copy() for k, v in self.dense.items()},
                         {k: v.copy() for k, v in self.U.items()},
                         {k: v.copy() for k, v in self.V.items()})


def truncation_rank_relfro(s: np.ndarray, tol: float) -> int:
    """Smallest r with ||s[r:]||_2 <= tol * ||s||_2 (restated STARS-H rule)."""
    s2 = s.astype(np.float64) ** 2
    total = float(s2.sum())
    if total == 0.0:
        return 0
    thr = tol * tol * total
    tail = 0.0
    r = len(s)
    while r > 0 and tail + s2[r - 1] <= thr:
        tail += s2[r - 1]
        r -= 1
    return r


def compress_tile(A: np.ndarray, tol: float, maxrank: int, oversample: int = 10):
    """Compress one off-band tile (``STARSH_gen.jdf:127-213``): returns
    (U, V, rank) with rank -1 when the tile is rejected.  The spectrum is
    restricted to the ``min(maxrank + oversample, NB)`` leading values, the
    sample size the reference sizes its workspace for (``:262-266``)."""
    m, n = A.shape
    u, s, vt = np.linalg.svd(A, full_matrices=False)
    ns = min(maxrank + oversample, min(m, n))
    s = s[:ns]
    r = truncation_rank_relfro(s, tol)
    if not (r < min(m, n) / 2 and r <= maxrank):
        return None, None, -1
    U = np.ascontiguousarray(u[:, :r])
    V = np.ascontiguousarray(vt[:r].T * s[:r])
    return U, V, r


def compress_tile_rsvd(A: np.ndarray, tol: float, maxrank: int, oversample: int = 10, seed: int = 0):
    """Randomized variant of :func:`compress_tile` (range finder with
    ``min(maxrank + oversample, NB)`` Gaussian samples, then an exact SVD of
    the projected tile), the algorithm the CUDA generator implements."""
    m, n = A.shape
    s = min(maxrank + oversample, min(m, n))
    Om = np.random.default_rng(seed).standard_normal((n, s))
    Q, _ = np.linalg.qr(A @ Om)
    Qw, Rw = np.linalg.qr(A.T @ Q)
    u, sv, vt = np.linalg.svd(Rw.T)
    r = truncation_rank_relfro(sv, tol)
    if not (r < min(m, n) / 2 and r <= maxrank):
        return None, None, -1
    return (np.ascontiguousarray(Q @ u[:, :r]), np.ascontiguousarray(Qw @ (vt[:r].T * sv[:r])), r)


def generate(prob: Problem, n: int, nb: int, tol: float, maxrank: int, band: int = 1,
             pts: np.ndarray | None = None):
    """``STARSH_gen`` (``STARSH_gen.jdf:342-369``): dense band tiles
    ``m - band < n <= m`` (``:45-83``) and compressed off-band tiles
    (``:127-213``).  Returns (TLRMatrix, info) with info = -1 if a tile was
    rejected."""
    if n % nb != 0:
        raise ValueError("N must be a multiple of NB")
    if pts is None:
        pts = problem_points(prob, n, nb)
    T = TLRMatrix(n, nb, band, maxrank)
    nt = n // nb
    info = 0
    for m in range(nt):
        for c in range(max(m - band + 1, 0), m + 1):
            T.dense[(m, c)] = cov_block(prob, pts, m * nb, nb, c * nb, nb)
    for m in range(band, nt):
        for c in range(0, m - band + 1):
            U, V, r = compress_tile(cov_block(prob, pts, m * nb, nb, c * nb, nb), tol, maxrank)
            if r < 0:
                info = -1
                U = np.zeros((nb, 0))
                V = np.zeros((nb, 0))
            T.U[(m, c)] = U
            T.V[(m, c)] = V
    return T, info


def band_regenerate(T: TLRMatrix, prob: Problem, pts: np.ndarray, band: int) -> None:
    """``parsec_band_regenerate`` (``band_regenerate.jdf:27-64``): tiles with
    ``m - n < band`` become dense kernel tiles; the others keep their [U,V]."""
    nt, nb = T.nt, T.nb
    for m in range(nt):
        for c in range(max(m - band + 1, 0), m + 1):
            T.dense[(m, c)] = cov_block(prob, pts, m * nb, nb, c * nb, nb)
            T.U.pop((m, c), None)
            T.V.pop((m, c), None)
    T.band = band


# --------------------------------------------------------------------------
# Rank statistics and band auto-tuning
# --------------------------------------------------------------------------
def rank_stat(G: np.ndarray, nt: int, band: int):
    """``HICMA_get_stat2`` (``hicma_internal.c:52-71``): (min, max, avg) over
    tiles i >= band, j <= i - band."""
    vals = [int(G[j * nt + i]) for i in range(band, nt) for j in range(0, i - band + 1)]
    if not vals:
        return 2**31 - 1, 0, float("nan")
    return min(vals), max(vals), float(sum(vals)) / len(vals)


def band_autotune(G: np.ndarray, nt: int, nb: int, verbose: bool = False) -> int:
    """``parsec_band_size_auto_tuning`` (``band_size_auto_tuning.jdf:201-318``).

    For band b = 2..NT-1 it sums the modelled TLR and dense flops of the TRSMs
    (``:36-65``) and GEMMs (``:70-127``) on sub-diagonal b-1.  It records
    ``opt_min = b - 1`` at the first b with ``tlr * FLUCTUATION <= dense`` and
    returns ``opt_min`` at the first b with ``tlr <= dense`` (``:290-313``),
    else NT.  The reference keeps ``opt_min`` in file-static variables that
    are never reset between calls; this restatement resets them per call.
    """
    indicator_min = 0
    opt_min = 0
    for band in range(2, nt):
        t_tlr = t_dense = g_tlr = g_dense = 0
        for m in range(band - 1, nt):
            k = m + 1 - band
            ar = int(G[k * nt + m])
            t_tlr += nb * nb * ar
            t_dense += nb * nb * nb
        for k in range(0, nt - 2):
            for m in range(k + band, nt):
                n = m + 1 - band
                ar = int(G[k * nt + m])
                br = int(G[k * nt + n])
                cr = int(G[n * nt + m])
                ca = cr + ar
                qra = op_counts("q", nb, ca, 0, 0)
                qrb = op_counts("m", ar, br, nb, 0) + op_counts("m", ar, nb, br, 0) + op_counts("q", nb, ca, 0, 0)
                svd = op_counts("r", ca, ca, 2, 0) + op_counts("s", ca, 0, 0, 0) + ca * cr
                newu = op_counts("o", nb, cr, ca, 1)
                newv = op_counts("o", cr, nb, ca, 2)
                g_tlr += (qra + qrb + svd + newu + newv) & _U64
                if m - k < band:
                    g_dense += 2 * nb * nb * nb
                elif n - k < band and m - n < band:
                    g_dense += 4 * nb * nb * ar
                elif m - n < band:
                    g_dense += 2 * nb * nb * min(ar, br) + 4 * nb * ar * br
        s_tlr = t_tlr + g_tlr
        s_dense = t_dense + g_dense
        if verbose:
            print(f"band_size: {band}, ops_sum_tlr: {float(s_tlr):e}, ops_sum_dense: {float(s_dense):e}")
        if float(s_tlr) * FLUCTUATION <= float(s_dense) and indicator_min == 0:
            indicator_min = 1
            opt_min = band - 1
        if s_tlr <= s_dense:
            return opt_min
    return nt


# --------------------------------------------------------------------------
# Tile kernels (HCORE / CORE_d* restated)
# --------------------------------------------------------------------------
def qr_scholqr3(V: np.ndarray):
    """(Q, R) of V = Q R by shifted CholeskyQR3 as in :func:`r_factor_scholqr3`,
    with Q = V D^-1 R_1^-1 R_2^-1 R_3^-1 formed by three row-wise triangular
    solves.  The device's U side of a recompression: [Cu, Au] = Q_U R_U."""
    m, K = V.shape
    d = np.linalg.norm(V, axis=0)
    d[d == 0.0] = 1.0
    X = V / d
    R = np.eye(K)
    u = np.finfo(np.float64).eps / 2
    for p in range(3):
        G = X.T @ X
        shift = 11.0 * (m * K + K * (K + 1)) * u * float(np.trace(G))
        try:
            Rp = np.linalg.cholesky(G + (shift if p == 0 else 0.0) * np.eye(K)).T
        except np.linalg.LinAlgError:
            Rp = np.linalg.cholesky(G + shift * np.eye(K)).T
        X = sla.solve_triangular(Rp, X.T, trans="T", lower=False).T
        R = Rp @ R
    return X, R * d


def r_factor_scholqr3(V: np.ndarray) -> np.ndarray:
    """R of V = Q R (Q not formed) by shifted CholeskyQR3 (Fukaya, Kannan,
    Nakatsukasa, Yamamoto and Yanagisawa, SIAM J. Sci. Comput. 42(1), 2020):
    columns scaled to unit norm, then three passes of G = X^T X, R_p = chol(G)
    and X <- X R_p^-1, the first with the shift 11 (m K + K (K + 1)) u ||X||^2
    (||X||_F^2 bounds ||X||_2^2), later ones shifted the same way only if the
    plain Cholesky breaks down; R = R_3 R_2 R_1 D.  A candidate for the V side
    of the recompression built from Gram products and triangular multiplies
    (tensor-core friendly) instead of Householder reflections."""
    m, K = V.shape
    d = np.linalg.norm(V, axis=0)
    d[d == 0.0] = 1.0
    X = V / d
    R = np.eye(K)
    u = np.finfo(np.float64).eps / 2
    for p in range(3):
        G = X.T @ X
        shift = 11.0 * (m * K + K * (K + 1)) * u * float(np.trace(G))
        try:
            Rp = np.linalg.cholesky(G + (shift if p == 0 else 0.0) * np.eye(K)).T
        except np.linalg.LinAlgError:
            Rp = np.linalg.cholesky(G + shift * np.eye(K)).T
        X = sla.solve_triangular(Rp, X.T, trans="T", lower=False).T
        R = Rp @ R
    return R * d


# randomized CholeskyQR as the device runs it (k_cholqr.cu)
RCQ_ROWS = 256       # sketch rows (one per thread of the device's CTA)
RCQ_APPLY = 3        # passes over the rows at most
RCQ_GMAX = 1e4       # ||Y^T Y||_inf above this: the sketch missed a direction of range(X)
RCQ_TINY = 1e-200    # pivot floor when the Gram matrix is zero
RCQ_KMAX = 64        # widest stack the device factors this way


def sketch_signs(m: int) -> np.ndarray:
    """Signs of rows 0..m-1 in the CountSketch of :func:`qr_rcholqr`: the low
    bit of a 32-bit integer hash of the row index (xor-shift / multiply rounds
    of the "lowbias32" mixer; arithmetic modulo 2^32)."""
    x = np.arange(m, dtype=np.uint32)
    x ^= x >> np.uint32(16)
    x *= np.uint32(0x7FEB352D)
    x ^= x >> np.uint32(15)
    x *= np.uint32(0x846CA68B)
    x ^= x >> np.uint32(16)
    return np.where(x & np.uint32(1), -1.0, 1.0)


def _chol_local(G: np.ndarray, m: float, shifted: bool):
    """R = chol(G + shift)^T as the device factors it: right-looking
    elimination with s = 11 (m K + K (K + 1)) u tr(G) added to the diagonal
    when ``shifted``; a pivot that is not positive (a column dependent on the
    ones before it, or zero) becomes s (RCQ_TINY when s = 0) with its column
    below the diagonal zeroed and no trailing update, so the other columns keep
    their factor.  Returns (R, number of such null pivots)."""
    K = G.shape[0]
    u = np.finfo(np.float64).eps / 2
    s0 = 11.0 * (m * K + K * (K + 1)) * u * float(np.trace(G))
    floor = s0 if s0 > 0.0 else RCQ_TINY
    A = np.array(G, dtype=np.float64)
    if shifted and s0 > 0.0:
        A[np.diag_indices(K)] += s0
    L = np.zeros((K, K))
    nnull = 0
    for j in range(K):
        d = A[j, j]
        if not d > 0.0:
            nnull += 1
            L[j, j] = math.sqrt(floor)
            continue
        p = math.sqrt(d)
        L[j, j] = p
        L[j + 1:, j] = A[j + 1:, j] / p
        A[j + 1:, j + 1:] -= np.outer(A[j + 1:, j], A[j + 1:, j] / d)
    return L.T, nnull


def qr_rcholqr(X: np.ndarray):
    """QR of a tall-skinny X by randomized CholeskyQR, the device's form for
    stacks up to 64 columns (both sides of a recompression, the generation
    range finder): a 256-row CountSketch S (row i of X, times
    :func:`sketch_signs`, added to row i mod 256), Rs = R of S by shifted
    CholeskyQR3 (column norms D of S, R1 = chol(D^-1 S^T S D^-1 + s I) with
    m = 256, then two unshifted steps; Rs = R3 R2 R1 D), then
    Y = X Rs^-1, Rc = chol(Y^T Y), R = Rc Rs, Q = Y Rc^-1; repeated with R
    in place of Rs while ||Y^T Y||_inf > RCQ_GMAX (at most RCQ_APPLY passes).
    Every Cholesky factorization treats a non-positive pivot locally
    (:func:`_chol_local`).
    Published algorithms: Fan, Guo and Lin (2021) and Balabanov (2022) for the
    randomized preconditioning, Fukaya et al. (SIAM J. Sci. Comput. 42(1),
    2020) for shifted CholeskyQR3.  Returns (Y, Rc, R, passes)."""
    m, K = X.shape
    S = np.zeros((RCQ_ROWS, K))
    np.add.at(S, np.arange(m) % RCQ_ROWS, X * sketch_signs(m)[:, None])
    G = S.T @ S
    d = np.sqrt(np.diag(G)).copy()
    d[~(d > 0.0)] = 1.0
    R1, _ = _chol_local(G / np.outer(d, d), RCQ_ROWS, True)
    Rt = R1 * d
    Sk = sla.solve_triangular(R1, (S / d).T, trans="T", lower=False).T
    for rnd in range(2):
        Rp, _ = _chol_local(Sk.T @ Sk, RCQ_ROWS, False)
        Rt = Rp @ Rt
        if rnd == 0:
            Sk = sla.solve_triangular(Rp, Sk.T, trans="T", lower=False).T
    for p in range(RCQ_APPLY):
        Y = sla.solve_triangular(Rt, X.T, trans="T", lower=False).T
        G = Y.T @ Y
        gmax = float(np.abs(G).sum(axis=1).max()) if K else 0.0
        Rc, _ = _chol_local(G, m, False)
        Rt = Rc @ Rt
        if gmax <= RCQ_GMAX:
            break
    return Y, Rc, Rt, p + 1


def recompress(Cu, Cv, Au, Y, acc, maxrank, fixed_rank=0, v_side="householder", u_side="householder"):
    """C_new = [Cu, Au] [Cv, -Y]^T recompressed (restated
    ``HCORE_dgemm_qr_svd`` + ``HCORE_dgemm_ormqr``, call sites
    ``HiCMA_dpotrf_L_2flow.jdf:830-903,985-1058``).  Returns
    (U, V, rank, overflow).  ``v_side="scholqr3"`` takes R_V from
    :func:`r_factor_scholqr3` and forms the new V as [Cv, -Y] R_U^T U_r (no
    Q_V needed), and ``u_side="scholqr3"`` takes Q_U, R_U from
    :func:`qr_scholqr3`; ``"rcholqr"`` on either side takes them from
    :func:`qr_rcholqr` for stacks up to RCQ_KMAX columns (Householder for
    wider ones), as the device does."""
    Us = np.hstack([Cu, Au])
    Vs = np.hstack([Cv, -Y])
    nb, K = Us.shape
    if K == 0:
        return np.zeros((nb, 0)), np.zeros((nb, 0)), 0, False
    # the device takes the randomized CholeskyQR for stacks up to RCQ_KMAX columns
    if K > RCQ_KMAX:
        u_side = "householder" if u_side == "rcholqr" else u_side
        v_side = "householder" if v_side == "rcholqr" else v_side
    if u_side == "rcholqr":
        Yu, Rcu, Ru, _ = qr_rcholqr(Us)
        Qu = sla.solve_triangular(Rcu, Yu.T, trans="T", lower=False).T
    else:
        Qu, Ru = qr_scholqr3(Us) if u_side == "scholqr3" else np.linalg.qr(Us)
    if v_side == "scholqr3":
        Rv = r_factor_scholqr3(Vs)
    elif v_side == "rcholqr":
        Rv = qr_rcholqr(Vs)[2]
    else:
        Qv, Rv = np.linalg.qr(Vs)
    u, s, vt = np.linalg.svd(Ru @ Rv.T)
    if fixed_rank > 0:
        r = min(fixed_rank, K)
    else:
        r = int(np.count_nonzero(s >= acc))
    overflow = r > maxrank
    r = min(r, maxrank)
    if v_side in ("scholqr3", "rcholqr"):
        return (np.ascontiguousarray(Qu @ u[:, :r]), np.ascontiguousarray(Vs @ (Ru.T @ u[:, :r])), r, overflow)
    return (np.ascontiguousarray(Qu @ u[:, :r]),
            np.ascontiguousarray(Qv @ (vt[:r].T * s[:r])), r, overflow)


@dataclass
class FactorStats:
    info: int = 0
    overflow: int = 0
    tileopcounters: np.ndarray | None = None
    op_band: int = 0
    op_offband: int = 0
    op_path: int = 0
    op_offpath: int = 0
    # rank history (the reference's dcRank record, HiCMA_dpotrf_L_2flow.jdf:353-361,
    # 683-691,1101-1106): per off-band tile [m, n] the rank it entered with and the
    # smallest / largest rank it held; -1 outside the low-rank part
    rank_init: np.ndarray | None = None
    rank_min: np.ndarray | None = None
    rank_max: np.ndarray | None = None

    @property
    def total(self) -> int:
        return int(self.tileopcounters.sum())


def potrf_tile(A: np.ndarray):
    """Lower Cholesky of a dense tile; returns (L, iinfo) with iinfo the
    1-based order of the first non-positive leading minor (0 on success)."""
    try:
        return np.linalg.cholesky(A), 0
    except np.linalg.LinAlgError:
        n = A.shape[0]
        L = np.tril(A).copy()
        for j in range(n):
            d = L[j, j] - np.dot(L[j, :j], L[j, :j])
            if not d > 0.0:
                return L, j + 1
            L[j, j] = math.sqrt(d)
            L[j + 1:, j] = (L[j + 1:, j] - L[j + 1:, :j] @ L[j, :j]) / L[j, j]
        return L, 0


def tlr_potrf(T: TLRMatrix, acc: float, fixed_rank: int = 0, stop_on_error: bool = True,
              v_side: str = "householder", u_side: str = "householder") -> FactorStats:
    """In-place 2-flow TLR Cholesky (``HiCMA_dpotrf_L_2flow.jdf:175-1113``)
    run in a sequential order compatible with its data flow."""
    nt, nb, band = T.nt, T.nb, T.band
    st = FactorStats(tileopcounters=np.zeros((nt, nt), dtype=np.uint64))
    tile_ops = st.tileopcounters
    st.rank_init = np.full((nt, nt), -1, dtype=np.int64)
    for (m, n) in T.U:
        st.rank_init[m, n] = T.rank(m, n)
    st.rank_min = st.rank_init.copy()
    st.rank_max = st.rank_init.copy()

    def track(m, n, r):
        st.rank_min[m, n] = min(st.rank_min[m, n], r)
        st.rank_max[m, n] = max(st.rank_max[m, n], r)

    def log(cnt, i, j, region, path):
        tile_ops[i, j] += np.uint64(cnt & _U64)
        if region == "band":
            st.op_band += cnt
        else:
            st.op_offband += cnt
        if path:
            st.op_path += cnt
        else:
            st.op_offpath += cnt

    for k in range(nt):
        # potrf_dpotrf(k): :175-245
        log(op_counts("c", nb, 0, 0, 0), k, k, "band", True)
        L, iinfo = potrf_tile(T.dense[(k, k)])
        T.dense[(k, k)] = np.tril(L)
        if iinfo != 0:
            if st.info == 0:
                st.info = k * nb + iinfo
            if stop_on_error:
                return st
        Lkk = T.dense[(k, k)]
        # potrf_dtrsm(m, k): :366-401
        for m in range(k + 1, nt):
            if m - k < band:
                log(op_counts("t", nb, nb, 1, 0), m, k, "band", m - k == 1)
                T.dense[(m, k)] = sla.solve_triangular(Lkk, T.dense[(m, k)].T, lower=True).T
            else:
                r = T.U[(m, k)].shape[1]
                log(op_counts("t", nb, r, 1, 0), m, k, "offband", m - k == 1)
                if r == 0:
                    continue
                T.V[(m, k)] = sla.solve_triangular(Lkk, T.V[(m, k)], lower=True)
        # potrf_dsyrk(k, m): :503-565
        for m in range(k + 1, nt):
            if m - k < band:
                A = T.dense[(m, k)]
                log(op_counts("m", nb, nb, nb, 0), m, m, "band", m - k == 1)
                T.dense[(m, m)] = T.dense[(m, m)] - A @ A.T
            else:
                U, V = T.U[(m, k)], T.V[(m, k)]
                r = U.shape[1]
                cnt = op_counts("m", r, r, nb, 0) + op_counts("m", nb, r, r, 0) + op_counts("m", nb, nb, r, 0)
                log(cnt, m, m, "band", m - k == 1)
                if r == 0:
                    continue
                T.dense[(m, m)] = T.dense[(m, m)] - U @ ((V.T @ V) @ U.T)
        # potrf_dgemm(m, n, k): :699-1097
        for m in range(k + 2, nt):
            for n in range(k + 1, m):
                if m - k < band:                                   # (i) :699-708
                    log(op_counts("m", nb, nb, nb, 0), m, n, "band", False)
                    T.dense[(m, n)] = T.dense[(m, n)] - T.dense[(m, k)] @ T.dense[(n, k)].T
                elif n - k < band and m - n < band:                # (ii) :710-730
                    Au, Av = T.U[(m, k)], T.V[(m, k)]
                    ra = Au.shape[1]
                    log(op_counts("m", nb, nb, ra, 0) * 2, m, n, "band", False)
                    tmp = Av.T @ T.dense[(n, k)].T
                    T.dense[(m, n)] = T.dense[(m, n)] - Au @ tmp
                elif m - n < band:                                 # (iii) :732-782
                    Au, Av = T.U[(m, k)], T.V[(m, k)]
                    Bu, Bv = T.U[(n, k)], T.V[(n, k)]
                    ra, rb = Au.shape[1], Bu.shape[1]
                    log(op_counts("m", nb, nb, min(ra, rb), 0) + op_counts("m", nb, ra, rb, 0) * 2,
                        m, n, "band", False)
                    rr = Av.T @ Bv
                    if ra > rb:
                        T.dense[(m, n)] = T.dense[(m, n)] - (Au @ rr) @ Bu.T
                    else:
                        T.dense[(m, n)] = T.dense[(m, n)] - Au @ (rr @ Bu.T)
                elif n - k < band:                                 # (iv) :784-927
                    Au, Av = T.U[(m, k)], T.V[(m, k)]
                    ra = Au.shape[1]
                    rc_old = T.U[(m, n)].shape[1]
                    Y = T.dense[(n, k)] @ Av
                    U, V, r, ov = recompress(T.U[(m, n)], T.V[(m, n)], Au, Y, acc, T.maxrank, fixed_rank, v_side, u_side)
                    st.overflow += int(ov)
                    T.U[(m, n)], T.V[(m, n)] = U, V
                    track(m, n, r)
                    log(gemm_lr_opcount(nb, ra, 0, rc_old, r, True), m, n, "offband", False)
                else:                                              # (v) :929-1097
                    Au, Av = T.U[(m, k)], T.V[(m, k)]
                    Bu, Bv = T.U[(n, k)], T.V[(n, k)]
                    ra, rb = Au.shape[1], Bu.shape[1]
                    if ra == 0 or rb == 0:
                        continue
                    rc_old = T.U[(m, n)].shape[1]
                    Y = Bu @ (Bv.T @ Av)
                    U, V, r, ov = recompress(T.U[(m, n)], T.V[(m, n)], Au, Y, acc, T.maxrank, fixed_rank, v_side, u_side)
                    st.overflow += int(ov)
                    T.U[(m, n)], T.V[(m, n)] = U, V
                    track(m, n, r)
                    log(gemm_lr_opcount(nb, ra, rb, rc_old, r, False), m, n, "offband", False)
    return st


def tlr_potrf_dag(T: TLRMatrix, acc: float, threads: int, fixed_rank: int = 0) -> FactorStats:
    """The same 2-flow TLR Cholesky as :func:`tlr_potrf` (same task bodies),
    run as a task graph on ``threads`` host threads the way the reference's
    PaRSEC runtime runs it: a task starts as soon as the tiles it reads are
    final and the tile it writes has received every earlier update
    (``HiCMA_dpotrf_L_2flow.jdf`` flows), ready tasks are taken critical path
    first (lower panel index, then POTRF > TRSM > SYRK > GEMM, the order of the
    priorities at ``:50-61,189,290,429,611``), and every task calls BLAS and
    LAPACK on one thread (the reference links MKL sequential,
    ``hicma_parsec/CMakeLists.txt:47-54``).  The timed CPU baseline; results
    equal :func:`tlr_potrf`'s up to the rounding of single- versus
    multi-threaded BLAS.  Returns the op counts of the run."""
    import heapq
    import threading
    from threadpoolctl import threadpool_limits

    nt, nb, band = T.nt, T.nb, T.band
    st = FactorStats(tileopcounters=np.zeros((nt, nt), dtype=np.uint64))
    st.rank_init = np.full((nt, nt), -1, dtype=np.int64)
    for (m, n) in T.U:
        st.rank_init[m, n] = T.rank(m, n)
    st.rank_min = st.rank_init.copy()
    st.rank_max = st.rank_init.copy()
    lock = threading.Lock()
    ops = []          # (count, i, j)

    def potrf(k):
        L, iinfo = potrf_tile(T.dense[(k, k)])
        T.dense[(k, k)] = np.tril(L)
        if iinfo != 0:
            with lock:
                if st.info == 0 or k * nb + iinfo < st.info:
                    st.info = k * nb + iinfo
        return [(op_counts("c", nb, 0, 0, 0), k, k)]

    def trsm(m, k):
        Lkk = T.dense[(k, k)]
        if m - k < band:
            T.dense[(m, k)] = sla.solve_triangular(Lkk, T.dense[(m, k)].T, lower=True).T
            return [(op_counts("t", nb, nb, 1, 0), m, k)]
        r = T.U[(m, k)].shape[1]
        if r:
            T.V[(m, k)] = sla.solve_triangular(Lkk, T.V[(m, k)], lower=True)
        return [(op_counts("t", nb, r, 1, 0), m, k)]

    def syrk(k, m):
        if m - k < band:
            A = T.dense[(m, k)]
            T.dense[(m, m)] = T.dense[(m, m)] - A @ A.T
            return [(op_counts("m", nb, nb, nb, 0), m, m)]
        U, V = T.U[(m, k)], T.V[(m, k)]
        r = U.shape[1]
        cnt = op_counts("m", r, r, nb, 0) + op_counts("m", nb, r, r, 0) + op_counts("m", nb, nb, r, 0)
        if r:
            T.dense[(m, m)] = T.dense[(m, m)] - U @ ((V.T @ V) @ U.T)
        return [(cnt, m, m)]

    def gemm(m, n, k):
        if m - k < band:
            T.dense[(m, n)] = T.dense[(m, n)] - T.dense[(m, k)] @ T.dense[(n, k)].T
            return [(op_counts("m", nb, nb, nb, 0), m, n)]
        if n - k < band and m - n < band:
            Au, Av = T.U[(m, k)], T.V[(m, k)]
            T.dense[(m, n)] = T.dense[(m, n)] - Au @ (Av.T @ T.dense[(n, k)].T)
            return [(op_counts("m", nb, nb, Au.shape[1], 0) * 2, m, n)]
        if m - n < band:
            Au, Av = T.U[(m, k)], T.V[(m, k)]
            Bu, Bv = T.U[(n, k)], T.V[(n, k)]
            ra, rb = Au.shape[1], Bu.shape[1]
            rr = Av.T @ Bv
            if ra > rb:
                T.dense[(m, n)] = T.dense[(m, n)] - (Au @ rr) @ Bu.T
            else:
                T.dense[(m, n)] = T.dense[(m, n)] - Au @ (rr @ Bu.T)
            return [(op_counts("m", nb, nb, min(ra, rb), 0) + op_counts("m", nb, ra, rb, 0) * 2, m, n)]
        Au, Av = T.U[(m, k)], T.V[(m, k)]
        ra = Au.shape[1]
        rc_old = T.U[(m, n)].shape[1]
        if n - k < band:
            Y = T.dense[(n, k)] @ Av
            rb, bdense = 0, True
        else:
            Bu, Bv = T.U[(n, k)], T.V[(n, k)]
            rb, bdense = Bu.shape[1], False
            if ra == 0 or rb == 0:
                return []
            Y = Bu @ (Bv.T @ Av)
        U, V, r, ov = recompress(T.U[(m, n)], T.V[(m, n)], Au, Y, acc, T.maxrank, fixed_rank)
        T.U[(m, n)], T.V[(m, n)] = U, V
        with lock:
            st.overflow += int(ov)
            st.rank_min[m, n] = min(st.rank_min[m, n], r)
            st.rank_max[m, n] = max(st.rank_max[m, n], r)
        return [(gemm_lr_opcount(nb, ra, rb, rc_old, r, bdense), m, n)]

    # task graph: key -> (priority, body, successors), with in-degrees
    body, succ, indeg = {}, {}, {}

    def add(key, fn, deps):
        body[key] = fn
        succ.setdefault(key, [])
        indeg[key] = 0
        for d in deps:
            if d is not None:
                succ.setdefault(d, []).append(key)
                indeg[key] += 1

    last = {}     # tile -> last task that wrote it
    for k in range(nt):
        add(("P", k), (lambda k=k: potrf(k)), [last.get((k, k))])
        last[(k, k)] = ("P", k)
        for m in range(k + 1, nt):
            add(("T", m, k), (lambda m=m, k=k: trsm(m, k)), [("P", k), last.get((m, k))])
            last[(m, k)] = ("T", m, k)
        for m in range(k + 1, nt):
            add(("S", k, m), (lambda k=k, m=m: syrk(k, m)), [("T", m, k), last.get((m, m))])
            last[(m, m)] = ("S", k, m)
        for m in range(k + 2, nt):
            for n in range(k + 1, m):
                add(("G", m, n, k), (lambda m=m, n=n, k=k: gemm(m, n, k)),
                    [("T", m, k), ("T", n, k), last.get((m, n))])
                last[(m, n)] = ("G", m, n, k)
    order = {"P": 0, "T": 1, "S": 2, "G": 3}

    def prio(key):
        return (key[-1], order[key[0]], key)

    ready = [prio(k) for k, d in indeg.items() if d == 0]
    heapq.heapify(ready)
    cv = threading.Condition(lock)
    state = {"left": len(body), "error": None}

    def worker():
        while True:
            with cv:
                while not ready and state["left"] > 0 and state["error"] is None:
                    cv.wait()
                if state["left"] == 0 or state["error"] is not None:
                    cv.notify_all()
                    return
                key = heapq.heappop(ready)[2]
            try:
                with threadpool_limits(limits=1):
                    res = body[key]()
            except BaseException as e:   # noqa: BLE001 - surfaced to the caller below
                with cv:
                    state["error"] = e
                    cv.notify_all()
                return
            with cv:
                ops.extend(res)
                state["left"] -= 1
                for s2 in succ[key]:
                    indeg[s2] -= 1
                    if indeg[s2] == 0:
                        heapq.heappush(ready, prio(s2))
                cv.notify_all()

    ths = [threading.Thread(target=worker, daemon=True) for _ in range(max(1, threads))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    if state["error"] is not None:
        raise state["error"]
    for cnt, i, j in ops:
        st.tileopcounters[i, j] += np.uint64(cnt & _U64)
    return st


# --------------------------------------------------------------------------
# Checks, log-determinant, solve, likelihood
# --------------------------------------------------------------------------
def uncompress(T: TLRMatrix) -> np.ndarray:
    """Lower-triangular dense N x N matrix from the TLR storage
    (``STARSH_check.jdf:90-143``: band tiles copied, ``U V^T`` expanded)."""
    nb, nt = T.nb, T.nt
    D = np.zeros((T.n, T.n))
    for (m, n), t in T.dense.items():
        D[m * nb:(m + 1) * nb, n * nb:(n + 1) * nb] = t
    for (m, n), u in T.U.items():
        D[m * nb:(m + 1) * nb, n * nb:(n + 1) * nb] = u @ T.V[(m, n)].T
    return np.tril(D)


def sym_fro_lower(X: np.ndarray) -> float:
    """Frobenius norm of the symmetric matrix whose lower triangle is
    tril(X) (``dplasma_dlansy(Frobenius, Lower)``)."""
    L = np.tril(X)
    d = np.diag(L)
    off = L - np.diag(d)
    return math.sqrt(float(np.sum(d * d) + 2.0 * np.sum(off * off)))


def check_dpotrf2(L: np.ndarray, A: np.ndarray) -> float:
    """||L L^T - A||_F / ||A||_F as ``check_dpotrf2`` (``testing_dpotrf.c:111-180``)."""
    L = np.tril(L)
    return sym_fro_lower(L @ L.T - A) / sym_fro_lower(A)


def check_diff(L: np.ndarray, L0: np.ndarray) -> float:
    """||L - L0|| / ||L|| as ``check_diff`` (``testing_dpotrf.c:183-230``)."""
    return sym_fro_lower(np.tril(L) - np.tril(L0)) / sym_fro_lower(L)


def logdet(T: TLRMatrix) -> float:
    """log det(A) = 2 sum log L_ii over the diagonal tiles."""
    return float(sum(2.0 * np.sum(np.log(np.diag(T.dense[(k, k)]))) for k in range(T.nt)))


def solve(T: TLRMatrix, y: np.ndarray) -> np.ndarray:
    """x = A^{-1} y from the TLR factor: forward L z = y, backward L^T x = z."""
    nb, nt = T.nb, T.nt
    y = np.asarray(y, dtype=np.float64)
    squeeze = y.ndim == 1
    Y = y.reshape(T.n, -1).copy()

    def blk(i):
        return slice(i * nb, (i + 1) * nb)

    for k in range(nt):
        for j in range(k):
            if T.is_dense(k, j):
                Y[blk(k)] -= T.dense[(k, j)] @ Y[blk(j)]
            else:
                Y[blk(k)] -= T.U[(k, j)] @ (T.V[(k, j)].T @ Y[blk(j)])
        Y[blk(k)] = sla.solve_triangular(T.dense[(k, k)], Y[blk(k)], lower=True)
    for k in reversed(range(nt)):
        for m in range(k + 1, nt):
            if T.is_dense(m, k):
                Y[blk(k)] -= T.dense[(m, k)].T @ Y[blk(m)]
            else:
                Y[blk(k)] -= T.V[(m, k)] @ (T.U[(m, k)].T @ Y[blk(m)])
        Y[blk(k)] = sla.solve_triangular(T.dense[(k, k)], Y[blk(k)], lower=True, trans="T")
    return Y[:, 0] if squeeze else Y


def loglik(T: TLRMatrix, y: np.ndarray):
    """Gaussian log-likelihood -1/2 (y^T A^{-1} y + log det A + N log 2 pi);
    returns (loglik, logdet, x)."""
    x = solve(T, y)
    ld = logdet(T)
    q = float(np.dot(np.asarray(y).ravel(), x.ravel()))
    return -0.5 * (q + ld + T.n * math.log(2.0 * math.pi)), ld, x
