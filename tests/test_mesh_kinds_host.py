"""RBF mesh-deformation problems (``-D 6`` md-3d-virus, ``-D 7`` md-3d-cube;
hicma_parsec/testing_dpotrf.c:366-381) on the host: the library's point
generators against the oracle (bit for bit), the argument checks, and the
oracle's own properties (every basis function with the add_diag
regularisation gives an SPD matrix whose TLR factor meets the reference
check).  STARS-H's mesh generators are absent from the reference tree, so the
point rules are the restatement's own (documented in include/hicma_tlr.h)."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import tlr_oracle as O


def fib_sphere(m: int, spikes: int = 0) -> np.ndarray:
    """m nodes on the unit sphere (Fibonacci lattice); every (m // spikes)-th
    node pushed out to radius 1.3 (a virus-like surface with spikes)."""
    i = np.arange(m, dtype=np.float64) + 0.5
    z = 1.0 - 2.0 * i / m
    r = np.sqrt(1.0 - z * z)
    phi = math.pi * (3.0 - math.sqrt(5.0)) * i
    P = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    if spikes:
        P[:: max(1, m // spikes)] *= 1.3
    return P


def write_mesh(path, P: np.ndarray) -> str:
    with open(path, "w") as f:
        f.write("# test mesh: x y z per node\n")
        for x, y, z in P:
            f.write(f"{float(x)!r} {float(y)!r} {float(z)!r}\n")
    return str(path)


@pytest.fixture(scope="module")
def tlr():
    from hicma_parsec_b200 import tlr as T
    T.load_library()
    return T


@pytest.mark.parametrize("n,order", [(1, 1), (27, 1), (1000, 0), (2700, 1), (3001, 1)])
def test_cube_points_bit_identical(tlr, n, order):
    P = tlr.points(tlr.Problem(kind=tlr.KIND_MD_CUBE, radius=0.3, order=order), n)
    Q = O.cube_points(n, order)
    assert P.shape == (3, n)
    assert np.array_equal(P.T, Q)
    assert np.all((Q > 0.0) & (Q < 1.0))
    assert len({tuple(q) for q in Q}) == n


@pytest.mark.parametrize("numobj,density,order", [(1, -1.0, 1), (4, 0.3, 1), (8, -1.0, 1), (5, 0.6, 0)])
def test_mesh_points_bit_identical(tlr, tmp_path, numobj, density, order):
    mesh = fib_sphere(300, spikes=20)
    path = write_mesh(tmp_path / "virus.xyz", mesh)
    n = numobj * 300 - 7
    prob = tlr.Problem(kind=tlr.KIND_MD_VIRUS, radius=0.5, numobj=numobj, density=density, order=order, seed=3)
    P = tlr.points_mesh(prob, path, n)
    oprob = O.Problem(kind=O.KIND_MD_VIRUS, radius=0.5, numobj=numobj, density=density, order=order, seed=3)
    Q = O.virus_points(O.read_mesh(path), n, oprob)
    assert np.array_equal(P.T, Q)
    if density > 0:
        # lattice placement: copies of diameter d at spacing >= d never overlap
        assert len({tuple(q) for q in Q}) == n


def test_mesh_argument_errors(tlr, tmp_path):
    path = write_mesh(tmp_path / "m.xyz", fib_sphere(50))
    bad = tmp_path / "bad.xyz"
    bad.write_text("0 1\n")
    ok = dict(kind=tlr.KIND_MD_VIRUS, radius=0.5, numobj=2)
    with pytest.raises(tlr.TLRError):
        tlr.points_mesh(tlr.Problem(**ok), path, 101)                 # N > numobj * nodes
    with pytest.raises(tlr.TLRError):
        tlr.points_mesh(tlr.Problem(**ok), str(bad), 1)               # not x y z triples
    with pytest.raises(tlr.TLRError):
        tlr.points_mesh(tlr.Problem(**ok), str(tmp_path / "none"), 1)  # no file
    with pytest.raises(tlr.TLRError):
        tlr.points_mesh(tlr.Problem(**{**ok, "radius": 0.0}), path, 10)
    with pytest.raises(tlr.TLRError):
        tlr.points_mesh(tlr.Problem(**{**ok, "rbf_kernel": 9}), path, 10)
    with pytest.raises(tlr.TLRError):
        tlr.points_mesh(tlr.Problem(**{**ok, "order": 2}), path, 10)   # Hilbert: not in STARS-H
    with pytest.raises(tlr.TLRError):
        tlr.points_mesh(tlr.Problem(kind=tlr.KIND_MD_CUBE, radius=0.5), path, 10)
    assert tlr.points_mesh(tlr.Problem(**ok), path, 100).shape == (3, 100)


def test_mesh_file_format(tlr, tmp_path):
    """The reader takes x y z triples in any line layout (here every node on
    one line of about 20 KB, with comments and CRLF endings) and refuses
    tokens that are not finite numbers."""
    mesh = fib_sphere(500)
    one = tmp_path / "one_line.xyz"
    one.write_text("# header\r\n" + " ".join(repr(float(v)) for v in mesh.ravel()) + "  # tail\r\n")
    prob = tlr.Problem(kind=tlr.KIND_MD_VIRUS, radius=0.5, numobj=2, density=0.3)
    P = tlr.points_mesh(prob, str(one), 1000)
    Q = O.virus_points(O.read_mesh(str(one)), 1000, O.Problem(kind=O.KIND_MD_VIRUS, radius=0.5, numobj=2,
                                                                density=0.3))
    assert np.array_equal(P.T, Q)
    for bad in ("0 0 0\n1 abc 2\n", "0 0 0\n1 nan 2\n", "0 0 0\ninf 1 2\n"):
        f = tmp_path / "bad.xyz"
        f.write_text(bad)
        with pytest.raises(tlr.TLRError):
            tlr.points_mesh(prob, str(f), 2)
        with pytest.raises(ValueError):
            O.read_mesh(str(f))


def test_rbf_functions():
    s = np.array([0.0, 0.25, 0.5, 1.0, 2.0])
    e = np.exp(-s)
    want = {
        O.RBF_GAUSSIAN: np.exp(-s * s), O.RBF_EXPON: e, O.RBF_INVQUAD: 1 / (1 + s * s),
        O.RBF_INVMQUAD: 1 / np.sqrt(1 + s * s), O.RBF_MATERNC1: (1 + s) * e,
        O.RBF_MATERNC2: (1 + s + s * s / 3) * e,
        O.RBF_TPS: np.array([0.0] + [x * x * math.log(x) for x in s[1:]]),
        O.RBF_CTPS: np.where(s < 1, (1 - s) ** 5, 0.0), O.RBF_WENDLAND: np.where(s < 1, (1 - s) ** 4 * (4 * s + 1), 0.0),
    }
    for f, w in want.items():
        assert np.allclose(O.rbf_phi(f, s), w, rtol=1e-15, atol=0), f


@pytest.mark.parametrize("rbf", range(9))
def test_cube_every_rbf_factors(rbf):
    """md-3d-cube, every basis function, radius 0.1, add_diag = N: SPD, and the
    TLR factor of the oracle meets the reference check.  The 2700 nodes fill
    the cube densely, so neighbouring tiles compress only at a loose accuracy:
    e = 1e-4 with a band of 2 (at e = 1e-8 and band 1 the generator rejects
    tiles of the infinitely supported functions, as the reference would).  The
    thin-plate spline is only conditionally definite: at radius 2 its entries
    lie in [-0.19, 0] and add_diag = N keeps the matrix SPD."""
    n, nb, tol = 2700, 270, 1e-4
    prob = O.Problem(kind=O.KIND_MD_CUBE, rbf_kernel=rbf, radius=2.0 if rbf == O.RBF_TPS else 0.1)
    pts = O.problem_points(prob, n, nb)
    A = O.dense_matrix(prob, pts)
    assert np.allclose(A, A.T) and np.all(np.diag(A) == n + O.rbf_phi(rbf, np.zeros(1))[0])
    assert np.linalg.eigvalsh(A)[0] > 0
    T, info = O.generate(prob, n, nb, tol, 130, 2, pts)
    assert info == 0
    assert O.tlr_potrf(T, tol).info == 0
    assert O.check_dpotrf2(O.uncompress(T), A) <= 10 * tol


def test_range_finder_orthogonality_check():
    """Why generation checks the range finder's Q: on a sparse md-3d-cube tile
    (Wendland, radius 0.1: each node couples only to its grid neighbours) the
    64-column sample Y = A Omega has exactly the tile's low rank, and the
    randomized CholeskyQR (the oracle's restatement of the device kernel)
    returns a Q far from orthonormal; on the statistics tiles ||Q^T Q - I||
    stays near 1e-14.  The device compresses a tile again on the Householder
    path when the check exceeds 1e-10."""
    import scipy.linalg as sla

    def orth(A):
        Y, Rc, _, _ = O.qr_rcholqr(A @ O.gaussian_counter(7, A.shape[1], 64))
        Q = sla.solve_triangular(Rc, Y.T, trans="T", lower=False).T
        G = Q.T @ Q
        nz = np.diag(G) != 0
        return np.abs((G - np.eye(64))[np.ix_(nz, nz)]).max()

    n, nb = 2700, 270
    rbf = O.Problem(kind=O.KIND_MD_CUBE, rbf_kernel=O.RBF_WENDLAND, radius=0.1)
    pts = O.cube_points(n, 1)
    assert orth(O.cov_block(rbf, pts, 5 * nb, nb, 4 * nb, nb)) > 1e-10
    st = O.Problem(kind=O.KIND_SQEXP_2D, noise=1e-4)
    spts = O.gen_points(n, 2)
    assert orth(O.cov_block(st, spts, 5 * nb, nb, 4 * nb, nb)) < 1e-12
