"""RBF mesh-deformation problems on the GPU against the oracle: md-3d-cube
(``-D 7``) and md-3d-virus (``-D 6``), hicma_parsec/testing_dpotrf.c:366-381.

A_ij = phi(|x_i - x_j| / radius) plus add_diag (default N) where i == j, phi
one of the nine basis functions of ``-B`` (hicma_parsec/hicma_parsec.c:80).
Bars: tile entries within 1e-12 absolute of the oracle (CUDA's exp/log/sqrt
against the host libm; off-diagonal entries are at most 1 in size);
generation ranks within +/-3 of the oracle's exact-SVD ranks; residual
||A - L L^T||_F / ||A||_F <= 10 e and log-determinant within 10 e relative of
a dense FP64 Cholesky.  The mesh of ``-D 6`` is a spiked sphere written by
the test (the reference's virus meshes are not shipped with it).
"""
import numpy as np
import pytest

from oracle import tlr_oracle as O
from test_mesh_kinds_host import fib_sphere, write_mesh

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N, NB, MAXRANK = 2700, 270, 130


@pytest.mark.parametrize("rbf", range(9))
def test_cube_tiles_match_oracle(rbf):
    from hicma_parsec_b200 import tlr
    rad = 2.0 if rbf == tlr.RBF_TPS else 0.1
    prob = tlr.Problem(kind=tlr.KIND_MD_CUBE, rbf_kernel=rbf, radius=rad)
    P = tlr.points(prob, N)
    dP = torch.from_numpy(P).cuda()
    pts = P.T.copy()
    oprob = O.Problem(kind=O.KIND_MD_CUBE, rbf_kernel=rbf, radius=rad)
    st = torch.cuda.current_stream().cuda_stream
    for (m, c) in [(0, 0), (3, 1), (9, 0), (5, 5)]:
        out = torch.zeros((NB, NB), dtype=torch.float64, device="cuda")
        rc = tlr.load_library().hicma_tlr_k_cov(prob.c(), dP.data_ptr(), N, m * NB, NB, c * NB, NB,
                                               out.data_ptr(), NB, st)
        assert rc == 0, tlr.last_error()
        got = out.cpu().numpy().T
        ref = O.cov_block(oprob, pts, m * NB, NB, c * NB, NB)
        assert np.max(np.abs(got - ref)) <= 1e-12, (m, c)


def _factor_against_oracle(ctx, prob, oprob, pts, tol, band, pts_arg=None):
    from hicma_parsec_b200 import tlr
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, band)
    try:
        assert A.generate(prob, tol, MAXRANK, pts_arg) == 0
        T, info = O.generate(oprob, N, NB, tol, MAXRANK, band, pts)
        assert info == 0
        G0, Gref = A.rank_map(), T.rank_array()
        off = Gref >= 0
        assert np.max(np.abs(G0[off] - Gref[off])) <= 3
        assert A.potrf(tol) == 0
        Aexact = O.dense_matrix(oprob, pts)
        res = O.check_dpotrf2(A.uncompress(), Aexact)
        assert res <= 10 * tol, res
        ld_exact = 2.0 * np.sum(np.log(np.diag(np.linalg.cholesky(Aexact))))
        assert abs(A.logdet() - ld_exact) / abs(ld_exact) <= 10 * tol
    finally:
        A.close()


@pytest.mark.parametrize("rbf,rad,tol,band", [(8, 0.1, 1e-8, 1), (0, 0.1, 1e-4, 2), (3, 0.1, 1e-6, 2)])
def test_cube_factorization_matches_oracle(ctx, rbf, rad, tol, band):
    from hicma_parsec_b200 import tlr
    prob = tlr.Problem(kind=tlr.KIND_MD_CUBE, rbf_kernel=rbf, radius=rad)
    oprob = O.Problem(kind=O.KIND_MD_CUBE, rbf_kernel=rbf, radius=rad)
    _factor_against_oracle(ctx, prob, oprob, O.cube_points(N, 1), tol, band)


@pytest.mark.parametrize("density,rbf,rad,tol", [(0.3, 8, 0.5, 1e-8), (-1.0, 8, 0.5, 1e-8), (0.3, 0, 0.3, 1e-6)])
def test_virus_factorization_matches_oracle(ctx, tmp_path, density, rbf, rad, tol):
    from hicma_parsec_b200 import tlr
    path = write_mesh(tmp_path / "virus.xyz", fib_sphere(675, spikes=40))
    kw = dict(rbf_kernel=rbf, radius=rad, numobj=4, density=density, seed=1)
    prob = tlr.Problem(kind=tlr.KIND_MD_VIRUS, **kw)
    oprob = O.Problem(kind=O.KIND_MD_VIRUS, **kw)
    P = tlr.points_mesh(prob, path, N)
    pts = O.virus_points(O.read_mesh(path), N, oprob)
    assert np.array_equal(P.T, pts)
    _factor_against_oracle(ctx, prob, oprob, pts, tol, 1, pts_arg=P)


def test_virus_without_points_is_an_argument_error(ctx):
    from hicma_parsec_b200 import tlr
    A = tlr.TLRMatrix(ctx, N, NB, MAXRANK, 1)
    try:
        with pytest.raises(tlr.TLRError):
            A.generate(tlr.Problem(kind=tlr.KIND_MD_VIRUS, radius=0.5), 1e-8, MAXRANK)
    finally:
        A.close()


@pytest.mark.parametrize("kind", [6, 7])
def test_cli_mesh_kinds(tmp_path, kind):
    """The driver with the reference's RBF flags (-D 6/7 -B -R -O -K -S -M):
    factors and checks, and the R-LO record carries the five RBF fields
    (testing_dpotrf.c:1044-1047)."""
    import subprocess
    from hicma_parsec_b200 import build, ranklog
    args = [build.CLI, "-N", "2700", "-t", "270", "-e", "1e-8", "-u", "130", "-D", str(kind), "-B", "8",
            "-R", "0.1" if kind == 7 else "0.5", "-O", "1", "-E", "0", "-Z", "1", "-v", "--check"]
    if kind == 6:
        args += ["-M", write_mesh(tmp_path / "virus.xyz", fib_sphere(675, spikes=40)), "-K", "4", "-S", "0.3"]
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-2000:])
    assert "Factorization is CORRECT" in r.stdout
    rec = ranklog.parse_log(r.stdout).records[0]
    assert rec["kind"] == kind and rec["problem"] == ("md-3d-virus" if kind == 6 else "md-3d-cube")
    assert (rec["order"], rec["rbf_kernel"]) == (1, 8)
    assert rec["numobj"] == (4 if kind == 6 else 1)
