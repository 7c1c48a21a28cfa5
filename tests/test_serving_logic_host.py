"""serving.solve_request's decisions on the CPU, with a stand-in matrix class:
rejected tiles widen the dense band to cover them (band_regenerate.jdf), an
accepted generation goes through the band auto-tuning, a factorization that
is not positive definite returns its info, and a library error becomes the
request's status.  The same rules are in hicma_tlr_serve_loglik."""
import numpy as np
import pytest

from hicma_parsec_b200 import serving, tlr


class FakeMatrix:
    script = {}
    calls = []

    def __init__(self, ctx, n, nb, maxrank, band):
        self.n, self.nb, self.nt, self._band = n, nb, n // nb, band
        self.s = FakeMatrix.script

    def generate(self, prob, acc, maxrank):
        if self.s.get("raise"):
            raise tlr.TLRError(tlr.ERR_OOM, "hicma_tlr_generate", "out of memory")
        return -1 if self.s.get("rejected") else 0

    def rank_map(self):
        nt = self.nt
        G = np.full(nt * nt, -1, dtype=np.int32)
        for n in range(nt):
            for m in range(n + 1, nt):
                G[n * nt + m] = self.s.get("rank", 10)
        return G

    def rejected_tiles(self):
        return self.s.get("rejected", [])

    def band_regenerate(self, prob, band):
        FakeMatrix.calls.append(("band", band))
        self._band = band

    @property
    def band_size(self):
        return self._band

    def potrf(self, acc, maxrank):
        return self.s.get("info", 0)

    def loglik(self, y):
        return -1.0, 2.0, np.zeros_like(y)

    def stats(self):
        return np.zeros(12)

    def close(self):
        FakeMatrix.calls.append(("close",))


def req(**kw):
    base = dict(rid=0, kind=2, n=8000, nb=1000, beta=0.1, sigma=1.0, noise=1e-3, acc=1e-8, seed=1)
    base.update(kw)
    return serving.MLERequest(**base)


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(serving.tlr, "TLRMatrix", FakeMatrix)
    FakeMatrix.calls = []
    yield FakeMatrix


def test_rejected_tiles_widen_the_band(fake):
    fake.script = {"rejected": [(5, 2), (6, 4), (3, 2)]}
    r = serving.solve_request(None, req())
    assert r.status == 0 and ("band", 4) in fake.calls and r.band == 4     # max(m - n) + 1 = 4
    assert fake.calls[-1] == ("close",)


def test_accepted_generation_uses_the_auto_band(fake):
    fake.script = {"rank": 400}
    G = FakeMatrix(None, 8000, 1000, 499, 1).rank_map()
    b = tlr.parsec_band_size_auto_tuning(G, 8, 1000)
    r = serving.solve_request(None, req(maxrank=499))
    assert r.status == 0 and r.band == (b if b > 1 else 1)
    assert (("band", b) in fake.calls) == (b > 1)
    fake.calls.clear()
    serving.solve_request(None, req(autoband=False))
    assert not [c for c in fake.calls if c[0] == "band"]


def test_not_positive_definite_and_library_errors(fake):
    fake.script = {"info": 1234}
    r = serving.solve_request(None, req())
    assert r.status == 1234 and "positive definite" in r.error and fake.calls[-1] == ("close",)
    fake.script = {"raise": True}
    r = serving.solve_request(None, req())
    assert r.status == tlr.ERR_OOM and "out of memory" in r.error


def test_mle_evaluator_decisions(monkeypatch):
    """mle.device_loglik: the same band rules, -inf for a factorization that is
    not positive definite, and the matrix released every time."""
    from hicma_parsec_b200 import mle
    monkeypatch.setattr(mle.tlr, "TLRMatrix", FakeMatrix)
    FakeMatrix.calls = []
    y = np.zeros(8000)
    ev = mle.device_loglik(None, 2, 8000, 1000, y, 1e-8, 499, seed=3, autoband=False)
    FakeMatrix.script = {"rejected": [(7, 1)]}
    assert ev(0.1, 1.0, 1e-3) == -1.0 and ("band", 7) in FakeMatrix.calls
    FakeMatrix.script = {"info": 5}
    assert ev(0.1, 1.0, 1e-3) == -np.inf
    assert sum(1 for c in FakeMatrix.calls if c == ("close",)) == 2
