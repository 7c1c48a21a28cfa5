"""The bounds-checked build on the GPU: generation, band auto-tuning and
regeneration, factorization, log-likelihood, the matrix-free check and the
kernel-level POTRF run through libhicma_tlr_checked.so (every batched launch
validated on the host first) without a refused launch, and give the same
numbers as the default build (same kernels in the same order, so the values
are expected to agree bit for bit; bar 1e-12 relative)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
import numpy as np
import torch
from hicma_parsec_b200 import tlr
lib = tlr.load_library()
ctx = tlr.Context(0, 1 << 30)
out = {"checked": lib.hicma_tlr_bounds_checked()}
for kind, n, nb, mr in ((2, 2700, 270, 130), (4, 8000, 1000, 499), (0, 2700, 270, 130)):
    prob = tlr.Problem(kind=kind, noise=1e-4)
    A = tlr.TLRMatrix(ctx, n, nb, mr, 1)
    assert A.generate(prob, 1e-8, mr) == 0
    b = tlr.parsec_band_size_auto_tuning(A.rank_map(), n // nb, nb)
    if b > 1:
        A.band_regenerate(prob, b)
    assert A.potrf(1e-8, mr) == 0
    ll, ld, x = A.loglik(np.random.default_rng(3).standard_normal(n))
    out[str(kind)] = {"ll": ll, "ld": ld, "probe": A.check_probe(prob, 4, 0), "band": A.band_size}
    A.close()
rng = np.random.default_rng(1)
M = rng.standard_normal((300, 300))
S = M @ M.T + 300 * np.eye(300)
dA = torch.from_numpy(S.copy()).cuda()
dL = torch.zeros((300, 300), dtype=torch.float64, device="cuda")
info = torch.zeros(1, dtype=torch.int32, device="cuda")
rc = lib.hicma_tlr_k_potrf(ctx.h, 300, dA.data_ptr(), 300, dL.data_ptr(), info.data_ptr(), 0)
out["k_potrf"] = [rc, int(info.item()), float(np.abs(np.triu(dA.cpu().numpy()).T - np.linalg.cholesky(S)).max())]
ctx.close()
print(json.dumps(out))
"""


def run(env):
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, capture_output=True, text=True, timeout=600,
                       env={**os.environ, "HICMA_TLR_LIB": env})
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_checked_build_runs_the_paths_and_agrees():
    plain, checked = run(""), run("checked")
    assert plain["checked"] == 0 and checked["checked"] == 1
    for kind in ("2", "4", "0"):
        a, b = plain[kind], checked[kind]
        assert a["band"] == b["band"]
        for key in ("ll", "ld", "probe"):
            assert abs(a[key] - b[key]) <= 1e-12 * abs(a[key]), (kind, key)
    assert checked["k_potrf"][0] == 0 and checked["k_potrf"][1] == 0 and checked["k_potrf"][2] < 1e-10
