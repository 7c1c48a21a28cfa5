"""The C ABI used from C, the reference's own language: a small program is
compiled with gcc against include/hicma_tlr.h, linked with the library, and
calls the entry points that need no GPU (point generation of a statistics
problem and of the md-3d-cube mesh problem, rank statistics,
band auto-tuning, the op-count model, argument errors); its output is compared
with the CPU oracle.  This is the shape of the binding a maintainer adds to
the reference's driver."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import tlr_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "hicma_tlr.h"

int main(void) {
    hicma_tlr_problem prob = {HICMA_TLR_KIND_SQEXP_2D, 0.1, 0.5, 1e-4, 1.0, 0, 50.0, 0.0};
    enum { N = 100, NT = 6 };
    double pts[2 * N];
    if (hicma_tlr_points(&prob, N, pts) != 0) return 1;
    for (int i = 0; i < 2 * N; ++i) printf("p %.17g\n", pts[i]);
    int G[NT * NT];
    for (int n = 0; n < NT; ++n)
        for (int m = 0; m < NT; ++m) G[n * NT + m] = m > n ? (7 * m + 3 * n) % 40 : -1;
    int mn = 0, mx = 0; double av = 0;
    if (hicma_tlr_rank_stat(G, NT, 1, &mn, &mx, &av) != 0) return 2;
    printf("stat %d %d %.17g\n", mn, mx, av);
    printf("band %d\n", hicma_tlr_band_autotune(G, NT, 270, 0));
    printf("q %lu\n", hicma_tlr_op_counts('q', 2700, 150, 0, 0));
    printf("o %lu\n", hicma_tlr_op_counts('o', 2700, 75, 150, 2));
    /* md-3d-cube nodes (an RBF mesh problem), C99 designated initializers */
    hicma_tlr_problem cube = {.kind = HICMA_TLR_KIND_MD_CUBE, .rbf_kernel = HICMA_TLR_RBF_WENDLAND,
                              .radius = 0.3, .numobj = 1, .order = 1};
    double cpts[3 * 27];
    if (hicma_tlr_points(&cube, 27, cpts) != 0) return 3;
    for (int i = 0; i < 3 * 27; ++i) printf("c %.17g\n", cpts[i]);
    prob.kind = 9;   /* no such problem kind */
    printf("err %d\n", hicma_tlr_points(&prob, N, pts));
    printf("msg %s\n", hicma_tlr_last_error());
    return 0;
}
"""


def test_c_program_against_oracle(tmp_path):
    from hicma_parsec_b200 import build
    if not os.path.exists(build.LIB) or shutil.which("gcc") is None:
        pytest.skip("library or C compiler missing")
    src = tmp_path / "consumer.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "consumer"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", build.LIBDIR, "-lhicma_tlr", f"-Wl,-rpath,{build.LIBDIR}"],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=60).stdout.splitlines()
    pts = np.array([float(l.split()[1]) for l in out if l.startswith("p ")]).reshape(2, 100)
    np.testing.assert_array_equal(pts.T, O.gen_points(100, 2, 0))
    G = np.full(36, -1, dtype=np.int64)
    for n in range(6):
        for m in range(n + 1, 6):
            G[n * 6 + m] = (7 * m + 3 * n) % 40
    cube = np.array([float(l.split()[1]) for l in out if l.startswith("c ")]).reshape(3, 27)
    np.testing.assert_array_equal(cube.T, O.cube_points(27, 1))
    kv = {l.split()[0]: l.split()[1:] for l in out if not l.startswith(("p ", "c "))}
    mn, mx, av = O.rank_stat(G, 6, 1)
    assert (int(kv["stat"][0]), int(kv["stat"][1])) == (mn, mx) and float(kv["stat"][2]) == pytest.approx(av)
    assert int(kv["band"][0]) == O.band_autotune(G, 6, 270)
    assert int(kv["q"][0]) == O.op_counts("q", 2700, 150, 0, 0)
    assert int(kv["o"][0]) == O.op_counts("o", 2700, 75, 150, 2)
    assert int(kv["err"][0]) == -1 and "kind" in " ".join(kv["msg"])
