"""The testing_dpotrf_tlr driver's argument handling, which runs before any
GPU call (options of hicma_parsec/hicma_parsec.c:89-309): usage text, problem
kind range, required sizes.  CPU only."""
import os
import subprocess

import pytest


@pytest.fixture(scope="module")
def cli():
    from hicma_parsec_b200 import build
    if not os.path.exists(build.CLI):
        pytest.skip("driver not built")
    return build.CLI


def run(cli, *args):
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=60)


def test_usage_lists_problem_kinds(cli):
    r = run(cli, "-h")
    assert r.returncode == 0
    for name in ("randtlr", "ed-2d-sin", "st-2d-sqexp", "st-3d-sqexp", "st-3d-exp", "ed-3d-sin", "md-3d-virus",
                 "md-3d-cube"):
        assert name in r.stderr
    assert "--wavek" in r.stderr and "--adddiag" in r.stderr
    for flag in ("--mesh_file", "--numobj", "--rbf_kernel", "--radius", "--order", "--density"):
        assert flag in r.stderr


@pytest.mark.parametrize("kind", ["8", "-1"])
def test_unsupported_kind_is_rejected_before_gpu_use(cli, kind):
    r = run(cli, "-N", "2700", "-t", "270", "-D", kind)
    assert r.returncode == 1
    assert "kind_of_problem" in r.stderr


@pytest.mark.parametrize("args,msg", [(["-D", "6", "-R", "0.5"], "mesh file"), (["-D", "7"], "radius"),
                                      (["-D", "6", "-M", "m.xyz"], "radius")])
def test_mesh_kind_arguments_checked_before_gpu_use(cli, args, msg):
    r = run(cli, "-N", "2700", "-t", "270", *args)
    assert r.returncode == 1
    assert msg in r.stderr


def test_sizes_are_required(cli):
    r = run(cli, "-e", "1e-8")
    assert r.returncode == 1
    assert "NB" in r.stderr


def test_n_must_be_a_multiple_of_nb(cli):
    r = run(cli, "-N", "2701", "-t", "270", "-D", "2")
    assert r.returncode == 1
    assert "multiple" in r.stderr


def test_reference_option_spellings_parse(cli):
    """The reference driver's long options (hicma_parsec/hicma_parsec.c:89-161),
    including the RBF mesh flags, parse; the run then stops at a kind that does
    not exist (8) before any GPU use."""
    r = run(cli, "--N", "2700", "--NB", "270", "--fixedacc", "1e-8", "--maxrank", "130", "--wavek", "25",
            "--adddiag", "3000", "--grid-rows", "1", "--grid-cols", "1", "--rbf_kernel", "0", "--numobj", "1",
            "--mesh_file", "x", "--order", "1", "--radius", "0.5", "--density", "0.1", "--kind_of_problem", "8")
    assert r.returncode == 1
    assert "kind_of_problem" in r.stderr and "unrecognized" not in r.stderr
