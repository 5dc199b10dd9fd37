"""CPU tests of bench.py's algorithmic work counts (the numerators of its
roofline figures) against the per-step totals of the headline workload
(lmax = 255, nlat = 384, nr = 129): Legendre contractions 58 nlm nlat nr
flops per step (4 vector + 1 four-field scalar syntheses, 2 vector + 1 scalar
analyses, each counted once), CNAB2 5 fields x (read u, N, N_prev; write u)
= 1.36 GB, and the exponential schemes' matrix-vector products."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


@pytest.fixture(scope="module")
def headline():
    p = bench.workload_params()
    nlm = (p["lmax"] + 1) * (p["lmax"] + 2) // 2
    return p, nlm


def test_legendre_flops_per_step(headline):
    p, nlm = headline
    per_step = {"legendre_synth_vector_tc": 4, "legendre_synth_scalar_tc": 1,
                "legendre_analysis_vector_tc": 2, "legendre_analysis_scalar_tc": 1}
    total = sum(bench.kernel_work(k, p, nlm, "mixed")["flops"] * n for k, n in per_step.items())
    assert total == 58.0 * nlm * p["nlat"] * p["nr"]
    assert abs(total - 94.5e9) < 0.05e9
    # the FP64 step counts the same algorithmic flops
    total64 = sum(bench.kernel_work(k.replace("_tc", "_fp64"), p, nlm, "fp64")["flops"] * n
                  for k, n in per_step.items())
    assert total64 == total


def test_cnab2_bytes(headline):
    p, nlm = headline
    b = bench.kernel_work("cnab2_solve", p, nlm, "mixed")["bytes"]
    assert b == 5 * 4 * (2 * p["nr"] * nlm) * 8
    assert abs(b - 1.36e9) < 0.01e9


def test_exponential_scheme_flops(headline):
    p, nlm = headline
    n, cols = p["nr"], 5 * 2 * nlm   # columns over the five fields, both planes
    assert bench.kernel_work("eab2_update", p, nlm, "mixed")["flops"] == cols * n * 2 * n * 2
    assert bench.kernel_work("erk2_prepare", p, nlm, "mixed")["flops"] == cols * n * 4 * n * 2
    assert bench.kernel_work("erk2_finalize", p, nlm, "mixed")["flops"] == cols * n * n * 2


def test_reference_arm_other_ranks_exit_quietly():
    # under torchrun only rank 0 runs and prints the reference arm's line
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
