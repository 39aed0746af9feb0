"""The drop-in end to end: the reference's own force benchmark
(benchmarks/benchmark_force.c) with the `cuda` and `barnes_hut_cuda` arms added
to its algorithm chain (oracle/benchmark_cuda_arms.sed), linked against the
reference engine and libn_body_sim_pro_cuda.so, selects and runs the two new
algorithms through the reference's plugin signature (integrator.h:47-49).
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "oracle", "_ref", "n_body_sim_pro_benchmark_cuda")
PATCHED = os.path.join(ROOT, "oracle", "_ref", "build", "benchmark_force_cuda.c")

needs_binary = pytest.mark.skipif(not os.path.exists(BINARY),
                                  reason="integrated benchmark not built (needs the reference "
                                         "sources at build time)")


def run(*args):
    return subprocess.run([BINARY, *args], capture_output=True, text=True, timeout=300)


@pytest.mark.skipif(not os.path.exists(PATCHED), reason="integrated benchmark not built")
def test_arms_added_to_the_reference_chain():
    src = open(PATCHED).read()
    assert src.count('strcmp(algorithm, "cuda") == 0') == 2
    assert src.count('strcmp(algorithm, "barnes_hut_cuda") == 0') == 2
    assert src.count("n_body_sim_pro_cuda_context_destroy(cuda);") == 2
    assert "n_body_sim_pro_barnes_hut_compute_acceleration_cuda(view, gravity, cuda" in src
    assert "n_body_sim_pro_gravity_compute_acceleration_cuda(view, gravity, cuda" in src


@needs_binary
@pytest.mark.gpu
@pytest.mark.parametrize("algorithm", ["cuda", "barnes_hut_cuda"])
def test_reference_benchmark_runs_the_cuda_algorithms(algorithm):
    r = run("--particles", "20000", "--steps", "3", "--algorithm", algorithm, "--theta", "0.7")
    assert r.returncode == 0, r.stderr
    assert f"algorithm={algorithm}" in r.stdout
    ms = float(re.search(r"ms/evaluation=([0-9.]+)", r.stdout).group(1))
    assert ms > 0.0
    print(r.stdout)


@needs_binary
@pytest.mark.gpu
def test_reference_benchmark_still_runs_its_own_algorithms():
    r = run("--particles", "20000", "--steps", "1", "--algorithm", "barnes_hut")
    assert r.returncode == 0, r.stderr
    assert "algorithm=barnes_hut" in r.stdout


@needs_binary
def test_unknown_algorithm_fails_like_the_reference():
    r = run("--particles", "1000", "--steps", "1", "--algorithm", "cuda_nonexistent")
    assert r.returncode == 1
    assert "force evaluation failed" in r.stderr
