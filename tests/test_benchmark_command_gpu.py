"""The reference's `benchmark` command with the two new algorithms.

The reference's own command line (src/main.cpp), its headless runner
(src/cpp/benchmark/HeadlessRunner.cpp) and its simulation controller
(src/cpp/simulation/SimulationController.cpp) are compiled from build copies
with the `cuda` and `barnes_hut_cuda` arms added by oracle/benchmark_command/*.sed
(main.cpp:120-134 --algorithm, HeadlessRunner.hpp:19-28 options,
SimulationController.cpp:81-122 force selection), linked against the reference
engine and libn_body_sim_pro_cuda.so.  Here the `benchmark` command runs both
algorithms and its JSON report (HeadlessRunner.cpp:154-164) is checked, and the
controller's steps with each algorithm are compared with the CPU oracle.
"""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
CLI = os.path.join(REF_DIR, "n_body_sim_pro_cuda_cli")
STEPS_DRIVER = os.path.join(REF_DIR, "controller_steps")
PATCHED = os.path.join(REF_DIR, "build", "cmd")

needs_cli = pytest.mark.skipif(not os.path.exists(CLI),
                               reason="headless CLI not built (needs the reference sources "
                                      "at build time)")


@pytest.mark.skipif(not os.path.isdir(PATCHED), reason="headless CLI not built")
def test_arms_added_to_the_reference_command_path():
    main = open(os.path.join(PATCHED, "main.cpp")).read()
    assert 'std::strcmp(value, "cuda") == 0' in main
    assert 'std::strcmp(value, "barnes_hut_cuda") == 0' in main
    assert "Application" not in main.split("int main(")[0]
    ctrl = open(os.path.join(PATCHED, "simulation", "SimulationController.cpp")).read()
    assert "n_body_sim_pro_barnes_hut_compute_acceleration_cuda" in ctrl
    assert "n_body_sim_pro_gravity_compute_acceleration_cuda" in ctrl
    opts = open(os.path.join(PATCHED, "benchmark", "HeadlessRunner.hpp")).read()
    assert "bool cuda = false;" in opts


def _machine_readable(stdout: str) -> dict:
    lines = stdout.splitlines()
    k = lines.index("--- machine-readable ---")
    return json.loads(lines[k + 1])


@needs_cli
@pytest.mark.gpu
@pytest.mark.parametrize("algorithm,n", [("cuda", 8192), ("barnes_hut_cuda", 20000)])
def test_benchmark_command_runs_the_cuda_algorithms(algorithm, n):
    r = subprocess.run([CLI, "benchmark", "--algorithm", algorithm, "--particles", str(n),
                        "--steps", "3", "--preset", "globular_cluster", "--theta", "0.5"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    report = _machine_readable(r.stdout)
    assert report["algorithm"] == algorithm
    assert report["particles"] == n and report["steps"] == 3
    assert report["avg_step_ms"] > 0.0 and report["first_step_ms"] > 0.0
    # N <= 20000: the controller tracks the energy (SimulationController.hpp:107);
    # its softening is the controller's default 0, so close pairs are unsoftened
    assert report["energy_drift"] is not None
    assert 0.0 <= report["energy_drift"] < 1e-2
    assert report["momentum_error"] < 1e-6


def _read_checkpoint(path: str) -> dict:
    raw = open(path, "rb").read()
    head = O.CheckpointHeader.from_buffer_copy(raw[8:8 + C.sizeof(O.CheckpointHeader)])
    n = head.particle_count
    arrays = np.frombuffer(raw[8 + C.sizeof(O.CheckpointHeader):], dtype=np.float64)
    assert arrays.size == 10 * n
    return {f: arrays[k * n:(k + 1) * n] for k, f in enumerate(O.FIELDS)}


@needs_cli
@pytest.mark.gpu
@pytest.mark.parametrize("algorithm,theta,acc_tol,pos_tol", [
    ("cuda", 0.7, 2e-6, 1e-10),          # all-pairs bars of tests/test_allpairs_gpu.py
    ("barnes_hut_cuda", 0.5, 1e-2, 1e-7),  # the reference's own theta-0.3 bar, at 0.5
    ("cuda_resident", 0.7, 2e-6, 1e-10),
    ("barnes_hut_cuda_resident", 0.5, 1e-2, 1e-7),
])
def test_controller_steps_match_the_oracle(tmp_path, algorithm, theta, acc_tol, pos_tol):
    """Three controller steps against the oracle's FP64 leapfrog with the exact
    all-pairs sum on the same sequential preset: the reference's host leapfrog
    (integrator.c:47-85) with the device force function, or (`_resident`) the
    controller's device-resident step — the state uploaded once, advanced by
    n_body_sim_pro_cuda_advance and downloaded only when the checkpoint is
    written."""
    n, seed, eps, dt, steps = 4096, 42, 0.01, 1e-3, 3
    out = str(tmp_path / "state.ckpt")
    r = subprocess.run([STEPS_DRIVER, "globular_cluster", str(n), str(seed), algorithm,
                        str(theta), str(eps), str(dt), str(steps), out],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    got = _read_checkpoint(out)
    p = O.preset("globular_cluster", n, seed)  # the controller's sequential generation
    O.gravity_reference(p, 1.0, eps)
    O.advance(p, 1.0, eps, dt, steps, integrator=1, force=0)
    acc = np.stack([got["ax"], got["ay"], got["az"]], axis=1)
    assert O.rms_relative_error(acc, p.acc()) < acc_tol
    for f in ("x", "y", "z"):
        assert np.max(np.abs(got[f] - getattr(p, f))) < pos_tol, f
    assert np.array_equal(got["m"], p.m)
