"""The CPU oracle, pinned.

1. Bit-identical to the reference engine compiled from its own sources
   (oracle/_ref, built by `make -C oracle ref`) on the same seeds: presets,
   all-pairs forces, Morton keys + permutation, Barnes-Hut forces and stats,
   integrator steps, diagnostics.
2. The reference test suite's known answers (tests/numerical/*.c,
   tests/regression/two_body_test.c).
3. The committed golden fixtures (tests/golden/, made by make_golden.py from
   oracle/_ref), so the pin holds where the reference is not built.
"""
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")

STATE = ("x", "y", "z", "vx", "vy", "vz", "m")


@needs_ref
@pytest.mark.parametrize("name,n,seed", [("random_cloud", 512, 42), ("random_cloud", 300, 7),
                                         ("globular_cluster", 2000, 42),
                                         ("spiral_galaxy", 400, 99), ("two_body", 2, 1)])
def test_presets_bit_identical_to_reference(name, n, seed):
    a, b = O.preset(name, n, seed), O.ref_preset(name, n, seed)
    for f in STATE:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def _reference_openmp_single_thread():
    """The reference's random_cloud sums velocities in an OpenMP reduction
    (presets_parallel.c:232); with one thread that sum runs in index order."""
    import ctypes
    ctypes.CDLL("libgomp.so.1").omp_set_num_threads(1)


@needs_ref
@pytest.mark.parametrize("name,n,seed", [
    ("two_body", 2, 1), ("random_cloud", 777, 42), ("solar_system", 9, 3),
    ("open_cluster", 500, 5), ("globular_cluster", 1500, 42), ("spiral_galaxy", 640, 99),
    ("elliptical_galaxy", 333, 8), ("galaxy_collision", 801, 12), ("triple_galaxy", 1001, 4)])
def test_parallel_presets_bit_identical_to_reference(name, n, seed):
    """presets_parallel.c restated: every filled particle equals the reference's."""
    _reference_openmp_single_thread()
    a, b = O.preset_parallel(name, n, seed), O.ref_preset(name, n, seed, parallel=True)
    k = O.filled_count(name, n)
    for f in STATE:
        assert np.array_equal(getattr(a, f)[:k], getattr(b, f)[:k]), f
    if k < n:  # the unfilled tail only gets the approach velocity (collision)
        assert np.all(a.x[k:] == 0.0)


@needs_ref
@pytest.mark.parametrize("n,seed", [(1000, 42), (777, 5)])
def test_plummer_collision_blocks_are_the_reference_plummer_block(n, seed):
    """The two-Plummer collision (parallel-preset form) is pinned to the
    reference's own fill_plummer_block through its exported presets: with no
    separation and no shear, block 0 holds the positions of the reference's
    parallel globular cluster of n/2 particles seeded mix_seed(seed, 0), block 1
    particles [n/2, n) of the one of n particles seeded mix_seed(seed, 1), bit
    for bit; block 0's velocities are that preset's scaled by sqrt(1/2) (the
    dispersion of a sphere of mass 1/2) and its masses are half its masses."""
    _reference_openmp_single_thread()
    half = n // 2
    c = O.plummer_collision_parallel(n, seed, separation=0.0, relative_speed=0.0)
    b0 = O.ref_preset("globular_cluster", half, O.lib().oracle_mix_seed(seed, 0), parallel=True)
    b1 = O.ref_preset("globular_cluster", n, O.lib().oracle_mix_seed(seed, 1), parallel=True)
    for f in ("x", "y", "z"):
        assert np.array_equal(getattr(c, f)[:half], getattr(b0, f)), f
        assert np.array_equal(getattr(c, f)[half:], getattr(b1, f)[half:]), f
    assert np.array_equal(c.m[:half], 0.5 * b0.m)
    assert np.allclose(c.m[half:], 0.5 / (n - half), rtol=0, atol=0)
    for f in ("vx", "vy", "vz"):
        v, ref = getattr(c, f)[:half], np.sqrt(0.5) * getattr(b0, f)
        assert np.max(np.abs(v - ref)) <= 1e-14 * np.max(np.abs(ref)), f
    # the workload's geometry: centres -/+ 5 on x, zero net momentum per block,
    # then -/+ 0.15 on y
    w = O.plummer_collision_parallel(n, seed)
    assert np.array_equal(w.x[:half], c.x[:half] + -5.0)
    assert np.array_equal(w.x[half:], c.x[half:] + 5.0)
    assert np.array_equal(w.vy[:half], c.vy[:half] + -0.15)
    for blk in (slice(0, half), slice(half, n)):
        assert abs(np.sum(c.m[blk] * c.vx[blk])) < 1e-15


@needs_ref
@pytest.mark.parametrize("eps", [0.02, 0.0])
def test_gravity_bit_identical_to_reference(eps):
    p = O.preset("random_cloud", 512, 42)
    a = O.gravity_reference(p.copy(), 1.0, eps)
    b = O.ref_gravity(p.copy(), 1.0, eps)
    assert np.array_equal(a, b)
    c = O.gravity_reference(p.copy(), 1.0, eps, openmp=True)
    assert np.array_equal(a, c)


@needs_ref
@pytest.mark.parametrize("name,n,seed", [("random_cloud", 4096, 42), ("globular_cluster", 5000, 3),
                                         ("plummer_collision", 6000, 42),
                                         ("spiral_galaxy", 3000, 99), ("two_body", 2, 1)])
def test_morton_order_bit_identical_to_reference(name, n, seed):
    p = O.preset(name, n, seed)
    k1, p1, r1 = O.morton_order(p)
    k2, p2, r2 = O.ref_morton_order(p)
    assert np.array_equal(r1, r2)
    assert np.array_equal(k1, k2)
    assert np.array_equal(p1, p2)
    assert np.all(np.diff(k1.astype(np.float64)) >= 0)


@needs_ref
def test_morton_duplicates_keep_index_order():
    p = O.preset("random_cloud", 256, 5)
    p.x[100:140] = p.x[7]
    p.y[100:140] = p.y[7]
    p.z[100:140] = p.z[7]
    k1, p1, _ = O.morton_order(p)
    k2, p2, _ = O.ref_morton_order(p)
    assert np.array_equal(k1, k2) and np.array_equal(p1, p2)


@needs_ref
@pytest.mark.parametrize("theta", [0.3, 0.7, 1.2])
def test_barnes_hut_bit_identical_to_reference(theta):
    p = O.preset("random_cloud", 400, 7)
    a, sa = O.barnes_hut(p.copy(), 1.0, 0.02, theta)
    b, sb = O.ref_barnes_hut(p.copy(), 1.0, 0.02, theta)
    assert np.array_equal(a, b)
    assert sa == sb


@needs_ref
def test_integrator_and_diagnostics_bit_identical_to_reference():
    import ctypes as C

    R = O.ref()
    g = O.Gravity()
    R.n_body_sim_pro_gravity_init(C.byref(g), 1.0, 0.02)
    p = O.preset("globular_cluster", 256, 11)
    q = p.copy()
    O.gravity_reference(p, 1.0, 0.02)
    O.gravity_reference(q, 1.0, 0.02)
    err = O.Error()
    force = C.cast(R.n_body_sim_pro_gravity_compute_acceleration_reference, C.c_void_p)
    for integrator in (1, 2, 0):
        for _ in range(3):
            O.advance(p, 1.0, 0.02, 1e-3, 1, integrator=integrator)
            v = q.view()
            assert R.n_body_sim_pro_integrator_advance(C.byref(v), C.byref(g), integrator, 1e-3,
                                                       force, None, C.byref(err)) == 0
    for f in O.FIELDS:
        assert np.array_equal(getattr(p, f), getattr(q, f)), f
    d = (C.c_double * 11)()
    v = q.view()
    R.n_body_sim_pro_diagnostics_compute_global(C.byref(v), C.byref(d), C.byref(err))
    assert np.array_equal(np.array(d[:]), O.diagnostics(p))
    pe = C.c_double()
    R.n_body_sim_pro_diagnostics_compute_potential_energy(C.byref(v), C.byref(g), C.byref(pe),
                                                          C.byref(err))
    assert pe.value == O.potential_energy(p, 1.0, 0.02)


# ---- the reference's analytic known answers --------------------------------------


def _two(eps=0.0):
    p = O.preset("two_body", 2, 1)
    p.vx[:] = p.vy[:] = p.vz[:] = 0.0
    return p


def test_two_body_analytic_acceleration():
    """tests/numerical/gravity_test.c:30-60: a0 = (1,0,0), a1 = (-1,0,0)."""
    a = O.gravity_reference(_two(), 1.0, 0.0)
    np.testing.assert_allclose(a, [[1, 0, 0], [-1, 0, 0]], atol=1e-15)


def test_self_force_excluded():
    """gravity_test.c:62-89."""
    p = O.Particles.zeros(1)
    p.x[:] = p.y[:] = p.z[:] = 1.0
    p.m[:] = 1000.0
    assert np.all(O.gravity_reference(p, 1.0, 0.0) == 0.0)


def test_softening_bounds_force():
    """gravity_test.c:91-124."""
    p = O.Particles.zeros(2)
    p.x[1] = 1e-8
    p.m[:] = 1.0
    a = O.gravity_reference(p, 1.0, 1e-2)
    assert abs(a[1, 0]) < 1e6 and a[1, 0] < 0


def test_mutual_force_antisymmetry():
    """gravity_test.c:126-152."""
    a = O.gravity_reference(_two(), 1.0, 0.3)
    np.testing.assert_allclose(a[0], -a[1], atol=1e-15)


def test_global_quantities_analytic():
    """tests/numerical/diagnostics_test.c:13-50."""
    p = O.Particles.zeros(2)
    p.x[:], p.y[:], p.z[:] = [1, 4], [2, 5], [3, 6]
    p.vx[:], p.vy[:] = [1, 0], [0, 1]
    p.m[:] = [2, 3]
    np.testing.assert_allclose(O.diagnostics(p), [2.5, 5, 2, 3, 0, -18, 6, 8, 14 / 5, 19 / 5, 24 / 5],
                               atol=1e-15)


def test_potential_energy_single_pair():
    """diagnostics_test.c:53-80."""
    assert abs(O.potential_energy(_two(), 1.0, 0.0) + 1.0) < 1e-15


def test_empty_system_quantities_are_zero():
    """diagnostics_test.c:82-103."""
    assert np.all(O.diagnostics(O.Particles.zeros(0)) == 0.0)


def test_leapfrog_two_body_orbit():
    """tests/regression/two_body_test.c:137-151 (8 orbits x 500 steps)."""
    p = O.preset("two_body", 2, 1)
    O.gravity_reference(p, 1.0, 0.0)
    e0 = O.diagnostics(p)[0] + O.potential_energy(p, 1.0, 0.0)
    dt = 2 * np.pi / np.sqrt(2.0) / 500
    O.advance(p, 1.0, 0.0, dt, 8 * 500, integrator=1)
    q = O.diagnostics(p)
    e1 = q[0] + O.potential_energy(p, 1.0, 0.0)
    assert abs(e1 - e0) / abs(e0) < 1e-3
    sep = np.hypot(p.x[1] - p.x[0], p.y[1] - p.y[0])
    assert abs(sep - 1.0) < 1e-2
    assert np.linalg.norm(q[2:5]) < 1e-12 and np.linalg.norm(q[8:11]) < 1e-12


def test_theta_tradeoff_cpu():
    """tests/numerical/barnes_hut_test.c:105-160 on the oracle."""
    p = O.preset("random_cloud", 400, 7)
    ref = O.gravity_reference(p.copy(), 1.0, 0.02)
    a3, s3 = O.barnes_hut(p.copy(), 1.0, 0.02, 0.3)
    a12, s12 = O.barnes_hut(p.copy(), 1.0, 0.02, 1.2)
    e3, e12 = O.rms_relative_error(a3, ref), O.rms_relative_error(a12, ref)
    assert e3 < 0.01 and e3 < e12
    w = lambda s: s["accepted_approximations"] + s["exact_interactions"]  # noqa: E731
    assert w(s3) > w(s12)


# ---- golden fixtures ---------------------------------------------------------------


def _golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.fail(f"missing golden fixture {path}: run tests/golden/make_golden.py")
    return np.load(path)


def test_golden_plummer_forces_and_energy():
    g = _golden("plummer_2048.npz")
    p = O.preset("globular_cluster", 2048, 42)
    for f in STATE:
        assert np.array_equal(getattr(p, f), g[f]), f
    a = O.gravity_reference(p, 1.0, 0.01)
    assert np.array_equal(a, g["acc"])
    assert O.potential_energy(p, 1.0, 0.01) == float(g["potential"])
    O.advance(p, 1.0, 0.01, 1e-3, 3)
    assert np.array_equal(p.pos(), g["pos_after_3"])
    assert np.array_equal(O.diagnostics(p), g["diag_after_3"])


def test_golden_morton():
    g = _golden("morton.npz")
    for tag, name, n, seed in (("cloud", "random_cloud", 4096, 42),
                               ("collision", "plummer_collision", 8192, 42)):
        k, perm, root = O.morton_order(O.preset(name, n, seed))
        assert np.array_equal(k, g[f"{tag}_keys"])
        assert np.array_equal(perm, g[f"{tag}_perm"])
        assert np.array_equal(root, g[f"{tag}_root"])


def test_golden_barnes_hut():
    g = _golden("barnes_hut.npz")
    p = O.preset("random_cloud", 400, 7)
    a, s = O.barnes_hut(p, 1.0, 0.02, 0.7)
    assert np.array_equal(a, g["acc_theta07"])
    assert [s[k] for k in ("node_count", "leaf_count", "internal_node_count",
                           "accepted_approximations", "exact_interactions",
                           "maximum_depth")] == list(g["stats_theta07"])


def _header(n: int) -> "O.CheckpointHeader":
    h = O.CheckpointHeader()
    h.magic, h.version, h.particle_count = O.CHECKPOINT_MAGIC, O.CHECKPOINT_VERSION, n
    h.simulation_time, h.timestep, h.integrator = 0.125, 1e-3, 1
    h.theta, h.barnes_hut_enabled, h.random_seed, h.preset = 0.7, 1, 42, 4
    return h


@needs_ref
def test_checkpoint_format_equals_reference_writer(tmp_path):
    """checkpoint.c:9-76 restated: the oracle's bytes are the reference's file."""
    p = O.preset("globular_cluster", 1000, 42)
    O.gravity_reference(p, 1.0, 0.01)
    path = str(tmp_path / "ref.hpcs")
    assert O.ref_checkpoint_write(path, _header(p.n), p) == 0
    with open(path, "rb") as f:
        assert f.read() == O.checkpoint_bytes(_header(p.n), p)
