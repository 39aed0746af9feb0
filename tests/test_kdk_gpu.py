"""Device-resident leapfrog / Verlet / Euler steps and FP64 diagnostics vs the
oracle (src/c/physics/integrator.c, src/c/diagnostics/numerics.c), mirroring
tests/regression/two_body_test.c and tests/numerical/diagnostics_test.c."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def to_system(nb, p):
    return nb.ParticleSystem(*[getattr(p, f).copy() for f in O.FIELDS])


def run_orbit(nb, integrator, orbits, steps_per_orbit):
    p = O.preset("two_body", 2, 1)
    g = nb.gravity_init(1.0, 0.0)
    ctx = nb.CudaContext()
    s = to_system(nb, p)
    ctx.upload(s)
    ctx.compute_acceleration(g, nb.Algorithm.ALL_PAIRS)
    q0, pe0 = ctx.diagnostics(g, potential=True)
    dt = 2 * np.pi / np.sqrt(2.0) / steps_per_orbit
    ctx.advance(g, dt, orbits * steps_per_orbit, nb.Algorithm.ALL_PAIRS, integrator)
    q1, pe1 = ctx.diagnostics(g, potential=True)
    ctx.download(s)
    ctx.close()
    e0, e1 = q0[0] + pe0, q1[0] + pe1
    sep = np.sqrt((s.x[1] - s.x[0]) ** 2 + (s.y[1] - s.y[0]) ** 2 + (s.z[1] - s.z[0]) ** 2)
    return abs(e1 - e0) / abs(e0), abs(sep - 1.0), np.linalg.norm(q1[2:5]), np.linalg.norm(q1[8:11])


@pytest.mark.parametrize("integrator", ["LEAPFROG", "VELOCITY_VERLET"])
def test_circular_orbit_stays_stable(cuda, integrator):
    """two_body_test.c:137-167: 8 orbits x 500 steps."""
    drift, sep_err, p, com = run_orbit(cuda, cuda.Integrator[integrator], 8, 500)
    assert drift < 1e-3
    assert sep_err < 1e-2
    assert p < 1e-12
    assert com < 1e-12


def test_euler_drifts_more_than_symplectic(cuda):
    """two_body_test.c:169-184."""
    euler, *_ = run_orbit(cuda, cuda.Integrator.EULER, 1, 500)
    verlet, *_ = run_orbit(cuda, cuda.Integrator.VELOCITY_VERLET, 1, 500)
    assert euler > 1e-3 and euler > verlet


def test_plummer_3_steps_match_reference(cuda, ctx):
    """Config 1: Plummer N=16384 seed 42, eps 0.01, leapfrog KDK dt=1e-3 x 3."""
    p = O.preset("globular_cluster", 16384, 42)
    g = cuda.gravity_init(1.0, 0.01)
    q = p.copy()
    O.gravity_reference(q, 1.0, 0.01, openmp=True)
    O.advance(q, 1.0, 0.01, 1e-3, 3, integrator=1, force=1)
    s = to_system(cuda, p)
    ctx.upload(s)
    ctx.compute_acceleration(g, cuda.Algorithm.ALL_PAIRS)
    ctx.advance(g, 1e-3, 3)
    ctx.download(s)
    for f in ("x", "y", "z"):
        assert np.max(np.abs(getattr(s, f) - getattr(q, f))) < 1e-10
    for f in ("vx", "vy", "vz"):
        assert np.max(np.abs(getattr(s, f) - getattr(q, f))) < 1e-8
    assert O.rms_relative_error(s.acc(), q.acc()) < 2e-6
    np.testing.assert_allclose(ctx.diagnostics(g), O.diagnostics(q), rtol=1e-7, atol=1e-12)
    # the FP64 device reductions on the oracle's own state
    ctx.upload(to_system(cuda, q))
    np.testing.assert_allclose(ctx.diagnostics(g), O.diagnostics(q), rtol=1e-12, atol=1e-15)


def test_diagnostics_analytic(cuda, ctx):
    """diagnostics_test.c:13-50."""
    s = cuda.ParticleSystem.zeros(2)
    s.x[:], s.y[:], s.z[:] = [1, 4], [2, 5], [3, 6]
    s.vx[:], s.vy[:] = [1, 0], [0, 1]
    s.m[:] = [2, 3]
    ctx.upload(s)
    np.testing.assert_allclose(ctx.diagnostics(),
                               [2.5, 5, 2, 3, 0, -18, 6, 8, 14 / 5, 19 / 5, 24 / 5], atol=1e-15)


def test_potential_energy_single_pair(cuda, ctx):
    """diagnostics_test.c:53-80: U = -1."""
    p = O.preset("two_body", 2, 1)
    ctx.upload(to_system(cuda, p))
    _, pe = ctx.diagnostics(cuda.gravity_init(1.0, 0.0), potential=True)
    assert abs(pe + 1.0) < 1e-15


def test_empty_system_diagnostics_are_zero(cuda, ctx):
    """diagnostics_test.c:82-103."""
    ctx.upload(cuda.ParticleSystem.zeros(0))
    q, pe = ctx.diagnostics(cuda.gravity_init(1.0, 0.01), potential=True)
    assert np.all(q == 0.0) and pe == 0.0


def test_potential_energy_matches_oracle(cuda, ctx):
    p = O.preset("globular_cluster", 6000, 2)
    ctx.upload(to_system(cuda, p))
    _, pe = ctx.diagnostics(cuda.gravity_init(1.0, 0.01), potential=True)
    ref = O.potential_energy(p, 1.0, 0.01)
    assert abs(pe - ref) <= 1e-12 * abs(ref)


def test_advance_rejects_bad_arguments(cuda, ctx):
    """integrator.c:145-156: timestep <= 0 -> INVALID_ARGUMENT; no state -> INVALID_STATE."""
    g = cuda.gravity_init(1.0, 0.01)
    with pytest.raises(cuda.CudaError) as e:
        ctx.advance(g, 1e-3, 1)
    assert e.value.status == cuda.Status.INVALID_STATE
    ctx.upload(to_system(cuda, O.preset("random_cloud", 64, 1)))
    for dt in (0.0, -1.0):
        with pytest.raises(cuda.CudaError) as e:
            ctx.advance(g, dt, 1)
        assert e.value.status == cuda.Status.INVALID_ARGUMENT


def test_nonfinite_position_is_reported(cuda, ctx):
    p = O.preset("random_cloud", 300, 3)
    p.x[17] = np.nan
    s = to_system(cuda, p)
    with pytest.raises(cuda.CudaError) as e:
        cuda.n_body_sim_pro_gravity_compute_acceleration_cuda(s, cuda.gravity_init(1.0, 0.01), ctx)
    assert e.value.status == cuda.Status.INVALID_ARGUMENT
    # the context stays usable
    p.x[17] = 0.1
    s = to_system(cuda, p)
    cuda.n_body_sim_pro_gravity_compute_acceleration_cuda(s, cuda.gravity_init(1.0, 0.01), ctx)
