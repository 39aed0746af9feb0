"""Device generation of the reference's parallel presets
(n_body_sim_pro_preset_generate_parallel, src/c/generation/presets_parallel.c)
against the oracle restatement, which tests/test_oracle.py pins bit for bit to
the reference itself.

Tolerance: the integer random streams are the reference's, the FP64 products
and sums round as on the CPU (no FMA contraction), and only CUDA's log, cos,
sin, pow and cbrt differ from the host libm (a few ulp).  The Plummer radius
a / sqrt(u^(-2/3) - 1) amplifies those ulp near u = 1, so each value is held
to 1e-9 relative (absolute below 1) and the whole state to 1e-13 rms; masses,
which involve no transcendental function, are equal.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

CASES = [("two_body", 2, 1), ("random_cloud", 5000, 42), ("solar_system", 17, 3),
         ("open_cluster", 3000, 5), ("globular_cluster", 20000, 42),
         ("spiral_galaxy", 4096, 99), ("elliptical_galaxy", 999, 8),
         ("galaxy_collision", 4001, 12), ("triple_galaxy", 3002, 4)]


def download(cuda, ctx, n):
    s = cuda.ParticleSystem.zeros(n)
    ctx.download(s)
    return s


@pytest.mark.parametrize("name,n,seed", CASES)
def test_device_preset_matches_oracle(cuda, ctx, name, n, seed):
    ctx.generate_preset(name, n, seed)
    got = download(cuda, ctx, n)
    ref = O.preset_parallel(name, n, seed)
    k = O.filled_count(name, n)
    assert np.array_equal(got.m[:k], ref.m[:k])
    worst = 0.0
    num = den = 0.0
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        a, b = getattr(got, f)[:k], getattr(ref, f)[:k]
        rel = np.abs(a - b) / np.maximum(np.abs(b), 1.0)
        worst = max(worst, float(rel.max()))
        num += float(np.sum((a - b) ** 2))
        den += float(np.sum(b ** 2))
    print(f"{name} n={n}: worst {worst:.2e} rms {np.sqrt(num / den):.2e}")
    assert worst <= 1e-9
    assert np.sqrt(num / den) <= 1e-13
    # accelerations start at zero; the unfilled tail is zero but for the
    # collision's approach velocity
    assert np.all(got.ax == 0.0) and np.all(got.ay == 0.0) and np.all(got.az == 0.0)
    if k < n:
        assert np.all(got.x[k:] == 0.0) and np.all(got.m[k:] == 0.0)
        if name == "galaxy_collision":
            assert np.all(got.vx[k:] == -0.35)


def test_device_preset_is_deterministic(cuda, ctx):
    ctx.generate_preset("globular_cluster", 50000, 7)
    a = download(cuda, ctx, 50000)
    ctx.generate_preset("globular_cluster", 50000, 7)
    b = download(cuda, ctx, 50000)
    for f in ("x", "y", "z", "vx", "vy", "vz", "m"):
        assert np.array_equal(getattr(a, f), getattr(b, f))
    # zero net momentum, as the reference's mean subtraction
    assert abs(float(np.sum(a.vx))) < 1e-12 and abs(float(np.sum(a.vz))) < 1e-12


def test_device_preset_argument_errors_like_reference(cuda, ctx):
    with pytest.raises(cuda.CudaError) as e:
        ctx.generate_preset("two_body", 3, 1)  # presets_parallel.c:343-347
    assert e.value.status == cuda.Status.INVALID_ARGUMENT
    with pytest.raises(cuda.CudaError) as e:
        ctx.generate_preset(42, 10, 1)
    assert e.value.status == cuda.Status.INVALID_ARGUMENT


def test_device_preset_then_step(cuda, ctx):
    """A generated system is resident: it steps without any upload."""
    g = cuda.gravity_init(1.0, 0.01)
    ctx.generate_preset("globular_cluster", 4096, 42)
    ctx.compute_acceleration(g, cuda.Algorithm.ALL_PAIRS)
    ctx.advance(g, 1e-3, 2, cuda.Algorithm.ALL_PAIRS)
    got = download(cuda, ctx, 4096)
    ref = O.preset_parallel("globular_cluster", 4096, 42)
    O.gravity_reference(ref, 1.0, 0.01, openmp=True)
    O.advance(ref, 1.0, 0.01, 1e-3, 2, integrator=1, force=1)
    assert np.max(np.abs(got.x - ref.x)) < 1e-9


@pytest.mark.parametrize("n,seed", [(20001, 42), (4096, 7)])
def test_device_plummer_collision_matches_oracle(cuda, ctx, n, seed):
    """The two-Plummer collision of the Barnes-Hut workloads (two spheres of
    mass 1/2 from the parallel presets' streams, -/+5 on x, -/+0.15 on y)
    against its oracle restatement, which tests/test_oracle.py pins to the
    reference's own Plummer block; same bars as the presets above."""
    ctx.generate_plummer_collision(n, seed)
    got = download(cuda, ctx, n)
    ref = O.plummer_collision_parallel(n, seed)
    assert np.array_equal(got.m, ref.m)
    num = den = worst = 0.0
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        a, b = getattr(got, f), getattr(ref, f)
        worst = max(worst, float((np.abs(a - b) / np.maximum(np.abs(b), 1.0)).max()))
        num += float(np.sum((a - b) ** 2))
        den += float(np.sum(b ** 2))
    assert worst <= 1e-9
    assert np.sqrt(num / den) <= 1e-13
    half = n // 2
    assert abs(np.mean(got.x[:half]) + 5.0) < 0.1 and abs(np.mean(got.x[half:]) - 5.0) < 0.1
    assert abs(np.sum(got.m[:half] * got.vy[:half]) / np.sum(got.m[:half]) + 0.15) < 1e-12
    assert np.all(got.ax == 0.0)
