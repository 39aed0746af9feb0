"""Batched ensembles: every system must evolve exactly like the oracle's
per-system leapfrog with all-pairs forces (src/c/physics/integrator.c:47-85,
gravity.c:37-67), in both the persistent graph-captured launch and the
one-launch-per-system baseline.

Tolerances (FP32 forces, FP64 state, T = steps x dt): an FP32 force carries a
relative error of ~1e-6, so per system with largest acceleration A the bounds
are |dx| <= 1e-6 A T^2 + 1e-12 and |dv| <= 2e-6 A T + 1e-12 against the FP64
oracle run (a tight binary of a small system has A ~ 1e3).
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def make_ensemble(nb, sizes_seed=5, count=40, lo=32, hi=512, extra=()):
    members = [O.ensemble_member(sizes_seed, k, lo, hi) for k in range(count)]
    members += list(extra)
    n = sum(p.n for p in members)
    s = nb.ParticleSystem.zeros(n)
    offsets = [0]
    for p in members:
        o = offsets[-1]
        for f in O.FIELDS:
            getattr(s, f)[o:o + p.n] = getattr(p, f)
        offsets.append(o + p.n)
    return members, s, np.array(offsets, dtype=np.uint64)


def oracle_run(members, eps, dt, steps):
    out = []
    for p in members:
        q = p.copy()
        O.gravity_reference(q, 1.0, eps)
        O.advance(q, 1.0, eps, dt, steps)
        out.append(q)
    return out


def check(nb, s, offsets, expected, span=1e-2):
    for k, q in enumerate(expected):
        a, b = int(offsets[k]), int(offsets[k + 1])
        amax = float(np.max(np.linalg.norm(q.acc(), axis=1)))
        tx, tv = 1e-6 * amax * span * span + 1e-12, 2e-6 * amax * span + 1e-12
        for f in ("x", "y", "z"):
            assert np.max(np.abs(getattr(s, f)[a:b] - getattr(q, f))) < tx, (k, f)
        for f in ("vx", "vy", "vz"):
            assert np.max(np.abs(getattr(s, f)[a:b] - getattr(q, f))) < tv, (k, f)


@pytest.mark.parametrize("per_system", [False, True])
def test_ensemble_matches_per_system_oracle(cuda, per_system):
    single = O.Particles.zeros(1)
    single.m[:] = 1.0
    big = O.ensemble_member(9, 0, 4096, 4096)
    members, s, offsets = make_ensemble(cuda, extra=(single, big))
    g = cuda.gravity_init(1.0, 0.01)
    expected = oracle_run(members, 0.01, 1e-3, 10)
    with cuda.CudaEnsemble() as e:
        e.upload(s, offsets)
        ms = e.advance(g, 1e-3, 10, one_launch_per_system=per_system)
        assert ms > 0
        out = cuda.ParticleSystem.zeros(s.n)
        e.download(out)
        info = e.info()
    check(cuda, out, offsets, expected)
    assert info["systems"] == len(members) and info["grid"] >= 1
    if not per_system:
        assert info["threads_per_block"] * info["targets_per_thread"] >= 4096
        assert sum(1 for t in info["autotune_ms"] if t > 0) >= 2


def test_ensemble_many_tiny_systems(cuda):
    """Hundreds of 1..40-particle systems share work items: each is padded to
    whole source tiles inside its own shared-memory slots."""
    members, s, offsets = make_ensemble(cuda, sizes_seed=21, count=300, lo=1, hi=40)
    g = cuda.gravity_init(1.0, 0.01)
    expected = oracle_run(members, 0.01, 1e-3, 5)
    with cuda.CudaEnsemble() as e:
        e.upload(s, offsets)
        e.advance(g, 1e-3, 5)
        out = cuda.ParticleSystem.zeros(s.n)
        e.download(out)
    check(cuda, out, offsets, expected, span=5e-3)


def test_ensemble_zero_softening(cuda):
    """eps = 0: the guarded kernel drops each target's own r^2 = 0 pair."""
    members, s, offsets = make_ensemble(cuda, sizes_seed=3, count=12, lo=32, hi=200)
    g = cuda.gravity_init(1.0, 0.0)
    expected = oracle_run(members, 0.0, 1e-4, 3)
    with cuda.CudaEnsemble() as e:
        e.upload(s, offsets)
        e.advance(g, 1e-4, 3)
        out = cuda.ParticleSystem.zeros(s.n)
        e.download(out)
    assert all(np.all(np.isfinite(getattr(out, f))) for f in O.FIELDS)
    check(cuda, out, offsets, expected, span=3e-4)


def test_ensemble_repeated_advance_and_graph_reuse(cuda):
    members, s, offsets = make_ensemble(cuda, count=24)
    g = cuda.gravity_init(1.0, 0.01)
    expected = oracle_run(members, 0.01, 1e-3, 6)
    with cuda.CudaEnsemble() as e:
        e.upload(s, offsets)
        for _ in range(3):  # the same captured graph, launched three times
            e.advance(g, 1e-3, 2)
        out = cuda.ParticleSystem.zeros(s.n)
        e.download(out)
    # each advance recomputes the initial forces of its first step: same physics
    check(cuda, out, offsets, expected, span=6e-3)


def test_ensemble_rejects_oversized_systems(cuda):
    s = cuda.ParticleSystem.zeros(4097)
    s.m[:] = 1.0
    s.x[:] = np.arange(4097)
    with cuda.CudaEnsemble() as e:
        with pytest.raises(cuda.CudaError) as err:
            e.upload(s, [0, 4097])
        assert err.value.status == cuda.Status.INVALID_ARGUMENT
        with pytest.raises(cuda.CudaError):
            e.upload(s, [0, 10, 4000])  # does not end at the particle count
