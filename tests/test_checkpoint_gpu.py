"""Checkpoints of device-resident state in the reference's file format
(src/c/checkpoint/checkpoint.c), written and read straight from the device.

Parity: the file written from the device is byte-identical to the oracle's
restatement of the reference writer (pinned to the reference in
tests/test_oracle.py); a state read back and stepped matches, bit for bit,
the same state stepped without the round trip.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def to_system(nb, p):
    return nb.ParticleSystem(*[getattr(p, f).copy() for f in O.FIELDS])


def header(nb, n, t=0.0):
    h = nb.CheckpointHeader()
    h.magic, h.version, h.particle_count = nb.CHECKPOINT_MAGIC, nb.CHECKPOINT_VERSION, n
    h.simulation_time, h.timestep, h.integrator = t, 1e-3, 1
    h.theta, h.barnes_hut_enabled, h.random_seed, h.preset = 0.7, 1, 42, 4
    return h


def oracle_header(nb_header):
    h = O.CheckpointHeader()
    C_bytes = bytes(nb_header)
    assert len(C_bytes) == len(bytes(h))
    import ctypes
    ctypes.memmove(ctypes.addressof(h), C_bytes, len(C_bytes))
    return h


@pytest.mark.parametrize("n", [1, 1000, 1_200_000])
def test_device_checkpoint_bytes_equal_reference_format(cuda, ctx, tmp_path, n):
    """1.2M particles: 9.6 MB per array, more than one 8 MiB staging chunk."""
    p = O.preset("random_cloud", n, 5) if n > 2 else O.preset("random_cloud", n, 5)
    p.ax[:] = np.linspace(-1.0, 1.0, n)
    p.ay[:] = 2.0
    p.az[:] = -3.0
    ctx.upload(to_system(cuda, p))
    h = header(cuda, n, t=0.5)
    path = str(tmp_path / "gpu.hpcs")
    ctx.checkpoint_write(path, h)
    with open(path, "rb") as f:
        got = f.read()
    assert got == O.checkpoint_bytes(oracle_header(h), p)


def test_checkpoint_round_trip_resumes_bitwise(cuda, tmp_path):
    g = cuda.gravity_init(1.0, 0.01)
    p = O.preset("globular_cluster", 20000, 42)
    a = cuda.CudaContext(theta=0.7)
    a.upload(to_system(cuda, p))
    a.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
    a.advance(g, 1e-3, 3, cuda.Algorithm.BARNES_HUT)
    path = str(tmp_path / "mid.hpcs")
    a.checkpoint_write(path, header(cuda, p.n, t=3e-3))
    a.advance(g, 1e-3, 2, cuda.Algorithm.BARNES_HUT)
    straight = cuda.ParticleSystem.zeros(p.n)
    a.download(straight)
    a.close()

    b = cuda.CudaContext(theta=0.7)
    h = b.checkpoint_read(path)
    assert h.particle_count == p.n and h.simulation_time == 3e-3 and h.preset == 4
    b.advance(g, 1e-3, 2, cuda.Algorithm.BARNES_HUT)
    resumed = cuda.ParticleSystem.zeros(p.n)
    b.download(resumed)
    b.close()
    for f in O.FIELDS:
        assert np.array_equal(getattr(straight, f), getattr(resumed, f)), f


def test_checkpoint_errors_like_reference(cuda, ctx, tmp_path):
    p = O.preset("random_cloud", 100, 1)
    ctx.upload(to_system(cuda, p))
    with pytest.raises(cuda.CudaError) as e:  # checkpoint.c:18-22
        ctx.checkpoint_write(str(tmp_path / "x.hpcs"), header(cuda, 99))
    assert e.value.status == cuda.Status.INVALID_ARGUMENT
    with pytest.raises(cuda.CudaError) as e:  # unopenable file
        ctx.checkpoint_write(str(tmp_path / "no" / "such" / "dir.hpcs"), header(cuda, 100))
    assert e.value.status == cuda.Status.IO_ERROR
    with pytest.raises(cuda.CudaError) as e:
        ctx.checkpoint_read(str(tmp_path / "missing.hpcs"))
    assert e.value.status == cuda.Status.IO_ERROR
    bad = tmp_path / "bad.hpcs"
    bad.write_bytes(b"\x00" * 200)  # wrong magic (checkpoint.c:88-92)
    with pytest.raises(cuda.CudaError) as e:
        ctx.checkpoint_read(str(bad))
    assert e.value.status == cuda.Status.INVALID_STATE
    good = tmp_path / "good.hpcs"
    ctx.checkpoint_write(str(good), header(cuda, 100))
    short = tmp_path / "short.hpcs"
    short.write_bytes(good.read_bytes()[:-8])  # truncated last array
    with pytest.raises(cuda.CudaError) as e:
        ctx.checkpoint_read(str(short))
    assert e.value.status == cuda.Status.IO_ERROR
