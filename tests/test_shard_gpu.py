"""Target-sharded all-pairs (shard_begin / all-gather / shard_end) on one B200.

Several ranks' slices are emulated in one process: each slice lives in its own
context, shard_begin packs it into its part of one device buffer (what the
NCCL all-gather assembles across GPUs), shard_end evaluates its targets from
the whole buffer.  Tolerances as the all-pairs parity tests: rms relative
error <= 2e-6 against the FP64 oracle (gravity.c:46-61).
"""
import numpy as np
import pytest
import torch

import oracle as O

from n_body_sim_pro_b200 import shard

pytestmark = pytest.mark.gpu

RMS_TOL = 2e-6


def to_system(nb, p, first=0, count=None):
    count = p.n - first if count is None else count
    return nb.ParticleSystem(*[getattr(p, f)[first: first + count].copy() for f in O.FIELDS])


def accelerations(s):
    return np.stack([s.ax, s.ay, s.az], axis=1)


@pytest.mark.parametrize("world", [1, 2, 3])
def test_emulated_ranks_match_the_oracle(cuda, world):
    p = O.preset("globular_cluster", 5000, 7)
    g = cuda.gravity_init(1.0, 0.01)
    ref = O.gravity_reference(p.copy(), 1.0, 0.01, openmp=True)
    parts = shard.split(p.n, world)
    cap = shard.capacity_for([c for _, c in parts])
    sources = torch.zeros((world * cap, 4), dtype=torch.float32, device="cuda")
    centre = [np.dot(p.m, p.x) / p.m.sum(), np.dot(p.m, p.y) / p.m.sum(),
              np.dot(p.m, p.z) / p.m.sum()]
    ctxs = [cuda.CudaContext() for _ in range(world)]
    try:
        for r, (first, count) in enumerate(parts):
            ctxs[r].upload(to_system(cuda, p, first, count))
            view = sources[r * cap:(r + 1) * cap]
            ctxs[r].shard_begin(0.0, centre, view.data_ptr(), cap)
        torch.cuda.synchronize()
        got = np.zeros((p.n, 3))
        for r, (first, count) in enumerate(parts):
            ctxs[r].shard_end(g, 0.0, sources.data_ptr(), world * cap, r * cap)
            out = to_system(cuda, p, first, count)
            ctxs[r].download(out)
            got[first: first + count] = accelerations(out)
        err = O.rms_relative_error(got, ref)
        print(f"world={world} rms={err:.2e}")
        assert err < RMS_TOL
    finally:
        for c in ctxs:
            c.close()


def test_one_rank_steps_match_the_resident_advance(cuda):
    p = O.preset("globular_cluster", 4096, 3)
    g = cuda.gravity_init(1.0, 0.01)
    with cuda.CudaContext() as a, cuda.CudaContext() as b:
        sim = shard.ShardedAllPairs(to_system(cuda, p), g, shard.CudaShardBackend(a), "cuda")
        sim.step(1e-3, 3)
        mine = to_system(cuda, p)
        sim.download(mine)
        b.upload(to_system(cuda, p))
        b.compute_acceleration(g, cuda.Algorithm.ALL_PAIRS)
        b.advance(g, 1e-3, 3)
        theirs = to_system(cuda, p)
        b.download(theirs)
    for f in ("x", "y", "z"):
        np.testing.assert_allclose(getattr(mine, f), getattr(theirs, f), rtol=0, atol=1e-12)
    assert O.rms_relative_error(accelerations(mine), accelerations(theirs)) < 1e-6


def test_shard_arguments_checked(cuda):
    p = O.preset("random_cloud", 100, 1)
    g = cuda.gravity_init(1.0, 0.01)
    buf = torch.zeros((256, 4), dtype=torch.float32, device="cuda")
    with cuda.CudaContext() as c:
        c.upload(to_system(cuda, p))
        with pytest.raises(cuda.CudaError):  # capacity below the resident count
            c.shard_begin(0.0, [0, 0, 0], buf.data_ptr(), 64)
        with pytest.raises(cuda.CudaError):  # capacity not a multiple of 8
            c.shard_begin(0.0, [0, 0, 0], buf.data_ptr(), 250)
        c.shard_begin(0.0, [0, 0, 0], buf.data_ptr(), 256)
        with pytest.raises(cuda.CudaError):  # slice past the end of the sources
            c.shard_end(g, 0.0, buf.data_ptr(), 256, 200)
        with pytest.raises(cuda.CudaError):  # negative timestep
            c.shard_end(g, -1.0, buf.data_ptr(), 256, 0)
        c.shard_end(g, 0.0, buf.data_ptr(), 256, 0)
