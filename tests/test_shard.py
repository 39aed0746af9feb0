"""Host logic of the multi-GPU paths on CPU processes (gloo, world size 2):
the target-sharded all-pairs step (n_body_sim_pro_b200/shard.py) with a host
FP64 stand-in for the per-rank GPU work, the ensemble's system assignment, and
bench.py's barrier / max-over-ranks helpers.

The stand-in (HostShardBackend, test infrastructure) does what the library's
shard_begin / shard_end do — kick-drift, pack float4 relative to the centre,
direct-sum forces of the rank's targets from every gathered source, kick — so
the 2-rank run must reproduce the 1-rank run exactly: the same sources reach
every target in the same order, padding entries are massless.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from n_body_sim_pro_b200 import shard  # noqa: E402


class Slice:
    """The fields of a ParticleSystem the orchestration reads."""

    def __init__(self, x, y, z, vx, vy, vz, m):
        self.x, self.y, self.z = x.copy(), y.copy(), z.copy()
        self.vx, self.vy, self.vz = vx.copy(), vy.copy(), vz.copy()
        self.m = m.copy()
        self.ax = np.zeros_like(x)
        self.ay = np.zeros_like(x)
        self.az = np.zeros_like(x)
        self.n = x.shape[0]


class HostShardBackend:
    def __init__(self, eps):
        self.eps2 = eps * eps

    def upload(self, s):
        self.s = Slice(s.x, s.y, s.z, s.vx, s.vy, s.vz, s.m)

    def begin(self, dt, centre, slice_buf):
        s = self.s
        if dt > 0.0:
            for v, a, x in ((s.vx, s.ax, s.x), (s.vy, s.ay, s.y), (s.vz, s.az, s.z)):
                v += a * (0.5 * dt)
                x += v * dt
        rows = np.stack([s.x - centre[0], s.y - centre[1], s.z - centre[2], s.m], axis=1)
        slice_buf.zero_()
        slice_buf[: s.n] = torch.from_numpy(rows.astype(np.float32))

    def end(self, gravity, dt, sources, offset):
        s = self.s
        src = sources.numpy().astype(np.float64)
        tgt = src[offset: offset + s.n, :3]
        d = src[None, :, :3] - tgt[:, None, :]
        r2 = np.sum(d * d, axis=2) + self.eps2
        w = src[None, :, 3] / (r2 * np.sqrt(r2))
        a = gravity * np.einsum("ij,ijk->ik", w, d)
        s.ax, s.ay, s.az = a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy()
        for v, acc in ((s.vx, s.ax), (s.vy, s.ay), (s.vz, s.az)):
            v += acc * (0.5 * dt)

    def download(self, out):
        for f in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
            getattr(out, f)[:] = getattr(self.s, f)


def system(n, seed=5):
    rng = np.random.default_rng(seed)
    x, y, z = rng.normal(size=(3, n))
    vx, vy, vz = 0.1 * rng.normal(size=(3, n))
    m = rng.uniform(0.5, 1.5, n) / n
    return x, y, z, vx, vy, vz, m


def run_sharded(rank, world, n, steps, dt, eps, first_count):
    fields = system(n)
    first, count = first_count[rank]
    part = Slice(*[f[first: first + count] for f in fields])
    sim = shard.ShardedAllPairs(part, 1.0, HostShardBackend(eps), "cpu")
    sim.step(dt, steps)
    out = Slice(*[f[first: first + count] for f in fields])
    sim.download(out)
    return sim, out


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, steps, dt, eps, path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    w, r, _ = bench.dist_setup(world, backend="gloo")
    assert (w, r) == (world, rank)
    try:
        split = shard.split(n, world)
        sim, out = run_sharded(rank, world, n, steps, dt, eps, split)
        bench.barrier_sync(world)
        top = bench.max_over_ranks(float(rank) + 0.5, world)
        np.savez(f"{path}_{rank}.npz", x=out.x, vx=out.vx, ax=out.ax, centre=sim.centre,
                 counts=np.array(sim.counts), capacity=sim.capacity, offset=sim.offset,
                 top=top)
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def two_rank_run(tmp_path_factory):
    n, steps, dt, eps = 301, 3, 1e-3, 0.05
    path = str(tmp_path_factory.mktemp("shard") / "rank")
    mp.start_processes(_worker, args=(2, free_port(), n, steps, dt, eps, path), nprocs=2,
                       start_method="spawn", join=True)
    return n, steps, dt, eps, [dict(np.load(f"{path}_{r}.npz")) for r in range(2)]


def test_two_ranks_reproduce_one_rank(two_rank_run):
    n, steps, dt, eps, ranks = two_rank_run
    _, one = run_sharded(0, 1, n, steps, dt, eps, [(0, n)])
    split = shard.split(n, 2)
    for r, (first, count) in enumerate(split):
        np.testing.assert_array_equal(ranks[r]["x"], one.x[first: first + count])
        np.testing.assert_array_equal(ranks[r]["vx"], one.vx[first: first + count])
        np.testing.assert_array_equal(ranks[r]["ax"], one.ax[first: first + count])


def test_layout_and_centre_agree_across_ranks(two_rank_run):
    n, _, _, _, ranks = two_rank_run
    assert list(ranks[0]["counts"]) == [151, 150] == list(ranks[1]["counts"])
    assert int(ranks[0]["capacity"]) == int(ranks[1]["capacity"]) == 256
    assert [int(r["offset"]) for r in ranks] == [0, 256]
    np.testing.assert_array_equal(ranks[0]["centre"], ranks[1]["centre"])
    x, y, z, _, _, _, m = system(n)
    np.testing.assert_allclose(ranks[0]["centre"], [np.dot(m, x) / m.sum(),
                                                    np.dot(m, y) / m.sum(),
                                                    np.dot(m, z) / m.sum()], rtol=1e-12)


def test_max_over_ranks_and_barrier(two_rank_run):
    ranks = two_rank_run[4]
    assert [float(r["top"]) for r in ranks] == [1.5, 1.5]


def test_sharded_step_matches_the_oracle_direct_sum(two_rank_run):
    """The stand-in's forces are the reference's softened sum (gravity.c:46-61)
    on FP32-rounded relative coordinates: within 1e-6 of the FP64 oracle."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    n, steps, dt, eps, _ = two_rank_run
    x, y, z, vx, vy, vz, m = system(n)
    p = O.Particles.zeros(n)
    for f, v in zip(("x", "y", "z", "vx", "vy", "vz", "m"), (x, y, z, vx, vy, vz, m)):
        getattr(p, f)[:] = v
    ref = O.gravity_reference(p.copy(), 1.0, eps, openmp=False)
    sim = shard.ShardedAllPairs(Slice(x, y, z, vx, vy, vz, m), 1.0, HostShardBackend(eps), "cpu")
    sim.compute_forces()
    out = Slice(x, y, z, vx, vy, vz, m)
    sim.download(out)
    got = np.stack([out.ax, out.ay, out.az], axis=1)
    assert O.rms_relative_error(got, ref) < 1e-6


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_split_is_contiguous_and_balanced(world):
    n = 1001
    parts = shard.split(n, world)
    assert parts[0][0] == 0 and sum(c for _, c in parts) == n
    for (f0, c0), (f1, _) in zip(parts, parts[1:]):
        assert f1 == f0 + c0
    counts = [c for _, c in parts]
    assert max(counts) - min(counts) <= 1
    cap = shard.capacity_for(counts)
    assert cap % 256 == 0 and cap >= max(counts)


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_assign_systems_covers_each_once_and_balances(world):
    rng = np.random.default_rng(1)
    sizes = np.rint(np.exp(rng.uniform(np.log(32), np.log(4096), 4096))).astype(int)
    parts = shard.assign_systems(sizes, world)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(int(sizes[k]) ** 2 for k in p) for p in parts]
    assert max(loads) <= 1.01 * (sum(loads) / world) + max(sizes) ** 2
    assert parts == shard.assign_systems(sizes, world)  # deterministic
