"""All-pairs over several GPUs, sharded by targets: one process per GPU.

Rank r keeps its slice of the particles resident in its own context.  One
leapfrog kick-drift-kick step (src/c/physics/integrator.c:47-85) is

    shard_begin   opening kick + drift of the slice, slice packed as float4
                  (x - c, y - c, z - c, m) into `slice`         (library, GPU)
    all-gather    every rank's `slice` into `sources`, rank order (NCCL)
    shard_end     forces on the slice from all sources, closing kick (library)

so each step moves 16 bytes per particle over NVLink and every GPU evaluates
n_local x n pairs.  The reference point c of the packed coordinates is the
system's centre of mass at construction, the same on every rank (an
all-reduce); it only anchors the FP32 relative coordinates.

Slices are padded to a common capacity (a multiple of 256 entries) with
massless entries, which add exactly zero to every force.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

CAPACITY_ALIGN = 256


def split(n: int, world: int) -> list[tuple[int, int]]:
    """(first, count) of each rank's contiguous slice; counts differ by <= 1."""
    base, extra = divmod(int(n), int(world))
    out, first = [], 0
    for r in range(world):
        count = base + (1 if r < extra else 0)
        out.append((first, count))
        first += count
    return out


def assign_systems(sizes, world: int) -> list[list[int]]:
    """Independent systems (an ensemble) over `world` ranks with no collective:
    largest cost first (N^2 pairs per step) to the least loaded rank, ties to
    the lowest rank; each rank's list in ascending system order."""
    sizes = [int(v) for v in sizes]
    load = [0] * int(world)
    out: list[list[int]] = [[] for _ in range(int(world))]
    for k in sorted(range(len(sizes)), key=lambda j: (-sizes[j] * sizes[j], j)):
        r = min(range(int(world)), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += sizes[k] * sizes[k]
    return [sorted(v) for v in out]


def capacity_for(counts) -> int:
    """Common slice capacity: the largest count rounded up to CAPACITY_ALIGN."""
    top = max(int(c) for c in counts)
    return max(CAPACITY_ALIGN, -(-top // CAPACITY_ALIGN) * CAPACITY_ALIGN)


class CudaShardBackend:
    """The library's shard entry points on one context (this rank's GPU)."""

    def __init__(self, context):
        self.ctx = context

    def upload(self, system) -> None:
        self.ctx.upload(system)

    def begin(self, timestep: float, centre, slice_buf: torch.Tensor) -> None:
        self.ctx.shard_begin(timestep, centre, slice_buf.data_ptr(), slice_buf.shape[0])

    def end(self, gravity, timestep: float, sources: torch.Tensor, offset: int) -> None:
        self.ctx.shard_end(gravity, timestep, sources.data_ptr(), sources.shape[0], offset)

    def download(self, system) -> None:
        self.ctx.download(system)


class ShardedAllPairs:
    """Leapfrog KDK of one system whose particles are split over the ranks of
    `group` (the default process group, or a single process when
    torch.distributed is not initialised).

    `system` is this rank's slice (a ParticleSystem), `backend` runs the
    per-rank work (CudaShardBackend for the GPU), `device` holds the packed
    buffers (this rank's GPU for NCCL)."""

    def __init__(self, system, gravity, backend, device, group=None):
        self.group = group
        self.distributed = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if self.distributed else 0
        self.world = dist.get_world_size(group) if self.distributed else 1
        self.gravity = gravity
        self.backend = backend
        self.device = torch.device(device)
        self.n_local = int(system.n)
        counts = self._all_gather_scalars([self.n_local], torch.int64)
        self.counts = [int(c) for c in counts[:, 0]]
        self.n_total = sum(self.counts)
        self.first = sum(self.counts[: self.rank])
        self.capacity = capacity_for(self.counts)
        self.offset = self.rank * self.capacity
        self.slice = torch.zeros((self.capacity, 4), dtype=torch.float32, device=self.device)
        self.sources = (self.slice if self.world == 1 else
                        torch.zeros((self.world * self.capacity, 4), dtype=torch.float32,
                                    device=self.device))
        self.centre = self._centre_of_mass(system)
        backend.upload(system)
        self.have_forces = False

    # ---- collectives -------------------------------------------------------
    def _all_gather_scalars(self, values, dtype) -> np.ndarray:
        local = torch.tensor(values, dtype=dtype, device=self.device).reshape(1, -1)
        if self.world == 1:
            return local.cpu().numpy()
        out = torch.empty((self.world, local.shape[1]), dtype=dtype, device=self.device)
        dist.all_gather_into_tensor(out, local, group=self.group)
        return out.cpu().numpy()

    def _centre_of_mass(self, system) -> np.ndarray:
        m = np.asarray(system.m, dtype=np.float64)
        sums = [float(m.sum()), float(np.dot(m, system.x)), float(np.dot(m, system.y)),
                float(np.dot(m, system.z))]
        rows = self._all_gather_scalars(sums, torch.float64)
        total = rows.sum(axis=0)  # fixed rank order on every rank
        if total[0] == 0.0:
            return np.zeros(3)
        return total[1:] / total[0]

    def _gather_sources(self) -> None:
        if self.world > 1:
            dist.all_gather_into_tensor(self.sources, self.slice, group=self.group)
        if self.device.type == "cuda":
            torch.cuda.current_stream(self.device).synchronize()

    # ---- stepping ----------------------------------------------------------
    def compute_forces(self) -> None:
        """Accelerations of the current positions (before the first step)."""
        self.backend.begin(0.0, self.centre, self.slice)
        self._gather_sources()
        self.backend.end(self.gravity, 0.0, self.sources, self.offset)
        self.have_forces = True

    def step(self, timestep: float, steps: int = 1) -> None:
        if not timestep > 0.0:
            raise ValueError("timestep must be positive")
        if not self.have_forces:
            self.compute_forces()
        for _ in range(int(steps)):
            self.backend.begin(timestep, self.centre, self.slice)
            self._gather_sources()
            self.backend.end(self.gravity, timestep, self.sources, self.offset)

    def download(self, system) -> None:
        self.backend.download(system)
