"""n_body_sim_pro_b200 — B200-native force evaluation and time step.

Python mirror of the C ABI in include/n_body_sim_pro_cuda.h (the library
libn_body_sim_pro_cuda.so is built in-tree by ``n_body_sim_pro_b200.build``).
Names follow the reference engine's C API:

    n_body_sim_pro_gravity_compute_acceleration_cuda(view, gravity, context)
    n_body_sim_pro_barnes_hut_compute_acceleration_cuda(view, gravity, context)

are the two new ``NBodySimProForceFunction`` algorithms (``cuda`` and
``barnes_hut_cuda``); :class:`CudaContext` wraps ``NBodySimProCudaContext``
(the device-resident state, stepping and diagnostics).

There is no CPU fallback: importing works without a GPU, but every compute
call raises :class:`CudaError` with ``UNSUPPORTED_PLATFORM`` when no B200 is
present, and :func:`library` raises if the shared library was not built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from enum import IntEnum

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libn_body_sim_pro_cuda.so")


class Status(IntEnum):
    """NBodySimProStatus (include/n_body_sim_pro/core/status.h:18-28)."""

    OK = 0
    INVALID_ARGUMENT = 1
    OUT_OF_MEMORY = 2
    INVALID_STATE = 3
    NOT_IMPLEMENTED = 4
    UNSUPPORTED_PLATFORM = 5
    OVERFLOW = 6
    IO_ERROR = 7
    INSUFFICIENT_MEMORY = 8


class Integrator(IntEnum):
    """NBodySimProIntegratorType (include/n_body_sim_pro/physics/integrator.h:31-35)."""

    EULER = 0
    LEAPFROG = 1
    VELOCITY_VERLET = 2


class Algorithm(IntEnum):
    ALL_PAIRS = 0
    BARNES_HUT = 1


class Opening(IntEnum):
    """NBodySimProCudaOpening: the Barnes-Hut opening test."""
    REFERENCE = 0
    OFFSET = 1


class RelativeSource(IntEnum):
    """NBodySimProCudaRelativeSource: where the plugin functions take the
    relative opening test's previous accelerations."""
    FROM_VIEW = 0
    FROM_CONTEXT = 1


class View(C.Structure):
    """NBodySimProParticleSystemView (include/n_body_sim_pro/core/particle_system.h:38-50)."""

    _fields_ = [("particle_count", C.c_size_t)] + [
        (name, C.POINTER(C.c_double))
        for name in ("positions_x", "positions_y", "positions_z", "velocities_x",
                     "velocities_y", "velocities_z", "accelerations_x", "accelerations_y",
                     "accelerations_z", "masses")
    ]


class Gravity(C.Structure):
    """NBodySimProGravity (include/n_body_sim_pro/physics/gravity.h:25-29)."""

    _fields_ = [("gravitational_constant", C.c_double), ("softening_length", C.c_double),
                ("softening_squared", C.c_double)]


def gravity_init(gravitational_constant: float, softening_length: float) -> Gravity:
    """n_body_sim_pro_gravity_init (src/c/physics/gravity.c:5-13)."""
    return Gravity(gravitational_constant, softening_length, softening_length * softening_length)


class Error(C.Structure):
    """NBodySimProError (include/n_body_sim_pro/core/status.h:30-35)."""

    _fields_ = [("status", C.c_int), ("source_file", C.c_char_p), ("source_line", C.c_int),
                ("message", C.c_char * 256)]


class BarnesHutStats(C.Structure):
    """NBodySimProBarnesHutStats (include/n_body_sim_pro/barnes_hut/barnes_hut.h:31-40)."""

    _fields_ = [(n, C.c_size_t) for n in ("node_count", "leaf_count", "internal_node_count",
                                          "accepted_approximations", "exact_interactions",
                                          "maximum_depth")] + [
        ("build_time_seconds", C.c_double), ("evaluation_time_seconds", C.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class DiagnosticsQuantities(C.Structure):
    """NBodySimProDiagnosticsQuantities (include/n_body_sim_pro/diagnostics/numerics.h:22-34)."""

    _fields_ = [(n, C.c_double) for n in (
        "kinetic_energy", "total_mass", "total_momentum_x", "total_momentum_y",
        "total_momentum_z", "total_angular_momentum_x", "total_angular_momentum_y",
        "total_angular_momentum_z", "center_of_mass_x", "center_of_mass_y", "center_of_mass_z")]

    def as_array(self) -> np.ndarray:
        return np.array([getattr(self, f) for f, _ in self._fields_], dtype=np.float64)


class Timings(C.Structure):
    """NBodySimProCudaTimings: per-phase device milliseconds of the last call."""

    _fields_ = [(n, C.c_double) for n in ("bounds_ms", "keys_ms", "sort_ms", "build_ms",
                                          "moments_ms", "walk_ms", "integrate_ms", "total_ms")]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class EnsembleInfo(C.Structure):
    """NBodySimProCudaEnsembleInfo: the autotuned shape and the last device time."""

    _fields_ = [("systems", C.c_size_t), ("particles", C.c_size_t),
                ("threads_per_block", C.c_int), ("targets_per_thread", C.c_int),
                ("grid", C.c_int), ("work_items", C.c_int), ("last_advance_ms", C.c_double),
                ("autotune_ms", C.c_double * 3)]

    def as_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "autotune_ms"}
        d["autotune_ms"] = list(self.autotune_ms)
        return d


class CheckpointHeader(C.Structure):
    """NBodySimProCheckpointHeader (checkpoint/checkpoint.h:29-40), C layout with padding."""

    _fields_ = [("magic", C.c_uint32), ("version", C.c_uint32), ("particle_count", C.c_size_t),
                ("simulation_time", C.c_double), ("timestep", C.c_double),
                ("integrator", C.c_int32), ("theta", C.c_double),
                ("barnes_hut_enabled", C.c_int32), ("random_seed", C.c_uint64),
                ("preset", C.c_int32)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


CHECKPOINT_MAGIC = 0x53504348
CHECKPOINT_VERSION = 1


class CudaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{Status(status).name}: {message}")
        self.status = Status(status)


EXPORTS = (
    "n_body_sim_pro_cuda_context_create", "n_body_sim_pro_cuda_context_destroy",
    "n_body_sim_pro_cuda_context_set_theta", "n_body_sim_pro_cuda_context_theta",
    "n_body_sim_pro_cuda_context_set_multipole_order",
    "n_body_sim_pro_cuda_context_set_leaf_capacity", "n_body_sim_pro_cuda_context_stats",
    "n_body_sim_pro_cuda_context_timings", "n_body_sim_pro_gravity_compute_acceleration_cuda",
    "n_body_sim_pro_barnes_hut_compute_acceleration_cuda", "n_body_sim_pro_cuda_upload",
    "n_body_sim_pro_cuda_download", "n_body_sim_pro_cuda_compute_acceleration",
    "n_body_sim_pro_cuda_advance", "n_body_sim_pro_cuda_diagnostics",
    "n_body_sim_pro_cuda_reference_acceleration", "n_body_sim_pro_cuda_morton_order",
    "n_body_sim_pro_cuda_synchronize", "n_body_sim_pro_cuda_architecture",
    "n_body_sim_pro_cuda_kernel_launches", "n_body_sim_pro_cuda_context_walk_restarts",
    "n_body_sim_pro_cuda_context_corrected_cells", "n_body_sim_pro_cuda_context_set_relative_opening",
    "n_body_sim_pro_cuda_preset_generate_parallel", "n_body_sim_pro_cuda_checkpoint_write",
    "n_body_sim_pro_cuda_checkpoint_read", "n_body_sim_pro_cuda_context_set_opening",
    "n_body_sim_pro_cuda_shard_begin", "n_body_sim_pro_cuda_shard_end",
    "n_body_sim_pro_cuda_plummer_collision_generate", "n_body_sim_pro_cuda_correction_evaluate",
    "n_body_sim_pro_cuda_context_set_relative_source",
)

# NBodySimProCudaMlpEngine
MLP_ENGINES = {"tcgen05": 0, "mma_sync": 1}

# NBodySimProSimulationPreset (generation/presets.h:27-38)
PRESETS = {"two_body": 0, "random_cloud": 1, "solar_system": 2, "open_cluster": 3,
           "globular_cluster": 4, "spiral_galaxy": 5, "elliptical_galaxy": 6,
           "galaxy_collision": 7, "triple_galaxy": 8}


def kernel_launches() -> int:
    """CUDA kernels this process has launched through the library."""
    return int(library().n_body_sim_pro_cuda_kernel_launches())


def measure_fp32_peak() -> dict:
    """Measured FFMA / FFMA2 TFLOP/s and MUFU rsqrt/s of the current GPU."""
    vals = [C.c_double(0.0) for _ in range(4)]
    err = Error()
    _check(library().n_body_sim_pro_cuda_measure_fp32_peak(*[C.byref(v) for v in vals],
                                                          C.byref(err)), err)
    return {"ffma_tflops": vals[0].value, "ffma2_tflops": vals[1].value,
            "rsqrt_per_s": vals[2].value, "sm_clock_mhz": vals[3].value}

_lib = None


def library() -> C.CDLL:
    """Load the in-tree shared library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m n_body_sim_pro_b200.build`")
    L = C.CDLL(LIB_PATH)
    pv, pg, pe, vp = C.POINTER(View), C.POINTER(Gravity), C.POINTER(Error), C.c_void_p
    st = C.c_int
    sig = {
        "n_body_sim_pro_cuda_context_create": (vp, [pe]),
        "n_body_sim_pro_cuda_context_destroy": (None, [vp]),
        "n_body_sim_pro_cuda_context_set_theta": (None, [vp, C.c_double]),
        "n_body_sim_pro_cuda_context_theta": (C.c_double, [vp]),
        "n_body_sim_pro_cuda_context_set_multipole_order": (st, [vp, C.c_int, pe]),
        "n_body_sim_pro_cuda_context_set_leaf_capacity": (st, [vp, C.c_int, pe]),
        "n_body_sim_pro_cuda_context_set_walk": (st, [vp, C.c_int, pe]),
        "n_body_sim_pro_cuda_context_set_opening": (st, [vp, C.c_int, pe]),
        "n_body_sim_pro_cuda_context_set_relative_opening": (st, [vp, C.c_double, pe]),
        "n_body_sim_pro_cuda_context_set_relative_source": (st, [vp, C.c_int, pe]),
        "n_body_sim_pro_cuda_context_stats": (C.c_int, [vp, C.POINTER(BarnesHutStats)]),
        "n_body_sim_pro_cuda_context_timings": (C.c_int, [vp, C.POINTER(Timings)]),
        "n_body_sim_pro_cuda_context_walk_restarts": (C.c_size_t, [vp]),
        "n_body_sim_pro_cuda_context_corrected_cells": (C.c_size_t, [vp]),
        "n_body_sim_pro_cuda_preset_generate_parallel": (C.c_int, [vp, C.c_int,
                                                                   C.POINTER(C.c_size_t * 2), pe]),
        "n_body_sim_pro_cuda_plummer_collision_generate": (st, [vp, C.c_size_t, C.c_uint64,
                                                                C.c_double, C.c_double,
                                                                C.c_double, pe]),
        "n_body_sim_pro_cuda_checkpoint_write": (C.c_int, [vp, C.c_char_p,
                                                           C.POINTER(CheckpointHeader), pe]),
        "n_body_sim_pro_cuda_checkpoint_read": (C.c_int, [vp, C.c_char_p,
                                                          C.POINTER(CheckpointHeader), pe]),
        "n_body_sim_pro_gravity_compute_acceleration_cuda": (st, [pv, pg, vp, pe]),
        "n_body_sim_pro_barnes_hut_compute_acceleration_cuda": (st, [pv, pg, vp, pe]),
        "n_body_sim_pro_cuda_upload": (st, [vp, pv, pe]),
        "n_body_sim_pro_cuda_download": (st, [vp, pv, pe]),
        "n_body_sim_pro_cuda_compute_acceleration": (st, [vp, pg, C.c_int, pe]),
        "n_body_sim_pro_cuda_advance": (st, [vp, pg, C.c_int, C.c_double, C.c_int, C.c_int, pe]),
        "n_body_sim_pro_cuda_shard_begin": (st, [vp, C.c_double, C.POINTER(C.c_double), vp,
                                                 C.c_size_t, pe]),
        "n_body_sim_pro_cuda_shard_end": (st, [vp, pg, C.c_double, vp, C.c_size_t, C.c_size_t,
                                               pe]),
        "n_body_sim_pro_cuda_diagnostics": (st, [vp, pg, C.POINTER(DiagnosticsQuantities),
                                                 C.POINTER(C.c_double), pe]),
        "n_body_sim_pro_cuda_reference_acceleration": (st, [vp, pg, C.POINTER(C.c_int64),
                                                            C.c_size_t, C.POINTER(C.c_double), pe]),
        "n_body_sim_pro_cuda_morton_order": (st, [vp, C.POINTER(C.c_uint64),
                                                  C.POINTER(C.c_uint64), C.POINTER(C.c_double),
                                                  pe]),
        "n_body_sim_pro_cuda_synchronize": (st, [vp, pe]),
        "n_body_sim_pro_cuda_architecture": (C.c_char_p, []),
        "n_body_sim_pro_cuda_kernel_launches": (C.c_ulonglong, []),
        "n_body_sim_pro_cuda_ensemble_create": (vp, [pe]),
        "n_body_sim_pro_cuda_ensemble_destroy": (None, [vp]),
        "n_body_sim_pro_cuda_ensemble_upload": (st, [vp, pv, C.POINTER(C.c_uint64), C.c_size_t,
                                                     pe]),
        "n_body_sim_pro_cuda_ensemble_download": (st, [vp, pv, pe]),
        "n_body_sim_pro_cuda_ensemble_autotune": (st, [vp, pg, C.c_double, pe]),
        "n_body_sim_pro_cuda_ensemble_advance": (st, [vp, pg, C.c_double, C.c_int, C.c_int, pe]),
        "n_body_sim_pro_cuda_ensemble_info": (st, [vp, C.POINTER(EnsembleInfo), pe]),
        "n_body_sim_pro_cuda_measure_fp32_peak": (st, [C.POINTER(C.c_double)] * 4 + [pe]),
        "n_body_sim_pro_cuda_correction_create": (vp, [C.c_uint64, pe]),
        "n_body_sim_pro_cuda_correction_destroy": (None, [vp]),
        "n_body_sim_pro_cuda_correction_generate": (st, [vp, vp, pg, C.c_double, C.c_size_t,
                                                         C.c_uint64, pe]),
        "n_body_sim_pro_cuda_correction_train": (st, [vp, C.c_int, C.c_int, C.c_double,
                                                      C.POINTER(C.c_double),
                                                      C.POINTER(C.c_double), pe]),
        "n_body_sim_pro_cuda_correction_get_parameters": (st, [vp, C.POINTER(C.c_float),
                                                               C.POINTER(C.c_float), pe]),
        "n_body_sim_pro_cuda_correction_set_parameters": (st, [vp, C.POINTER(C.c_float),
                                                               C.POINTER(C.c_float), pe]),
        "n_body_sim_pro_cuda_correction_gradient": (st, [vp, C.POINTER(C.c_float),
                                                         C.POINTER(C.c_float), C.c_size_t,
                                                         C.POINTER(C.c_float),
                                                         C.POINTER(C.c_double), pe]),
        "n_body_sim_pro_cuda_correction_samples": (st, [vp, C.POINTER(C.c_size_t),
                                                        C.POINTER(C.c_float),
                                                        C.POINTER(C.c_float), C.c_size_t, pe]),
        "n_body_sim_pro_cuda_context_set_correction": (st, [vp, vp, pe]),
        "n_body_sim_pro_cuda_correction_evaluate": (st, [vp, C.POINTER(C.c_float), C.c_size_t,
                                                         C.POINTER(C.c_float), C.c_int, pe]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    _lib = L
    return L


def _check(status: int, err: Error) -> None:
    if status != Status.OK:
        raise CudaError(status, err.message.decode(errors="replace"))


# ---------------------------------------------------------------------------
# particle storage
# ---------------------------------------------------------------------------

_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")


@dataclass
class ParticleSystem:
    """SoA float64 storage with the reference's field set; ``view()`` gives the
    NBodySimProParticleSystemView the C ABI takes.  Arrays may be numpy arrays
    in pinned memory (see :func:`pinned_empty`)."""

    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    ax: np.ndarray
    ay: np.ndarray
    az: np.ndarray
    m: np.ndarray

    @classmethod
    def zeros(cls, n: int, allocator=None) -> "ParticleSystem":
        alloc = allocator or (lambda k: np.zeros(k, dtype=np.float64))
        return cls(*[alloc(n) for _ in _FIELDS])

    @classmethod
    def from_arrays(cls, pos: np.ndarray, vel: np.ndarray, mass: np.ndarray,
                    acc: np.ndarray | None = None) -> "ParticleSystem":
        n = mass.shape[0]
        acc = np.zeros((n, 3)) if acc is None else acc
        cols = [np.ascontiguousarray(a, dtype=np.float64)
                for a in (pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2],
                          acc[:, 0], acc[:, 1], acc[:, 2], mass)]
        return cls(*cols)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def view(self) -> View:
        for f in _FIELDS:
            a = getattr(self, f)
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError(f"field {f} must be contiguous float64")
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        return View(self.n, *[p(getattr(self, f)) for f in _FIELDS])

    def acc(self) -> np.ndarray:
        return np.stack([self.ax, self.ay, self.az], axis=1)

    def copy(self) -> "ParticleSystem":
        return ParticleSystem(*[getattr(self, f).copy() for f in _FIELDS])


# ---------------------------------------------------------------------------
# force functions (NBodySimProForceFunction)
# ---------------------------------------------------------------------------

def _force(name: str, system: ParticleSystem, gravity: Gravity, context) -> np.ndarray:
    L = library()
    err = Error()
    v = system.view()
    ctx = context.handle if isinstance(context, CudaContext) else context
    _check(getattr(L, name)(C.byref(v), C.byref(gravity), ctx, C.byref(err)), err)
    return system.acc()


def n_body_sim_pro_gravity_compute_acceleration_cuda(system: ParticleSystem, gravity: Gravity,
                                                     context=None) -> np.ndarray:
    """`cuda` algorithm: exact all-pairs forces written into system.ax/ay/az."""
    return _force("n_body_sim_pro_gravity_compute_acceleration_cuda", system, gravity, context)


def n_body_sim_pro_barnes_hut_compute_acceleration_cuda(system: ParticleSystem, gravity: Gravity,
                                                        context=None) -> np.ndarray:
    """`barnes_hut_cuda` algorithm: GPU Barnes-Hut forces into system.ax/ay/az."""
    return _force("n_body_sim_pro_barnes_hut_compute_acceleration_cuda", system, gravity, context)


class CudaContext:
    """NBodySimProCudaContext: device-resident state, stepping and diagnostics."""

    def __init__(self, theta: float | None = None, multipole_order: int | None = None,
                 leaf_capacity: int | None = None, opening: int | None = None,
                 relative_opening: float | None = None):
        L = library()
        err = Error()
        h = L.n_body_sim_pro_cuda_context_create(C.byref(err))
        if not h:
            raise CudaError(err.status or Status.UNSUPPORTED_PLATFORM,
                            err.message.decode(errors="replace"))
        self.handle = C.c_void_p(h)
        self.n = 0
        if theta is not None:
            self.theta = theta
        if multipole_order is not None:
            self.set_multipole_order(multipole_order)
        if leaf_capacity is not None:
            self.set_leaf_capacity(leaf_capacity)
        if opening is not None:
            self.set_opening(opening)
        if relative_opening is not None:
            self.set_relative_opening(relative_opening)

    def close(self) -> None:
        if getattr(self, "handle", None):
            library().n_body_sim_pro_cuda_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def theta(self) -> float:
        return library().n_body_sim_pro_cuda_context_theta(self.handle)

    @theta.setter
    def theta(self, value: float) -> None:
        library().n_body_sim_pro_cuda_context_set_theta(self.handle, float(value))

    def set_multipole_order(self, order: int) -> None:
        err = Error()
        _check(library().n_body_sim_pro_cuda_context_set_multipole_order(self.handle, order,
                                                                         C.byref(err)), err)

    def set_walk(self, walk: int) -> None:
        """0: stackless skip-link walk; 1: interaction-list walk (default); 2: the
        interaction-list walk with the top of the tree shared by 4 groups."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_context_set_walk(self.handle, int(walk),
                                                              C.byref(err)), err)

    def set_opening(self, opening: int) -> None:
        """Opening.REFERENCE: (2h)^2 < theta^2 d^2 (default); Opening.OFFSET:
        2h / theta + shift < d with shift the cell's centre-of-mass offset."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_context_set_opening(self.handle, int(opening),
                                                                 C.byref(err)), err)

    def set_relative_opening(self, alpha: float) -> None:
        """Relative opening test G M (2h)^2 / d^4 <= alpha max(|a_old|, rms |a_old|)
        on top of the geometric one (alpha 0: off).  A state without previous
        accelerations is evaluated with the geometric test alone at
        min(theta, 0.5)."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_context_set_relative_opening(
            self.handle, float(alpha), C.byref(err)), err)

    def set_relative_source(self, source: int) -> None:
        """Where the plugin functions take the relative test's previous
        accelerations: RelativeSource.FROM_VIEW (default) or FROM_CONTEXT (this
        context's previous plugin result, kept on the device)."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_context_set_relative_source(
            self.handle, int(source), C.byref(err)), err)

    def set_correction(self, correction: "CudaCorrection | None") -> None:
        err = Error()
        h = correction.handle if correction is not None else None
        _check(library().n_body_sim_pro_cuda_context_set_correction(self.handle, h,
                                                                    C.byref(err)), err)

    def set_leaf_capacity(self, capacity: int) -> None:
        err = Error()
        _check(library().n_body_sim_pro_cuda_context_set_leaf_capacity(self.handle, capacity,
                                                                       C.byref(err)), err)

    def stats(self) -> dict:
        s = BarnesHutStats()
        if library().n_body_sim_pro_cuda_context_stats(self.handle, C.byref(s)) != 0:
            raise CudaError(Status.INVALID_ARGUMENT, "stats")
        return s.as_dict()

    def timings(self) -> dict:
        t = Timings()
        library().n_body_sim_pro_cuda_context_timings(self.handle, C.byref(t))
        return t.as_dict()

    def generate_preset(self, preset: "str | int", n: int, seed: int) -> None:
        """presets_parallel.c on the device: the preset becomes the resident state."""
        pid = PRESETS[preset] if isinstance(preset, str) else int(preset)
        params = (C.c_size_t * 2)(n, seed)
        err = Error()
        _check(library().n_body_sim_pro_cuda_preset_generate_parallel(self.handle, pid,
                                                                       C.byref(params),
                                                                       C.byref(err)), err)
        self.n = n

    def generate_plummer_collision(self, n: int, seed: int, scale_radius: float = 1.0,
                                   separation: float = 10.0, relative_speed: float = 0.3) -> None:
        """Two Plummer spheres (mass 1/2 each) from the parallel presets'
        per-particle streams, -/+ separation/2 on x, -/+ relative_speed/2 on y:
        the two-Plummer collision workload becomes the resident state."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_plummer_collision_generate(
            self.handle, n, seed, scale_radius, separation, relative_speed, C.byref(err)), err)
        self.n = n

    def checkpoint_write(self, path: str, header: CheckpointHeader) -> None:
        """The resident state to `path` in the reference's checkpoint format."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_checkpoint_write(
            self.handle, os.fsencode(path), C.byref(header), C.byref(err)), err)

    def checkpoint_read(self, path: str) -> CheckpointHeader:
        """A checkpoint file becomes the resident state; returns its header."""
        header = CheckpointHeader()
        err = Error()
        _check(library().n_body_sim_pro_cuda_checkpoint_read(
            self.handle, os.fsencode(path), C.byref(header), C.byref(err)), err)
        self.n = header.particle_count
        return header

    def walk_restarts(self) -> int:
        """Groups of the last Barnes-Hut evaluation that the interaction-list
        walk handed to the stackless walk (stack overflow)."""
        return int(library().n_body_sim_pro_cuda_context_walk_restarts(self.handle))

    def corrected_cells(self) -> int:
        """(cell, 32-target group) pairs the correction network evaluated in the
        last Barnes-Hut evaluation."""
        return int(library().n_body_sim_pro_cuda_context_corrected_cells(self.handle))

    def upload(self, system: ParticleSystem) -> None:
        err = Error()
        v = system.view()
        _check(library().n_body_sim_pro_cuda_upload(self.handle, C.byref(v), C.byref(err)), err)
        self.n = system.n

    def download(self, system: ParticleSystem) -> None:
        err = Error()
        v = system.view()
        _check(library().n_body_sim_pro_cuda_download(self.handle, C.byref(v), C.byref(err)), err)

    def download_accelerations(self) -> np.ndarray:
        """Only the resident accelerations, (n, 3) float64 (the view's other
        arrays are NULL, which download skips)."""
        out = np.zeros((3, self.n), dtype=np.float64)
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        null = C.POINTER(C.c_double)()
        v = View(self.n, null, null, null, null, null, null, p(out[0]), p(out[1]), p(out[2]), null)
        err = Error()
        _check(library().n_body_sim_pro_cuda_download(self.handle, C.byref(v), C.byref(err)), err)
        return out.T.copy()

    def compute_acceleration(self, gravity: Gravity, algorithm: Algorithm) -> None:
        err = Error()
        _check(library().n_body_sim_pro_cuda_compute_acceleration(
            self.handle, C.byref(gravity), int(algorithm), C.byref(err)), err)

    def advance(self, gravity: Gravity, timestep: float, steps: int,
                algorithm: Algorithm = Algorithm.ALL_PAIRS,
                integrator: Integrator = Integrator.LEAPFROG) -> None:
        err = Error()
        _check(library().n_body_sim_pro_cuda_advance(self.handle, C.byref(gravity),
                                                     int(integrator), float(timestep), int(steps),
                                                     int(algorithm), C.byref(err)), err)

    def shard_begin(self, timestep: float, centre, slice_ptr: int, slice_capacity: int) -> None:
        """Opening kick + drift of the resident slice, then its packed sources
        into the device buffer at `slice_ptr` (slice_capacity float4 entries)."""
        c3 = (C.c_double * 3)(*[float(v) for v in centre])
        err = Error()
        _check(library().n_body_sim_pro_cuda_shard_begin(self.handle, float(timestep), c3,
                                                         C.c_void_p(int(slice_ptr)),
                                                         int(slice_capacity), C.byref(err)), err)

    def shard_end(self, gravity: Gravity, timestep: float, sources_ptr: int, source_count: int,
                  slice_offset: int) -> None:
        """Forces of the resident slice from all gathered sources, then the
        closing kick."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_shard_end(self.handle, C.byref(gravity),
                                                       float(timestep),
                                                       C.c_void_p(int(sources_ptr)),
                                                       int(source_count), int(slice_offset),
                                                       C.byref(err)), err)

    def diagnostics(self, gravity: Gravity | None = None, potential: bool = False):
        err = Error()
        q = DiagnosticsQuantities()
        pe = C.c_double(0.0)
        g = C.byref(gravity) if gravity is not None else None
        _check(library().n_body_sim_pro_cuda_diagnostics(self.handle, g, C.byref(q),
                                                         C.byref(pe) if potential else None,
                                                         C.byref(err)), err)
        return (q.as_array(), pe.value) if potential else q.as_array()

    def reference_acceleration(self, gravity: Gravity, targets: np.ndarray) -> np.ndarray:
        t = np.ascontiguousarray(targets, dtype=np.int64)
        out = np.zeros((t.shape[0], 3), dtype=np.float64)
        err = Error()
        _check(library().n_body_sim_pro_cuda_reference_acceleration(
            self.handle, C.byref(gravity), t.ctypes.data_as(C.POINTER(C.c_int64)), t.shape[0],
            out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(err)), err)
        return out

    def morton_order(self):
        keys = np.zeros(self.n, dtype=np.uint64)
        perm = np.zeros(self.n, dtype=np.uint64)
        root = np.zeros(4, dtype=np.float64)
        err = Error()
        _check(library().n_body_sim_pro_cuda_morton_order(
            self.handle, keys.ctypes.data_as(C.POINTER(C.c_uint64)),
            perm.ctypes.data_as(C.POINTER(C.c_uint64)),
            root.ctypes.data_as(C.POINTER(C.c_double)), C.byref(err)), err)
        return keys, perm, root

    def synchronize(self) -> None:
        err = Error()
        _check(library().n_body_sim_pro_cuda_synchronize(self.handle, C.byref(err)), err)


class CudaEnsemble:
    """NBodySimProCudaEnsemble: many independent systems advanced together."""

    def __init__(self):
        L = library()
        err = Error()
        h = L.n_body_sim_pro_cuda_ensemble_create(C.byref(err))
        if not h:
            raise CudaError(err.status or Status.UNSUPPORTED_PLATFORM,
                            err.message.decode(errors="replace"))
        self.handle = C.c_void_p(h)
        self.offsets = None

    def close(self) -> None:
        if getattr(self, "handle", None):
            library().n_body_sim_pro_cuda_ensemble_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, system: ParticleSystem, offsets) -> None:
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        err = Error()
        v = system.view()
        _check(library().n_body_sim_pro_cuda_ensemble_upload(
            self.handle, C.byref(v), off.ctypes.data_as(C.POINTER(C.c_uint64)), off.shape[0] - 1,
            C.byref(err)), err)
        self.offsets = off

    def download(self, system: ParticleSystem) -> None:
        err = Error()
        v = system.view()
        _check(library().n_body_sim_pro_cuda_ensemble_download(self.handle, C.byref(v),
                                                               C.byref(err)), err)

    def autotune(self, gravity: Gravity, timestep: float) -> None:
        err = Error()
        _check(library().n_body_sim_pro_cuda_ensemble_autotune(self.handle, C.byref(gravity),
                                                               float(timestep), C.byref(err)), err)

    def advance(self, gravity: Gravity, timestep: float, steps: int,
                one_launch_per_system: bool = False) -> float:
        """Advance every system; returns the device milliseconds of the call."""
        err = Error()
        _check(library().n_body_sim_pro_cuda_ensemble_advance(
            self.handle, C.byref(gravity), float(timestep), int(steps),
            1 if one_launch_per_system else 0, C.byref(err)), err)
        return self.info()["last_advance_ms"]

    def info(self) -> dict:
        i = EnsembleInfo()
        err = Error()
        _check(library().n_body_sim_pro_cuda_ensemble_info(self.handle, C.byref(i), C.byref(err)),
               err)
        return i.as_dict()


CORRECTION_PARAMETERS = 5059
CORRECTION_SCALING = 46


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class CudaCorrection:
    """NBodySimProCudaCorrection: the learned far-field correction MLP."""

    def __init__(self, seed: int = 1):
        err = Error()
        h = library().n_body_sim_pro_cuda_correction_create(seed, C.byref(err))
        if not h:
            raise CudaError(err.status or Status.UNSUPPORTED_PLATFORM,
                            err.message.decode(errors="replace"))
        self.handle = C.c_void_p(h)

    def close(self) -> None:
        if getattr(self, "handle", None):
            library().n_body_sim_pro_cuda_correction_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def generate(self, context: CudaContext, gravity: Gravity, theta: float, samples: int,
                 seed: int = 7) -> None:
        err = Error()
        _check(library().n_body_sim_pro_cuda_correction_generate(
            self.handle, context.handle, C.byref(gravity), float(theta), int(samples), seed,
            C.byref(err)), err)

    def train(self, epochs: int, batch: int = 4096, learning_rate: float = 1e-3):
        tl = np.zeros(max(epochs, 1))
        vl = np.zeros(max(epochs, 1))
        err = Error()
        _check(library().n_body_sim_pro_cuda_correction_train(
            self.handle, int(epochs), int(batch), float(learning_rate),
            tl.ctypes.data_as(C.POINTER(C.c_double)), vl.ctypes.data_as(C.POINTER(C.c_double)),
            C.byref(err)), err)
        return tl[:epochs], vl[:epochs]

    def parameters(self):
        p = np.zeros(CORRECTION_PARAMETERS, dtype=np.float32)
        s = np.zeros(CORRECTION_SCALING, dtype=np.float32)
        err = Error()
        _check(library().n_body_sim_pro_cuda_correction_get_parameters(
            self.handle, _fptr(p), _fptr(s), C.byref(err)), err)
        return p, s

    def set_parameters(self, params=None, scaling=None) -> None:
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        s = None if scaling is None else np.ascontiguousarray(scaling, dtype=np.float32)
        err = Error()
        _check(library().n_body_sim_pro_cuda_correction_set_parameters(
            self.handle, None if p is None else _fptr(p), None if s is None else _fptr(s),
            C.byref(err)), err)

    def gradient(self, features: np.ndarray, labels: np.ndarray):
        x = np.ascontiguousarray(features, dtype=np.float32)
        y = np.ascontiguousarray(labels, dtype=np.float32)
        g = np.zeros(CORRECTION_PARAMETERS, dtype=np.float32)
        loss = C.c_double(0.0)
        err = Error()
        _check(library().n_body_sim_pro_cuda_correction_gradient(
            self.handle, _fptr(x), _fptr(y), x.shape[0], _fptr(g), C.byref(loss), C.byref(err)),
            err)
        return g, loss.value

    def evaluate(self, features: np.ndarray, engine: str = "tcgen05") -> np.ndarray:
        """The network on raw feature rows (n x 10) -> outputs (n x 3), on the
        tcgen05 tensor cores ("tcgen05") or with warp-level mma.sync ("mma_sync")."""
        x = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros((x.shape[0], 3), dtype=np.float32)
        err = Error()
        _check(library().n_body_sim_pro_cuda_correction_evaluate(
            self.handle, _fptr(x), x.shape[0], _fptr(out), MLP_ENGINES[engine], C.byref(err)),
            err)
        return out

    def samples(self, max_rows: int = 1 << 20):
        rows = C.c_size_t(0)
        f = np.zeros((max_rows, 10), dtype=np.float32)
        lab = np.zeros((max_rows, 3), dtype=np.float32)
        err = Error()
        _check(library().n_body_sim_pro_cuda_correction_samples(
            self.handle, C.byref(rows), _fptr(f), _fptr(lab), max_rows, C.byref(err)), err)
        k = min(rows.value, max_rows)
        return f[:k], lab[:k], rows.value
