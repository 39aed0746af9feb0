"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of bench.py import this module, and only as the
checker or the timed CPU baseline.  The product package never imports it.

Two libraries sit behind it:

* ``oracle/liboracle.so`` — the C restatement (nbody_oracle.c), always built;
* ``oracle/_ref/libnbody_ref.so`` — the reference engine compiled from its own
  sources by ``make -C oracle ref`` (present when the reference checkout was
  available at build time; the built file travels with the repository).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnbody_ref.so")
REF_BENCH = os.path.join(HERE, "_ref", "n_body_sim_pro_benchmark")


class View(C.Structure):
    """Same field order as the reference's NBodySimProParticleSystemView
    (include/n_body_sim_pro/core/particle_system.h:38-50)."""

    _fields_ = [("particle_count", C.c_size_t)] + [
        (name, C.POINTER(C.c_double))
        for name in (
            "positions_x", "positions_y", "positions_z",
            "velocities_x", "velocities_y", "velocities_z",
            "accelerations_x", "accelerations_y", "accelerations_z",
            "masses",
        )
    ]


class Gravity(C.Structure):
    """NBodySimProGravity (include/n_body_sim_pro/physics/gravity.h:25-29)."""

    _fields_ = [("gravitational_constant", C.c_double), ("softening_length", C.c_double),
                ("softening_squared", C.c_double)]


class Error(C.Structure):
    """NBodySimProError (include/n_body_sim_pro/core/status.h:30-35)."""

    _fields_ = [("status", C.c_int), ("source_file", C.c_char_p), ("source_line", C.c_int),
                ("message", C.c_char * 256)]


class BHStats(C.Structure):
    """NBodySimProBarnesHutStats (include/n_body_sim_pro/barnes_hut/barnes_hut.h:31-40)."""

    _fields_ = [(n, C.c_size_t) for n in ("node_count", "leaf_count", "internal_node_count",
                                          "accepted_approximations", "exact_interactions",
                                          "maximum_depth")] + [
        ("build_time_seconds", C.c_double), ("evaluation_time_seconds", C.c_double)]


FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")


@dataclass
class Particles:
    """SoA float64 particle storage; ``view()`` exposes it to the C libraries."""

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
    def zeros(cls, n: int) -> "Particles":
        return cls(*[np.zeros(n, dtype=np.float64) for _ in FIELDS])

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def copy(self) -> "Particles":
        return Particles(*[getattr(self, f).copy() for f in FIELDS])

    def view(self) -> View:
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        return View(self.n, p(self.x), p(self.y), p(self.z), p(self.vx), p(self.vy), p(self.vz),
                    p(self.ax), p(self.ay), p(self.az), p(self.m))

    def acc(self) -> np.ndarray:
        return np.stack([self.ax, self.ay, self.az], axis=1)

    def pos(self) -> np.ndarray:
        return np.stack([self.x, self.y, self.z], axis=1)


def build(ref: bool = True, reference_dir: str | None = None) -> None:
    """Compile the restatement and, when a reference checkout is given
    (`reference_dir`, else the environment variable NBSP_REFERENCE_DIR) and
    holds its C sources, the reference engine into _ref/."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    reference_dir = reference_dir or os.environ.get("NBSP_REFERENCE_DIR")
    if ref and reference_dir and os.path.isdir(os.path.join(reference_dir, "src", "c")):
        refdef = "REF=" + os.path.abspath(reference_dir)
        subprocess.run(["make", "-s", "-C", HERE, "-j8", refdef, "ref"], check=True)
        # the reference's force benchmark with the two CUDA algorithms (needs
        # the B200 library, built first by the package's own build step)
        if os.path.exists(os.path.join(HERE, "..", "n_body_sim_pro_b200", "lib",
                                       "libn_body_sim_pro_cuda.so")):
            subprocess.run(["make", "-s", "-C", HERE, refdef, "integrated"], check=True)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        pv = C.POINTER(View)
        d, u64, sz, i64p = C.c_double, C.c_uint64, C.c_size_t, C.POINTER(C.c_int64)
        sig = {
            "oracle_preset_two_body": (C.c_int, [pv]),
            "oracle_preset_random_cloud": (C.c_int, [pv, u64]),
            "oracle_preset_globular_cluster": (C.c_int, [pv, u64]),
            "oracle_preset_spiral_galaxy": (C.c_int, [pv, u64]),
            "oracle_preset_plummer_collision": (C.c_int, [pv, u64, d, d, d]),
            "oracle_preset_plummer_collision_parallel": (C.c_int, [pv, u64, d, d, d]),
            "oracle_preset_uniform_log_mass": (C.c_int, [pv, u64]),
            "oracle_ensemble_member_size": (sz, [u64, u64, sz, sz]),
            "oracle_ensemble_member_generate": (C.c_int, [pv, u64, u64, sz, sz]),
            "oracle_gravity_reference": (None, [pv, d, d]),
            "oracle_gravity_openmp": (None, [pv, d, d]),
            "oracle_gravity_subset": (None, [pv, d, d, i64p, sz, C.POINTER(d)]),
            "oracle_integrator_advance": (C.c_int, [pv, d, d, C.c_int, d, C.c_int, d]),
            "oracle_diagnostics_global": (None, [pv, C.POINTER(d)]),
            "oracle_potential_energy": (d, [pv, d, d]),
            "oracle_potential_energy_openmp": (d, [pv, d, d]),
            "oracle_morton_order": (C.c_int, [pv, C.POINTER(u64), C.POINTER(u64), C.POINTER(d)]),
            "oracle_barnes_hut": (C.c_int, [pv, d, d, d, C.POINTER(u64)]),
            "oracle_barnes_hut_residual_bands": (C.c_int, [pv, d, d, d, i64p, sz, C.c_int,
                                                           C.POINTER(d), C.POINTER(u64)]),
            "oracle_mix_seed": (u64, [u64, u64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> C.CDLL:
    """The reference engine compiled from its own sources (oracle/_ref)."""
    global _ref
    if _ref is None:
        R = C.CDLL(REF_SO)
        pv, pg, pe = C.POINTER(View), C.POINTER(Gravity), C.POINTER(Error)
        for name in ("n_body_sim_pro_gravity_compute_acceleration_reference",
                     "n_body_sim_pro_gravity_compute_acceleration_openmp",
                     "n_body_sim_pro_gravity_compute_acceleration_openmp_avx2",
                     "n_body_sim_pro_gravity_compute_acceleration_openmp_avx512",
                     "n_body_sim_pro_barnes_hut_compute_acceleration"):
            f = getattr(R, name)
            f.restype, f.argtypes = C.c_int, [pv, pg, C.c_void_p, pe]
        R.n_body_sim_pro_gravity_init.restype = None
        R.n_body_sim_pro_gravity_init.argtypes = [pg, C.c_double, C.c_double]
        R.n_body_sim_pro_barnes_hut_tree_create.restype = C.c_void_p
        R.n_body_sim_pro_barnes_hut_tree_create.argtypes = [pe]
        R.n_body_sim_pro_barnes_hut_tree_destroy.restype = None
        R.n_body_sim_pro_barnes_hut_tree_destroy.argtypes = [C.c_void_p]
        R.n_body_sim_pro_barnes_hut_tree_set_theta.restype = None
        R.n_body_sim_pro_barnes_hut_tree_set_theta.argtypes = [C.c_void_p, C.c_double]
        R.n_body_sim_pro_barnes_hut_tree_stats.restype = C.c_int
        R.n_body_sim_pro_barnes_hut_tree_stats.argtypes = [C.c_void_p, C.POINTER(BHStats)]
        R.n_body_sim_pro_integrator_advance.restype = C.c_int
        R.n_body_sim_pro_integrator_advance.argtypes = [pv, pg, C.c_int, C.c_double, C.c_void_p,
                                                        C.c_void_p, pe]
        R.n_body_sim_pro_diagnostics_compute_global.restype = C.c_int
        R.n_body_sim_pro_diagnostics_compute_global.argtypes = [pv, C.POINTER(C.c_double * 11), pe]
        R.n_body_sim_pro_diagnostics_compute_potential_energy.restype = C.c_int
        R.n_body_sim_pro_diagnostics_compute_potential_energy.argtypes = [pv, pg, C.POINTER(C.c_double), pe]
        R.n_body_sim_pro_particle_system_create.restype = C.c_void_p
        R.n_body_sim_pro_particle_system_create.argtypes = [C.c_size_t]
        R.n_body_sim_pro_particle_system_destroy.restype = None
        R.n_body_sim_pro_particle_system_destroy.argtypes = [C.c_void_p]
        R.n_body_sim_pro_particle_system_view.restype = C.c_int
        R.n_body_sim_pro_particle_system_view.argtypes = [C.c_void_p, pv, pe]
        R.n_body_sim_pro_preset_generate.restype = C.c_int
        R.n_body_sim_pro_preset_generate.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t * 2), pe]
        R.n_body_sim_pro_checkpoint_write.restype = C.c_int
        R.n_body_sim_pro_checkpoint_write.argtypes = [C.c_char_p, pv, C.POINTER(CheckpointHeader), pe]
        R.n_body_sim_pro_preset_generate_parallel.restype = C.c_int
        R.n_body_sim_pro_preset_generate_parallel.argtypes = [C.c_void_p, C.c_int,
                                                              C.POINTER(C.c_size_t * 2), pe]
        R.ref_shim_morton_order.restype = C.c_int
        R.ref_shim_morton_order.argtypes = [pv, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                            C.POINTER(C.c_double), C.POINTER(C.c_size_t)]
        _ref = R
    return _ref


# ---------------------------------------------------------------------------
# Presets (restatement)
# ---------------------------------------------------------------------------

PRESETS = {"two_body": 0, "random_cloud": 1, "globular_cluster": 4, "spiral_galaxy": 5}


def preset(name: str, n: int, seed: int) -> Particles:
    p = Particles.zeros(n)
    v = p.view()
    L = lib()
    if name == "two_body":
        rc = L.oracle_preset_two_body(C.byref(v))
    elif name == "random_cloud":
        rc = L.oracle_preset_random_cloud(C.byref(v), seed)
    elif name == "globular_cluster":
        rc = L.oracle_preset_globular_cluster(C.byref(v), seed)
    elif name == "spiral_galaxy":
        rc = L.oracle_preset_spiral_galaxy(C.byref(v), seed)
    elif name == "plummer_collision":
        rc = L.oracle_preset_plummer_collision(C.byref(v), seed, 1.0, 10.0, 0.3)
    elif name == "uniform_log_mass":
        rc = L.oracle_preset_uniform_log_mass(C.byref(v), seed)
    else:
        raise ValueError(name)
    if rc != 0:
        raise RuntimeError(f"oracle preset {name} failed ({rc})")
    return p


# NBodySimProSimulationPreset (include/n_body_sim_pro/generation/presets.h:27-38)
PRESET_IDS = {"two_body": 0, "random_cloud": 1, "solar_system": 2, "open_cluster": 3,
              "globular_cluster": 4, "spiral_galaxy": 5, "elliptical_galaxy": 6,
              "galaxy_collision": 7, "triple_galaxy": 8}


def preset_parallel(name: str, n: int, seed: int) -> Particles:
    """presets_parallel.c restated (per-particle generators seeded by index)."""
    p = Particles.zeros(n)
    v = p.view()
    if lib().oracle_preset_parallel(C.byref(v), PRESET_IDS[name], seed) != 0:
        raise RuntimeError(f"oracle parallel preset {name} failed")
    return p


def plummer_collision_parallel(n: int, seed: int, scale_radius: float = 1.0,
                               separation: float = 10.0, relative_speed: float = 0.3) -> Particles:
    """Two Plummer spheres in the parallel-preset form (per-particle streams,
    block b seeded with mix_seed(seed, b)): the two-Plummer collision workload."""
    p = Particles.zeros(n)
    v = p.view()
    if lib().oracle_preset_plummer_collision_parallel(C.byref(v), seed, scale_radius, separation,
                                                      relative_speed) != 0:
        raise RuntimeError("oracle plummer collision failed")
    return p


def filled_count(name: str, n: int) -> int:
    """Particles the parallel generator writes (galaxy_collision and
    triple_galaxy leave the last n % 2 / n % 3 untouched)."""
    if name == "galaxy_collision":
        return 2 * (n // 2)
    if name == "triple_galaxy":
        return 3 * (n // 3)
    return n


def ensemble_member(master_seed: int, k: int, lo: int = 32, hi: int = 4096) -> Particles:
    L = lib()
    n = L.oracle_ensemble_member_size(master_seed, k, lo, hi)
    p = Particles.zeros(n)
    v = p.view()
    if L.oracle_ensemble_member_generate(C.byref(v), master_seed, k, lo, hi) != 0:
        raise RuntimeError("ensemble member generation failed")
    return p


def ref_preset(name: str, n: int, seed: int, parallel: bool = False) -> Particles:
    """The same preset produced by the reference engine itself (`parallel`:
    n_body_sim_pro_preset_generate_parallel; unfilled entries come back as
    whatever the reference's allocation held)."""
    R = ref()
    ps = R.n_body_sim_pro_particle_system_create(n)
    err = Error()
    params = (C.c_size_t * 2)(n, seed)
    if parallel:
        rc = R.n_body_sim_pro_preset_generate_parallel(ps, PRESET_IDS[name], C.byref(params),
                                                       C.byref(err))
    else:
        rc = R.n_body_sim_pro_preset_generate(ps, PRESETS[name], C.byref(params), C.byref(err))
    if rc != 0:
        R.n_body_sim_pro_particle_system_destroy(ps)
        raise RuntimeError(f"reference preset failed: {err.message!r}")
    rv = View()
    R.n_body_sim_pro_particle_system_view(ps, C.byref(rv), C.byref(err))
    out = Particles.zeros(n)
    for f, name_ in zip(FIELDS, ("positions_x", "positions_y", "positions_z", "velocities_x",
                                 "velocities_y", "velocities_z", "accelerations_x",
                                 "accelerations_y", "accelerations_z", "masses")):
        src = np.ctypeslib.as_array(getattr(rv, name_), shape=(n,))
        getattr(out, f)[:] = src
    R.n_body_sim_pro_particle_system_destroy(ps)
    return out


# ---------------------------------------------------------------------------
# Forces, diagnostics, Morton order
# ---------------------------------------------------------------------------

def gravity_reference(p: Particles, G: float, eps: float, openmp: bool = False) -> np.ndarray:
    v = p.view()
    (lib().oracle_gravity_openmp if openmp else lib().oracle_gravity_reference)(C.byref(v), G, eps)
    return p.acc()


def gravity_subset(p: Particles, G: float, eps: float, targets: np.ndarray) -> np.ndarray:
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((t.shape[0], 3), dtype=np.float64)
    v = p.view()
    lib().oracle_gravity_subset(C.byref(v), G, eps, t.ctypes.data_as(C.POINTER(C.c_int64)),
                                t.shape[0], out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def diagnostics(p: Particles) -> np.ndarray:
    q = np.zeros(11, dtype=np.float64)
    v = p.view()
    lib().oracle_diagnostics_global(C.byref(v), q.ctypes.data_as(C.POINTER(C.c_double)))
    return q


def potential_energy(p: Particles, G: float, eps: float, openmp: bool = False) -> float:
    v = p.view()
    f = lib().oracle_potential_energy_openmp if openmp else lib().oracle_potential_energy
    return float(f(C.byref(v), G, eps))


def morton_order(p: Particles):
    n = p.n
    keys = np.zeros(n, dtype=np.uint64)
    perm = np.zeros(n, dtype=np.uint64)
    root = np.zeros(4, dtype=np.float64)
    v = p.view()
    rc = lib().oracle_morton_order(C.byref(v), keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                                   perm.ctypes.data_as(C.POINTER(C.c_uint64)),
                                   root.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError("oracle morton order failed")
    return keys, perm, root


def ref_morton_order(p: Particles):
    n = p.n
    keys = np.zeros(n, dtype=np.uint64)
    perm = np.zeros(n, dtype=np.uint64)
    root = np.zeros(4, dtype=np.float64)
    nodes = C.c_size_t(0)
    v = p.view()
    rc = ref().ref_shim_morton_order(C.byref(v), keys.ctypes.data_as(C.POINTER(C.c_uint64)),
                                     perm.ctypes.data_as(C.POINTER(C.c_uint64)),
                                     root.ctypes.data_as(C.POINTER(C.c_double)), C.byref(nodes))
    if rc not in (0, 6):  # 6: OVERFLOW from the insertion phase, keys still valid
        raise RuntimeError("reference morton order failed")
    return keys, perm, root


def barnes_hut(p: Particles, G: float, eps: float, theta: float):
    stats = np.zeros(6, dtype=np.uint64)
    v = p.view()
    rc = lib().oracle_barnes_hut(C.byref(v), G, eps, theta,
                                 stats.ctypes.data_as(C.POINTER(C.c_uint64)))
    if rc != 0:
        raise RuntimeError(f"oracle Barnes-Hut failed ({rc})")
    keys = ("node_count", "leaf_count", "internal_node_count", "accepted_approximations",
            "exact_interactions", "maximum_depth")
    return p.acc(), dict(zip(keys, (int(s) for s in stats)))


def barnes_hut_residual_bands(p: Particles, G: float, eps: float, theta: float,
                              targets: np.ndarray, bins: int):
    """The monopole error of the reference's walk at `theta` on each target,
    split by the apparent size (2h / d) / theta of the accepted cells:
    err[t, b, 3] (monopole minus the exact sum over the cell's particles) and
    count[t, b] (accepted cells).  err summed over the bins is the walk's force
    minus the direct sum."""
    tg = np.ascontiguousarray(targets, dtype=np.int64)
    err = np.zeros((len(tg), bins, 3))
    count = np.zeros((len(tg), bins), dtype=np.uint64)
    v = p.view()
    rc = lib().oracle_barnes_hut_residual_bands(
        C.byref(v), G, eps, theta, tg.ctypes.data_as(C.POINTER(C.c_int64)), len(tg), bins,
        err.ctypes.data_as(C.POINTER(C.c_double)), count.ctypes.data_as(C.POINTER(C.c_uint64)))
    if rc != 0:
        raise RuntimeError(f"oracle residual bands failed ({rc})")
    return err, count


def advance(p: Particles, G: float, eps: float, dt: float, steps: int, integrator: int = 1,
            force: int = 0, theta: float = 0.7) -> None:
    v = p.view()
    for _ in range(steps):
        rc = lib().oracle_integrator_advance(C.byref(v), G, eps, integrator, dt, force, theta)
        if rc != 0:
            raise RuntimeError(f"oracle integrator failed ({rc})")


def ref_gravity(p: Particles, G: float, eps: float, kind: str = "reference") -> np.ndarray:
    R = ref()
    g = Gravity()
    R.n_body_sim_pro_gravity_init(C.byref(g), G, eps)
    err = Error()
    v = p.view()
    f = getattr(R, f"n_body_sim_pro_gravity_compute_acceleration_{kind}")
    if f(C.byref(v), C.byref(g), None, C.byref(err)) != 0:
        raise RuntimeError(err.message)
    return p.acc()


def ref_barnes_hut(p: Particles, G: float, eps: float, theta: float):
    R = ref()
    g = Gravity()
    R.n_body_sim_pro_gravity_init(C.byref(g), G, eps)
    err = Error()
    tree = R.n_body_sim_pro_barnes_hut_tree_create(C.byref(err))
    R.n_body_sim_pro_barnes_hut_tree_set_theta(tree, theta)
    v = p.view()
    rc = R.n_body_sim_pro_barnes_hut_compute_acceleration(C.byref(v), C.byref(g), tree, C.byref(err))
    st = BHStats()
    R.n_body_sim_pro_barnes_hut_tree_stats(tree, C.byref(st))
    R.n_body_sim_pro_barnes_hut_tree_destroy(tree)
    if rc != 0:
        raise RuntimeError(err.message)
    return p.acc(), {f: int(getattr(st, f)) for f, _ in BHStats._fields_[:6]}


# ---------------------------------------------------------------------------
# Checkpoint files: src/c/checkpoint/checkpoint.c:9-76
# ---------------------------------------------------------------------------

class CheckpointHeader(C.Structure):
    """NBodySimProCheckpointHeader (include/n_body_sim_pro/checkpoint/checkpoint.h:29-40)."""

    _fields_ = [("magic", C.c_uint32), ("version", C.c_uint32), ("particle_count", C.c_size_t),
                ("simulation_time", C.c_double), ("timestep", C.c_double),
                ("integrator", C.c_int32), ("theta", C.c_double),
                ("barnes_hut_enabled", C.c_int32), ("random_seed", C.c_uint64),
                ("preset", C.c_int32)]


CHECKPOINT_MAGIC = 0x53504348   # checkpoint.h:27
CHECKPOINT_VERSION = 1


def checkpoint_bytes(header: CheckpointHeader, p: Particles) -> bytes:
    """The file n_body_sim_pro_checkpoint_write produces: magic and version
    (u32 each), the header struct as stored (padding included), then the ten
    FP64 arrays x y z vx vy vz ax ay az m (checkpoint.c:31-72)."""
    out = bytearray()
    out += np.uint32(CHECKPOINT_MAGIC).tobytes() + np.uint32(CHECKPOINT_VERSION).tobytes()
    out += bytes(header)
    for f in FIELDS:
        out += np.ascontiguousarray(getattr(p, f), dtype=np.float64).tobytes()
    return bytes(out)


def ref_checkpoint_write(path: str, header: CheckpointHeader, p: Particles) -> int:
    """The reference's own writer on the same state (status code)."""
    v = p.view()
    err = Error()
    return ref().n_body_sim_pro_checkpoint_write(os.fsencode(path), C.byref(v), C.byref(header),
                                                 C.byref(err))


def rms_relative_error(a: np.ndarray, ref_a: np.ndarray) -> float:
    """sqrt(sum|a - a_ref|^2 / sum|a_ref|^2) (tests/numerical/barnes_hut_test.c:38-57)."""
    den = float(np.sum(ref_a.astype(np.float64) ** 2))
    if den == 0.0:
        return 0.0
    return float(np.sqrt(np.sum((a.astype(np.float64) - ref_a) ** 2) / den))


def max_relative_error(a: np.ndarray, ref_a: np.ndarray) -> float:
    """Per component |a - ref| / (|ref| if |ref| > 1e-12 else 1)
    (tests/numerical/simd_equivalence_test.c:35-53)."""
    mag = np.abs(ref_a)
    scale = np.where(mag > 1e-12, mag, 1.0)
    return float(np.max(np.abs(a - ref_a) / scale)) if a.size else 0.0
