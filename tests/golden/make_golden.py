"""Generate the golden fixtures of tests/golden/ from the REFERENCE engine itself.

Runs oracle/_ref/libnbody_ref.so (the reference's own C sources compiled by
``make -C oracle ref``) — never the restatement — so the fixtures pin the
oracle restatement to the reference even where the reference is not built.

    python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
import oracle as O  # noqa: E402


def main() -> None:
    if not O.ref_available():
        O.build(ref=True)
    R = O.ref()
    g = O.Gravity()
    err = O.Error()

    # globular cluster (Plummer a=1, M=1), N=2048, seed 42, eps 0.01
    p = O.ref_preset("globular_cluster", 2048, 42)
    out = {f: getattr(p, f).copy() for f in ("x", "y", "z", "vx", "vy", "vz", "m")}
    out["acc"] = O.ref_gravity(p, 1.0, 0.01).copy()
    R.n_body_sim_pro_gravity_init(C.byref(g), 1.0, 0.01)
    pe = C.c_double()
    v = p.view()
    R.n_body_sim_pro_diagnostics_compute_potential_energy(C.byref(v), C.byref(g), C.byref(pe),
                                                          C.byref(err))
    out["potential"] = np.float64(pe.value)
    force = C.cast(R.n_body_sim_pro_gravity_compute_acceleration_reference, C.c_void_p)
    for _ in range(3):
        assert R.n_body_sim_pro_integrator_advance(C.byref(v), C.byref(g), 1, 1e-3, force, None,
                                                   C.byref(err)) == 0
    out["pos_after_3"] = p.pos()
    d = (C.c_double * 11)()
    R.n_body_sim_pro_diagnostics_compute_global(C.byref(v), C.byref(d), C.byref(err))
    out["diag_after_3"] = np.array(d[:])
    np.savez_compressed(os.path.join(HERE, "plummer_2048.npz"), **out)

    # Morton keys / permutation / root cube
    m = {}
    for tag, name, n, seed in (("cloud", "random_cloud", 4096, 42),
                               ("collision", "plummer_collision", 8192, 42)):
        # the collision preset exists only in the restatement; its positions are
        # plain inputs here, the keys and permutation come from the reference
        q = O.ref_preset(name, n, seed) if name != "plummer_collision" else O.preset(name, n, seed)
        k, perm, root = O.ref_morton_order(q)
        m[f"{tag}_keys"], m[f"{tag}_perm"], m[f"{tag}_root"] = k, perm, root
    np.savez_compressed(os.path.join(HERE, "morton.npz"), **m)

    # Barnes-Hut, random cloud N=400 seed 7, eps 0.02, theta 0.7
    q = O.ref_preset("random_cloud", 400, 7)
    a, s = O.ref_barnes_hut(q, 1.0, 0.02, 0.7)
    np.savez_compressed(os.path.join(HERE, "barnes_hut.npz"), acc_theta07=a,
                        stats_theta07=np.array([s[k] for k in (
                            "node_count", "leaf_count", "internal_node_count",
                            "accepted_approximations", "exact_interactions", "maximum_depth")],
                            dtype=np.int64))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
