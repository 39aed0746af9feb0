"""`barnes_hut_cuda`: Morton order bit-exact with the reference, forces vs the
FP64 all-pairs oracle, statistics and determinism — mirroring the reference's
tests/numerical/barnes_hut_test.c and simd_equivalence_test.c:279-433.

Tolerances: the Morton keys and permutation must be EQUAL.  Forces: the
reference's own BH tests bound the rms relative error (barnes_hut_test.c:
38-57 metric) against the FP64 all-pairs kernel: theta 0.3 -> < 1e-2; the GPU
walk must also be no less accurate than the CPU reference BH at the same theta
(warp-coherent opening only ever opens more cells), with 1e-6 of slack for
FP32 arithmetic.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def to_system(nb, p):
    return nb.ParticleSystem(*[getattr(p, f).copy() for f in O.FIELDS])


WALKS = [0, 1, 2]  # stackless skip-link walk, interaction-list walk, lists with a shared top


@pytest.fixture(params=WALKS, ids=["stackless", "lists", "shared"])
def walk(request):
    return request.param


def bh(nb, p, eps, theta, ctx, order=1, leaf=16, walk=1, opening=0):
    ctx.theta = theta
    ctx.set_multipole_order(order)
    ctx.set_leaf_capacity(leaf)
    ctx.set_walk(walk)
    ctx.set_opening(opening)
    s = to_system(nb, p)
    a = nb.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, nb.gravity_init(1.0, eps), ctx)
    return a, ctx.stats()


# 5M keys: 1221 sort tiles of 4096, about four waves of tiles per pass, so
# most tiles find their offsets by looking back over tiles of earlier waves
@pytest.mark.parametrize("name,n,seed", [("random_cloud", 4096, 42), ("globular_cluster", 100000, 3),
                                         ("plummer_collision", 1000000, 42),
                                         ("plummer_collision", 5000000, 7),
                                         ("spiral_galaxy", 3000, 99), ("two_body", 2, 1),
                                         ("random_cloud", 5001, 8)])
def test_morton_order_bit_exact(cuda, ctx, name, n, seed):
    p = O.preset(name, n, seed)
    ctx.upload(to_system(cuda, p))
    k, perm, root = ctx.morton_order()
    k_ref, perm_ref, root_ref = O.morton_order(p)
    assert np.array_equal(root, root_ref)
    assert np.array_equal(k, k_ref)
    assert np.array_equal(perm, perm_ref)


def test_morton_golden_fixture(cuda, ctx):
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "morton.npz"))
    p = O.preset("plummer_collision", 8192, 42)
    ctx.upload(to_system(cuda, p))
    k, perm, root = ctx.morton_order()
    assert np.array_equal(k, g["collision_keys"]) and np.array_equal(perm, g["collision_perm"])
    assert np.array_equal(root, g["collision_root"])


def test_morton_ties_keep_index_order(cuda, ctx):
    p = O.preset("random_cloud", 256, 5)
    p.x[100:140] = p.x[7] + 1e-12 * np.arange(40)  # distinct positions, one Morton cell
    p.y[100:140] = p.y[7]
    p.z[100:140] = p.z[7]
    ctx.upload(to_system(cuda, p))
    k, perm, _ = ctx.morton_order()
    k_ref, perm_ref, _ = O.morton_order(p)
    assert np.array_equal(k, k_ref) and np.array_equal(perm, perm_ref)


def test_two_body_is_exact(cuda, ctx, walk):
    """barnes_hut_test.c:59-103: leaves only, 0 approximations, 2 exact."""
    p = O.preset("two_body", 2, 1)
    ref = O.gravity_reference(p.copy(), 1.0, 0.02)
    a, st = bh(cuda, p, 0.02, 0.7, ctx, leaf=1, walk=walk)
    assert O.rms_relative_error(a, ref) < 1e-6
    assert st["leaf_count"] == 2
    assert st["accepted_approximations"] == 0
    assert st["exact_interactions"] == 2


@pytest.mark.parametrize("leaf", [1, 16])
def test_theta_tradeoff_and_accuracy(cuda, ctx, leaf, walk):
    """barnes_hut_test.c:105-160: random cloud N=400 seed 7, eps 0.02."""
    p = O.preset("random_cloud", 400, 7)
    ref = O.gravity_reference(p.copy(), 1.0, 0.02)
    a3, s3 = bh(cuda, p, 0.02, 0.3, ctx, leaf=leaf, walk=walk)
    a12, s12 = bh(cuda, p, 0.02, 1.2, ctx, leaf=leaf, walk=walk)
    e3, e12 = O.rms_relative_error(a3, ref), O.rms_relative_error(a12, ref)
    assert e3 < 0.01
    assert e3 < e12
    w = lambda s: s["accepted_approximations"] + s["exact_interactions"]  # noqa: E731
    assert w(s3) > w(s12)


def test_tree_structure_and_determinism(cuda, ctx, walk):
    """barnes_hut_test.c:162-214: spiral galaxy N=400 seed 99, one particle per leaf."""
    p = O.preset("spiral_galaxy", 400, 99)
    a, st = bh(cuda, p, 0.05, 0.7, ctx, leaf=1, walk=walk)
    assert st["leaf_count"] == 400
    assert st["node_count"] <= 800
    assert st["internal_node_count"] > 0
    assert st["maximum_depth"] >= 2
    b, _ = bh(cuda, p, 0.05, 0.7, ctx, leaf=1, walk=walk)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7, 1.0])
def test_no_less_accurate_than_reference_barnes_hut(cuda, ctx, theta, walk):
    p = O.preset("globular_cluster", 20000, 4)
    ref = O.gravity_reference(p.copy(), 1.0, 0.01, openmp=True)
    cpu, _ = O.barnes_hut(p.copy(), 1.0, 0.01, theta)
    gpu, _ = bh(cuda, p, 0.01, theta, ctx, walk=walk)
    e_cpu, e_gpu = O.rms_relative_error(cpu, ref), O.rms_relative_error(gpu, ref)
    print(f"theta={theta} cpu={e_cpu:.3e} gpu={e_gpu:.3e}")
    assert e_gpu <= e_cpu + 1e-6


def test_quadrupole_is_more_accurate(cuda, ctx, walk):
    p = O.preset("globular_cluster", 20000, 4)
    ref = O.gravity_reference(p.copy(), 1.0, 0.01, openmp=True)
    mono, _ = bh(cuda, p, 0.01, 0.7, ctx, order=1, walk=walk)
    quad, _ = bh(cuda, p, 0.01, 0.7, ctx, order=2, walk=walk)
    e1, e2 = O.rms_relative_error(mono, ref), O.rms_relative_error(quad, ref)
    print(f"monopole={e1:.3e} quadrupole={e2:.3e}")
    assert e2 < 0.5 * e1


def test_quadrupoles_follow_the_walk_order(cuda, walk):
    """The monopole walk's build skips the quadrupoles; a context switched to the
    quadrupole walk (or back) must give, bit for bit, what a fresh context of
    that order gives."""
    p = O.preset("plummer_collision", 50000, 7)
    fresh = {}
    for order in (1, 2):
        with cuda.CudaContext() as c:
            fresh[order], _ = bh(cuda, p, 0.01, 0.7, c, order=order, walk=walk)
    with cuda.CudaContext() as c:
        for order in (1, 2, 1, 2):
            a, _ = bh(cuda, p, 0.01, 0.7, c, order=order, walk=walk)
            assert np.array_equal(a, fresh[order]), order
    assert not np.array_equal(fresh[1], fresh[2])


def test_collision_config_accuracy(cuda, ctx, walk):
    """Config-2 shape at N=200k: two Plummer spheres 10 apart, eps 0.01, theta 0.7,
    vs the FP64 oracle on 1024 seeded targets."""
    p = O.preset("plummer_collision", 200000, 42)
    targets = np.random.default_rng(2).choice(p.n, 1024, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, targets)
    a, st = bh(cuda, p, 0.01, 0.7, ctx, walk=walk)
    e1 = O.rms_relative_error(a[targets], ref)
    a2, _ = bh(cuda, p, 0.01, 0.7, ctx, order=2, walk=walk)
    e2 = O.rms_relative_error(a2[targets], ref)
    print(f"collision200k mono={e1:.3e} quad={e2:.3e} stats={st}")
    assert e1 < 1e-2 and e2 < e1


def test_collision_1m_config_accuracy(cuda, ctx):
    """Config 2 at its full size: the 1M two-Plummer collision from the
    reference's parallel-preset streams, eps 0.01, theta 0.7, against the FP64
    oracle on 4096 seeded targets; and the relative opening test (alpha 0.0015,
    32-particle buckets, theta-1.0 safety bound) within the 1e-3 rms of the
    headline metric (measured on this state: alpha 0.004 gives 1.2e-3)."""
    n = 1_000_000
    ctx.generate_plummer_collision(n, 42)
    s = cuda.ParticleSystem.zeros(n)
    ctx.download(s)
    p = O.Particles.zeros(n)
    for f in O.FIELDS:
        getattr(p, f)[:] = getattr(s, f)
    targets = np.random.default_rng(11).choice(n, 4096, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, targets)
    g = cuda.gravity_init(1.0, 0.01)
    ctx.theta = 0.7
    ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
    a = ctx.download_accelerations()[targets]
    e_plain = O.rms_relative_error(a, ref)
    m_plain = float(np.max(np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)))
    ctx.theta = 1.0
    ctx.set_leaf_capacity(32)
    ctx.set_relative_opening(0.0015)
    ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)  # a_old: the theta-0.7 forces
    ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
    a_rel = ctx.download_accelerations()[targets]
    e_rel = O.rms_relative_error(a_rel, ref)
    print(f"collision1M theta0.7 rms={e_plain:.3e} max={m_plain:.3e} relative rms={e_rel:.3e}")
    assert e_plain < 2.5e-3 and m_plain < 0.1
    assert e_rel <= 1e-3


def test_headline_configuration_10m_accuracy(cuda, ctx):
    """The headline workload at its full size: the 10M two-Plummer collision
    from the reference's preset streams, against the FP64 oracle (gravity.c's
    sum restated) on the bench's 4096 seeded targets.  The method the matched
    study chooses — the relative opening test at alpha 0.0045 with the
    geometric test at theta 5.0 as the bound, 32-particle buckets, evaluated
    twice so the test reads the previous forces as in a run — holds rms <= 1e-3,
    and so does the plain walk at theta 0.5 it is compared with.  The first
    evaluation of the fresh state (no previous forces: the geometric test at
    the start angle 0.5) holds it too."""
    n = 10_000_000
    ctx.generate_plummer_collision(n, 42)
    s = cuda.ParticleSystem.zeros(n)
    ctx.download(s)
    p = O.Particles.zeros(n)
    for f in O.FIELDS:
        getattr(p, f)[:] = getattr(s, f)
    targets = np.random.default_rng(11).choice(n, 4096, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, targets)
    g = cuda.gravity_init(1.0, 0.01)
    ctx.theta = 0.5
    ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
    a_plain = ctx.download_accelerations()[targets]
    ctx.upload(s)  # the generated state again: accelerations zero
    ctx.theta = 5.0
    ctx.set_leaf_capacity(32)
    ctx.set_relative_opening(0.0045)
    ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
    a_first = ctx.download_accelerations()[targets]
    ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
    a_rel = ctx.download_accelerations()[targets]
    e_plain, e_rel = O.rms_relative_error(a_plain, ref), O.rms_relative_error(a_rel, ref)
    e_first = O.rms_relative_error(a_first, ref)
    m_rel = float(np.max(np.linalg.norm(a_rel - ref, axis=1) / np.linalg.norm(ref, axis=1)))
    print(f"10M: plain theta 0.5 rms={e_plain:.3e}; relative first={e_first:.3e} "
          f"rms={e_rel:.3e} max={m_rel:.3e}")
    assert e_plain <= 1e-3 and e_first <= 1e-3
    assert e_rel <= 1e-3 and m_rel < 0.05


@pytest.mark.parametrize("name,n,seed,theta,alpha", [
    ("plummer_collision", 200000, 42, 0.7, 0.0), ("plummer_collision", 200000, 42, 1.0, 0.004),
    ("globular_cluster", 40, 3, 0.7, 0.0), ("random_cloud", 1000, 8, 0.5, 0.0),
    ("globular_cluster", 50001, 5, 1.0, 0.003)])
def test_shared_top_walk_makes_the_same_decisions(cuda, ctx, name, n, seed, theta, alpha):
    """The walk whose top of the tree is traversed once per block of 4 groups
    accepts, opens and sums exactly the nodes of the per-group walk: the same
    counts of accepted cells and particle terms, and forces equal up to the
    order of the FP32 sums; partial blocks (n not a multiple of 128) included."""
    p = O.preset(name, n, seed)
    g = cuda.gravity_init(1.0, 0.01)
    if alpha > 0:  # the relative test reads previous forces: the same ones for both walks
        ctx.theta = theta
        ctx.upload(to_system(cuda, p))
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
        a_old = ctx.download_accelerations()
        p.ax[:], p.ay[:], p.az[:] = a_old.T
    out = {}
    for walk in (1, 2):
        ctx.set_walk(walk)
        ctx.theta = theta
        ctx.set_leaf_capacity(32 if alpha > 0 else 16)
        ctx.set_relative_opening(alpha)
        ctx.upload(to_system(cuda, p))
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
        out[walk] = (ctx.download_accelerations(), ctx.stats(), ctx.walk_restarts())
    (a1, s1, r1), (a2, s2, r2) = out[1], out[2]
    assert s1["accepted_approximations"] == s2["accepted_approximations"]
    assert s1["exact_interactions"] == s2["exact_interactions"]
    assert r1 == r2
    rel = np.linalg.norm(a1 - a2, axis=1) / np.maximum(np.linalg.norm(a1, axis=1), 1e-300)
    print(f"{name} n={n}: max rel {rel.max():.2e}, terms {s1['accepted_approximations']} + "
          f"{s1['exact_interactions']}")
    assert rel.max() < 1e-5
    assert O.rms_relative_error(a2, a1) < 1e-6


@pytest.mark.parametrize("theta", [0.5, 1.0])
def test_offset_opening_is_more_accurate(cuda, ctx, theta, walk):
    """The offset test (2h / theta + |com - cell centre| < d) accepts a subset of
    the reference test's cells: at theta 1.0 no target inside a cell accepts it,
    which removes most of the reference criterion's error there."""
    p = O.preset("plummer_collision", 200000, 42)
    targets = np.random.default_rng(2).choice(p.n, 1024, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, targets)
    a0, s0 = bh(cuda, p, 0.01, theta, ctx, walk=walk, opening=0)
    a1, s1 = bh(cuda, p, 0.01, theta, ctx, walk=walk, opening=1)
    e0 = O.rms_relative_error(a0[targets], ref)
    e1 = O.rms_relative_error(a1[targets], ref)
    print(f"theta={theta} reference={e0:.3e} offset={e1:.3e} "
          f"terms {s0['accepted_approximations'] + s0['exact_interactions']} -> "
          f"{s1['accepted_approximations'] + s1['exact_interactions']}")
    assert e1 < e0
    if theta == 1.0:
        assert e1 < 0.8 * e0
    b1, _ = bh(cuda, p, 0.01, theta, ctx, walk=walk, opening=1)
    assert np.array_equal(a1, b1)


def _resident(cuda, p, theta, opening=0, alpha=0.0, eps=0.01):
    ctx = cuda.CudaContext(theta=theta, opening=opening)
    ctx.set_relative_opening(alpha)
    ctx.upload(to_system(cuda, p))
    return ctx


@pytest.mark.parametrize("opening", [0, 1])
def test_relative_opening_limits_are_the_geometric_walk(cuda, opening):
    """alpha -> infinity: every relative test passes and the geometric test at
    theta alone decides.  No previous accelerations at all (a_old = 0, rms
    |a_old| = 0): the geometric test alone decides at the start angle
    min(theta, 0.5), so a fresh state under a loose bound (theta 1.0 or 5.0)
    gets an ordinary first evaluation, and the next one reads it."""
    p = O.preset("plummer_collision", 100000, 42)
    g = cuda.gravity_init(1.0, 0.01)

    def geometric(theta):
        with _resident(cuda, p, theta, opening=opening) as ctx:
            ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
            return ctx.download_accelerations()

    g10, g05, g04 = geometric(1.0), geometric(0.5), geometric(0.4)
    assert not np.array_equal(g10, g05)
    with _resident(cuda, p, 1.0, opening=opening) as ctx:
        ctx.set_relative_opening(1e30)
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)  # a_old = 0 here
        first = ctx.download_accelerations()
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)  # a_old = first
        huge = ctx.download_accelerations()
    assert np.array_equal(first, g05) and np.array_equal(huge, g10)
    for theta, expected in ((1.0, g05), (5.0, g05), (0.4, g04)):
        with _resident(cuda, p, theta, opening=opening, alpha=1e-3) as ctx:  # uploaded a = 0
            ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
            assert np.array_equal(ctx.download_accelerations(), expected), theta


def test_relative_opening_trades_accuracy_for_work(cuda):
    """G M (2h)^2 / d^4 <= alpha max(|a_old|, rms |a_old|): smaller alpha, more
    terms and a smaller error; at alpha 0.0025 the error is below the geometric
    theta 0.6 walk's with fewer terms."""
    p = O.preset("plummer_collision", 200000, 42)
    g = cuda.gravity_init(1.0, 0.01)
    targets = np.random.default_rng(2).choice(p.n, 1024, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, targets)
    rows = []
    with _resident(cuda, p, 0.6) as ctx:
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
        st = ctx.stats()
        geo = (O.rms_relative_error(ctx.download_accelerations()[targets], ref),
               st["accepted_approximations"] + st["exact_interactions"])
        ctx.theta = 1.0
        for alpha in (0.01, 0.0025, 0.001):
            ctx.set_relative_opening(alpha)
            ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)  # a_old: the last walk's
            st = ctx.stats()
            rows.append((alpha, O.rms_relative_error(ctx.download_accelerations()[targets], ref),
                         st["accepted_approximations"] + st["exact_interactions"]))
    print("geometric theta 0.6", geo, "relative", rows)
    assert rows[0][1] > rows[1][1] > rows[2][1]
    assert rows[0][2] < rows[1][2] < rows[2][2]
    assert rows[1][1] < geo[0] and rows[1][2] < geo[1]


def test_relative_opening_reads_the_views_accelerations(cuda):
    """Through the plugin function the previous accelerations come from the view;
    a view without them (all zero) gets the geometric walk at the start angle
    min(theta, 0.5), bit-equal to the plain theta-0.5 walk."""
    p = O.preset("plummer_collision", 100000, 42)
    g = cuda.gravity_init(1.0, 0.01)
    targets = np.random.default_rng(2).choice(p.n, 512, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, targets)
    s = to_system(cuda, p)
    with cuda.CudaContext(theta=0.5) as ctx:
        a0 = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, ctx).copy()
        st0 = ctx.stats()
        ctx.theta = 1.0
        ctx.set_relative_opening(0.0025)
        a = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, ctx)  # a_old = a0
        rel = O.rms_relative_error(a[targets], ref)
        st = ctx.stats()
        s.ax[:] = 0.0
        s.ay[:] = 0.0
        s.az[:] = 0.0
        b = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, ctx)  # no a_old
    work = lambda x: x["accepted_approximations"] + x["exact_interactions"]  # noqa: E731
    print(f"relative {rel:.3e} ({work(st)} terms) against theta 0.5 "
          f"{O.rms_relative_error(a0[targets], ref):.3e} ({work(st0)} terms)")
    assert rel < 2e-3 and work(st) < work(st0)
    assert np.array_equal(b, a0)


def test_relative_source_from_context_saves_the_upload(cuda):
    """FROM_CONTEXT: the plugin function takes the previous accelerations from
    the context's last result instead of uploading the view's.  Under a host
    leapfrog that passes the result back unchanged (integrator.c:47-85) the
    forces are bit-equal to FROM_VIEW's; the view's values are not read while
    the context's result is current, and they are again after a different
    acceleration array or a device-resident call."""
    p = O.preset("plummer_collision", 100000, 42)
    g = cuda.gravity_init(1.0, 0.01)
    h, dt = 5e-4, 1e-3
    systems, ctxs = [], []
    for source in (cuda.RelativeSource.FROM_VIEW, cuda.RelativeSource.FROM_CONTEXT):
        c = cuda.CudaContext(theta=1.0, leaf_capacity=32, relative_opening=0.003)
        c.set_relative_source(source)
        ctxs.append(c)
        systems.append(to_system(cuda, p))
    try:
        for s, c in zip(systems, ctxs):
            cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, c)
        for step in range(3):
            for s, c in zip(systems, ctxs):
                for v, a in ((s.vx, s.ax), (s.vy, s.ay), (s.vz, s.az)):
                    v += h * a
                for x, v in ((s.x, s.vx), (s.y, s.vy), (s.z, s.vz)):
                    x += dt * v
                cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, c)
                for v, a in ((s.vx, s.ax), (s.vy, s.ay), (s.vz, s.az)):
                    v += h * a
            assert np.array_equal(systems[0].acc(), systems[1].acc()), step
        (sv, cv), (sc, cc) = zip(systems, ctxs)
        again = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(sv, g, cv).copy()
        for a in (sc.ax, sc.ay, sc.az):
            a[:] = 0.0  # not read: the context's last result is current
        assert np.array_equal(
            cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(sc, g, cc), again)
        # another acceleration array (zeros): the view's are read, a fresh start
        fresh = to_system(cuda, p)
        for f in ("x", "y", "z", "m"):
            getattr(fresh, f)[:] = getattr(sc, f)
        start = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(fresh, g, cc).copy()
        with cuda.CudaContext(theta=0.5, leaf_capacity=32) as plain:
            ref = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(fresh, g, plain).copy()
        assert np.array_equal(start, ref)
        # a device-resident call in between: the view's are read again
        cc.upload(fresh)
        for a in (fresh.ax, fresh.ay, fresh.az):
            a[:] = 0.0
        assert np.array_equal(
            cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(fresh, g, cc), ref)
        with pytest.raises(cuda.CudaError):
            cc.set_relative_source(2)
    finally:
        for c in ctxs:
            c.close()


def test_opening_argument_checked(cuda, ctx):
    with pytest.raises(cuda.CudaError):
        ctx.set_opening(2)
    ctx.set_opening(cuda.Opening.REFERENCE)
    for bad in (-1.0, float("nan"), float("inf")):
        with pytest.raises(cuda.CudaError):
            ctx.set_relative_opening(bad)
    ctx.set_relative_opening(0.0)


@pytest.mark.parametrize("n", [1, 2, 3, 33, 4097, 10000])
def test_ragged_sizes(cuda, ctx, n, walk):
    p = O.preset("globular_cluster", n, 6)
    ref = O.gravity_reference(p.copy(), 1.0, 0.01)
    a, st = bh(cuda, p, 0.01, 0.5, ctx, walk=walk)
    if n == 1:
        assert np.all(a == 0.0)
    else:
        assert O.rms_relative_error(a, ref) < 1e-2
    assert st["node_count"] >= 1


def test_duplicate_positions_overflow_like_reference(cuda, ctx, walk):
    """barnes_hut.c:149-153: duplicate positions -> OVERFLOW."""
    p = O.preset("random_cloud", 500, 3)
    p.x[10], p.y[10], p.z[10] = p.x[20], p.y[20], p.z[20]
    s = to_system(cuda, p)
    with pytest.raises(cuda.CudaError) as e:
        cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, cuda.gravity_init(1.0, 0.01), ctx)
    assert e.value.status == cuda.Status.OVERFLOW
    p.x[10] += 1e-9
    bh(cuda, p, 0.01, 0.7, ctx)  # the context stays usable


def test_barnes_hut_kdk_steps(cuda, ctx, walk):
    """Leapfrog with barnes_hut_cuda forces tracks the all-pairs oracle run."""
    p = O.preset("globular_cluster", 20000, 12)
    g = cuda.gravity_init(1.0, 0.01)
    q = p.copy()
    O.gravity_reference(q, 1.0, 0.01, openmp=True)
    O.advance(q, 1.0, 0.01, 1e-3, 3, integrator=1, force=1)
    ctx.theta = 0.5
    ctx.set_multipole_order(2)
    ctx.set_walk(walk)
    s = to_system(cuda, p)
    ctx.upload(s)
    ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
    ctx.advance(g, 1e-3, 3, cuda.Algorithm.BARNES_HUT)
    ctx.download(s)
    assert O.rms_relative_error(s.acc(), q.acc()) < 5e-3
    assert np.max(np.abs(s.x - q.x)) < 1e-7


@pytest.mark.parametrize("order", [1, 2])
def test_zero_softening_is_finite_and_accurate(cuda, ctx, walk, order):
    """simd_equivalence_test.c:160-196 for the tree: eps = 0, the staged tiles
    drop each target's own r^2 = 0 term instead of dividing by zero."""
    p = O.preset("random_cloud", 3000, 7)
    ref = O.gravity_reference(p.copy(), 1.0, 0.0)
    cpu, _ = O.barnes_hut(p.copy(), 1.0, 0.0, 0.5)
    a, st = bh(cuda, p, 0.0, 0.5, ctx, order=order, walk=walk)
    assert np.all(np.isfinite(a))
    e_gpu, e_cpu = O.rms_relative_error(a, ref), O.rms_relative_error(cpu, ref)
    print(f"eps=0 order={order} gpu={e_gpu:.3e} cpu={e_cpu:.3e}")
    assert e_gpu <= e_cpu + 1e-6 and e_gpu < 1e-2


def test_heavy_masses_take_the_guarded_tiles(cuda, ctx, walk):
    """m / eps^3 beyond FP32 range (1e30 x 1e12): the self term cannot be
    W * 0, so the guarded tile loop runs; forces stay finite and scale with m."""
    p = O.preset("random_cloud", 2000, 3)
    light, _ = bh(cuda, p, 1e-4, 0.5, ctx, walk=walk)
    q = p.copy()
    q.m *= 1e30
    heavy, _ = bh(cuda, q, 1e-4, 0.5, ctx, walk=walk)
    assert np.all(np.isfinite(heavy))
    assert O.rms_relative_error(heavy / 1e30, light) < 1e-5
