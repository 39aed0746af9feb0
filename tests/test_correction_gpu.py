"""Learned far-field correction: the tensor-core backward pass against the FP64
CPU MLP (oracle/mlp_oracle.py), training on GPU-generated (cell, target)
pairs, and what the trained network gains over plain Barnes-Hut.

Gradient tolerance: the GPU rounds inputs, weights and the hidden activations
to BF16 (8-bit mantissa) between products; against the FP64 chain rule on the
same BF16-rounded inputs and weights the gradient agrees to ~1e-2 relative,
bounded here at 5e-2 (L2) with cosine similarity > 0.998, the loss to 2e-2.
"""
import numpy as np
import pytest

import mlp_oracle as M
import oracle as O

pytestmark = pytest.mark.gpu


def to_system(nb, p):
    return nb.ParticleSystem(*[getattr(p, f).copy() for f in O.FIELDS])


def test_gradient_matches_fp64_cpu(cuda):
    rng = np.random.default_rng(0)
    x = rng.standard_normal((512, 10)).astype(np.float32)
    y = (0.3 * rng.standard_normal((512, 3))).astype(np.float32)
    with cuda.CudaCorrection(seed=3) as corr:
        p, _ = corr.parameters()
        g, loss = corr.gradient(x, y)
    ref_loss, ref_g = M.loss_and_gradient(p, x, y)
    rel = np.linalg.norm(g - ref_g) / np.linalg.norm(ref_g)
    cos = float(np.dot(g, ref_g) / (np.linalg.norm(g) * np.linalg.norm(ref_g)))
    print(f"gradient rel={rel:.3e} cos={cos:.6f} loss={loss:.6f} ref={ref_loss:.6f}")
    assert abs(loss - ref_loss) <= 2e-2 * ref_loss
    assert rel < 5e-2 and cos > 0.998
    # every parameter block receives gradient
    k = 0
    for name, shape in M.SIZES:
        n = int(np.prod(shape))
        assert np.linalg.norm(g[k:k + n]) > 0, name
        k += n


@pytest.mark.parametrize("rows", [128, 1000])
def test_tcgen05_forward_matches_mma_sync_and_fp64(cuda, rows):
    """The tcgen05 inference (128-row tiles, operands in shared memory,
    accumulators in tensor memory) against the warp-level mma.sync forward and
    the FP64 CPU MLP on the same BF16-rounded inputs and weights.  Both GPU
    paths round the hidden activations to BF16, so they agree to ~1e-3 and the
    FP64 chain to ~1e-2 (relative L2)."""
    rng = np.random.default_rng(5)
    feat = rng.standard_normal((rows, 10)).astype(np.float32)
    with cuda.CudaCorrection(seed=7) as corr:
        p, s = corr.parameters()
        y_tc = corr.evaluate(feat, "tcgen05")
        y_ms = corr.evaluate(feat, "mma_sync")
    x_mean, x_inv, y_mean, y_std = s[0:10], s[10:20], s[40:43], s[43:46]
    x = M.bf16((feat - x_mean) * x_inv)
    w = M.unpack(p)
    for k in ("W1", "W2", "W3"):
        w[k] = M.bf16(w[k])
    ref = M.forward(M.pack(w), x) * y_std + y_mean
    assert np.all(np.isfinite(y_tc)) and np.all(np.isfinite(y_ms))
    d_sync = np.linalg.norm(y_tc - y_ms) / np.linalg.norm(y_ms)
    d_ref = np.linalg.norm(y_tc - ref) / np.linalg.norm(ref)
    print(f"rows={rows}: tcgen05 vs mma.sync {d_sync:.2e}, vs FP64 {d_ref:.2e}")
    assert d_sync < 1e-2
    assert d_ref < 2e-2


def test_parameters_round_trip(cuda):
    with cuda.CudaCorrection(seed=5) as corr:
        p, s = corr.parameters()
        q = p * 0.5
        corr.set_parameters(q, s)
        p2, s2 = corr.parameters()
    assert np.array_equal(p2, q) and np.array_equal(s2, s)


@pytest.fixture(scope="module")
def trained(cuda):
    """A correction trained on the collision config at N = 200k (theta 1.0)."""
    p = O.preset("plummer_collision", 200000, 42)
    g = cuda.gravity_init(1.0, 0.01)
    ctx = cuda.CudaContext(theta=1.0)
    ctx.upload(to_system(cuda, p))
    corr = cuda.CudaCorrection(seed=11)
    corr.generate(ctx, g, theta=1.0, samples=1 << 20, seed=3)
    tl, vl = corr.train(epochs=8, batch=1024, learning_rate=1e-3)
    yield p, ctx, corr, tl, vl
    corr.close()
    ctx.close()


def test_training_data_is_sane(cuda, trained):
    _, _, corr, _, _ = trained
    f, lab, rows = corr.samples(max_rows=4096)
    assert rows >= (1 << 20) * 0.9
    assert np.all(np.isfinite(f)) and np.all(np.isfinite(lab))
    assert np.all(f[:, 3] > 0) and np.all(f[:, 3] < 1.0 + 1e-6)  # accepted at theta = 1
    # the residual of the monopole is a fraction of the monopole itself
    assert np.median(np.linalg.norm(lab, axis=1)) < 1.0


def test_training_lowers_the_loss(cuda, trained):
    _, _, _, tl, vl = trained
    print("train loss", tl, "validation loss", vl)
    assert vl[-1] < 0.5 * vl[0] or vl[-1] < 0.2
    assert vl[-1] < 1.0  # below the variance of the standardised labels


def test_correction_beats_plain_barnes_hut(cuda, trained):
    p, ctx, corr, _, _ = trained
    g = cuda.gravity_init(1.0, 0.01)
    targets = np.random.default_rng(9).choice(p.n, 1024, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, targets)
    s = to_system(cuda, p)
    ctx.set_multipole_order(1)
    ctx.set_correction(None)
    plain = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, ctx)[targets].copy()
    assert ctx.corrected_cells() == 0
    ctx.set_correction(corr)
    fixed = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, ctx)[targets].copy()
    corrected = ctx.corrected_cells()
    accepted = ctx.stats()["accepted_approximations"]
    ctx.set_correction(None)
    # one network evaluation per corrected (cell, 32-target group) pair: never
    # more than the accepted cells summed over all targets
    assert 0 < corrected <= accepted
    e_plain = O.rms_relative_error(plain, ref)
    e_fixed = O.rms_relative_error(fixed, ref)
    print(f"theta=1.0 plain monopole rms={e_plain:.3e} corrected rms={e_fixed:.3e}")
    # The network is evaluated once per (cell, 32-target group) and only for
    # cells farther than a few group radii; with buckets accepted like any cell
    # the remaining near-field error is untouched, so the gain is ~10%.
    assert e_fixed < 0.93 * e_plain


def test_out_of_range_features_fall_back_to_plain(cuda, trained):
    p, ctx, corr, _, _ = trained
    g = cuda.gravity_init(1.0, 0.01)
    s = to_system(cuda, p)
    params, scaling = corr.parameters()
    ctx.set_correction(None)
    plain = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, ctx).copy()
    with cuda.CudaCorrection(seed=1) as empty:
        bad = scaling.copy()
        bad[20:30] = 1e30   # minimum above everything: no cell is in range
        bad[30:40] = -1e30
        empty.set_parameters(params, bad)
        ctx.set_correction(empty)
        guarded = cuda.n_body_sim_pro_barnes_hut_compute_acceleration_cuda(s, g, ctx).copy()
        assert ctx.corrected_cells() == 0
        ctx.set_correction(None)
    assert np.array_equal(guarded, plain)


def test_corrected_walk_on_the_1m_collision(cuda):
    """The bench's recipe at the config-2 size: the network trained on 2^22
    (cell, target) pairs of the 1M two-Plummer collision with the project's own
    kernels, then the corrected walk at theta 1.0 on the same state against the
    FP64 oracle on 4096 seeded targets.  The correction must remove at least a
    third of the plain monopole's rms error there (rms 1e-3 at theta 1.0 is out
    of its reach: the cells nearer a group than 1/0.3 of its radius keep the
    plain monopole), list only cells it can evaluate, and be bitwise repeatable."""
    n = 1_000_000
    g = cuda.gravity_init(1.0, 0.01)
    with cuda.CudaContext(theta=1.0) as ctx, cuda.CudaCorrection(seed=11) as corr:
        ctx.generate_plummer_collision(n, 42)
        s = cuda.ParticleSystem.zeros(n)
        ctx.download(s)
        p = O.Particles.zeros(n)
        for f in O.FIELDS:
            getattr(p, f)[:] = getattr(s, f)
        targets = np.random.default_rng(11).choice(n, 4096, replace=False)
        ref = O.gravity_subset(p, 1.0, 0.01, targets)
        corr.generate(ctx, g, theta=1.0, samples=1 << 22, seed=3)
        _, vl = corr.train(epochs=8, batch=1024, learning_rate=1e-3)
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
        plain = ctx.download_accelerations()[targets]
        ctx.set_correction(corr)
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
        a1 = ctx.download_accelerations()
        evals = ctx.corrected_cells()
        ctx.compute_acceleration(g, cuda.Algorithm.BARNES_HUT)
        a2 = ctx.download_accelerations()
    e_plain = O.rms_relative_error(plain, ref)
    e_corr = O.rms_relative_error(a1[targets], ref)
    print(f"1M theta 1.0: plain rms={e_plain:.3e} corrected rms={e_corr:.3e} "
          f"evaluations={evals} validation loss={vl[-1]:.4f}")
    assert np.array_equal(a1, a2)
    assert 0 < evals < n * 512 // 32
    assert e_corr <= 0.67 * e_plain
