"""How far a learned correction of the monopole could take theta 1.0.

The correction network sees one accepted cell and one evaluation point and
predicts the cell's monopole error there; it is trained on cells that look wide
from the target (2h / d >= 0.7 theta).  The oracle's walk (the reference's tree
and criterion, barnes_hut.c:549-636) splits the theta-1.0 monopole error of every
target exactly by the apparent size of the accepted cells, so the error left by
a PERFECT per-target correction of a band of cells, and the number of network
rows that band costs, follow without any network at all.

On the two-Plummer collision at theta 1.0: correcting the whole training band
perfectly still leaves the rms error above 1e-3, and reaching 1e-3 takes the
band down to about half of theta, i.e. most of the accepted cells -- hundreds
of network rows per target per step.
"""
import numpy as np

import oracle as O

BINS = 20


def _bands(n, targets, theta=1.0):
    p = O.plummer_collision_parallel(n, 42)
    tg = np.random.default_rng(11).choice(n, targets, replace=False)
    ref = O.gravity_subset(p, 1.0, 0.01, tg)
    err, count = O.barnes_hut_residual_bands(p, 1.0, 0.01, theta, tg, BINS)
    a_bh, _ = O.barnes_hut(p.copy(), 1.0, 0.01, theta)
    return ref, err, count, a_bh[tg]


def _left_after(err, ref, band):
    """rms relative error left when every accepted cell with (2h / d) / theta >=
    band is corrected exactly."""
    b = int(round(band * BINS))
    rest = err[:, :b].sum(axis=1)
    return float(np.sqrt((rest ** 2).sum() / (ref ** 2).sum()))


def test_bands_add_up_to_the_walk_error():
    ref, err, count, a_bh = _bands(20000, 256)
    assert np.abs(err.sum(axis=1) - (a_bh - ref)).max() <= 1e-12 * np.abs(ref).max()
    assert _left_after(err, ref, 0.0) == 0.0
    assert abs(_left_after(err, ref, 1.0) - O.rms_relative_error(a_bh, ref)) < 1e-12
    assert count.sum(axis=1).min() > 0


def test_a_perfect_band_correction_at_theta_1():
    ref, err, count, _ = _bands(100000, 512)
    plain = _left_after(err, ref, 1.0)
    band = _left_after(err, ref, 0.7)
    left = {b / BINS: _left_after(err, ref, b / BINS) for b in range(BINS + 1)}
    needed = max(b for b, e in left.items() if e <= 1e-3)  # widest band still short
    rows = count[:, int(round(needed * BINS)):].sum(axis=1).mean()
    cells = count.sum(axis=1).mean()
    print(f"theta 1.0: plain {plain:.3e}; training band exact {band:.3e}; 1e-3 needs "
          f"(2h/d)/theta >= {needed:.2f}: {rows:.0f} of {cells:.0f} cells per target")
    assert plain > 1e-2
    assert band > 2e-3            # even a perfect network on its band misses 1e-3
    assert needed <= 0.55         # 1e-3 needs the band down to about half of theta
    assert rows >= 0.5 * cells    # ... which is most of the accepted cells
    # from no correction through half the band to all of it (the partial sums of
    # error vectors need not fall at every step, the ends do)
    assert left[1.0] >= left[0.5] >= left[0.0] == 0.0
