"""The observables' schedule restatement against the reference's frame
schedule, and the pair sums on hand-made displacements.  CPU only."""
import numpy as np

from oracle import Oracle
from oracle.observables import log_pairs, offsets, pair_sums


def test_pairs_use_only_scheduled_frames():
    run, no = 20000, 200
    frames = set(int(s) for s in Oracle.log_schedule(run, no, 1.4))
    _, pairs = log_pairs(run, no, 1.4, 0, max_live=200)
    needed = {s for a, b, _ in pairs for s in (a, b)}
    # prepareSavingArray drops its largest entry (1-based shell sort on a
    # 0-based array); that one frame is the only one missing
    assert needed - frames == {max(needed)}


def test_offsets_follow_the_reference_rule():
    assert offsets(10 ** 6, 1.4, 100) == [1, 2, 3, 4, 5, 7, 9, 12, 16, 22, 30, 42, 58, 81]


def test_slots_limit_origins():
    _, p_all = log_pairs(600, 6, 1.4, 300, max_live=64)
    _, p_few = log_pairs(600, 6, 1.4, 300, max_live=1)
    assert len({a for a, _, _ in p_all}) == 6
    assert len({a for a, _, _ in p_few}) < 6


def test_pair_sums_by_hand():
    L = 10.0
    x0 = np.zeros((4, 3))
    x1 = np.array([[0.01, 0, 0], [0.1, 0, 0], [0.95, 0, 0], [0.02, 0.02, 0.0]])
    ov, r2, r4, r2sq, fs = pair_sums(x0, x1, L, 0.3, qvec=[[1, 0, 0]])
    # |dr| = 0.1, 1.0, 0.5 (after the minimum image, 9.5 without), 0.283
    assert ov == 2.0
    assert np.isclose(r2, 0.01 + 1.0 + 90.25 + 0.08)
    assert np.isclose(r4, 1e-4 + 1.0 + 9.5 ** 4 + 2 * 0.2 ** 4)
    assert np.isclose(fs, np.cos(2 * np.pi * 0.01) + np.cos(2 * np.pi * 0.1) + np.cos(2 * np.pi * 0.95)
                      + np.cos(2 * np.pi * 0.02))
