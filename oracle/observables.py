"""numpy restatement of the reference's trajectory analysis.  TEST
INFRASTRUCTURE ONLY: the device's in-place observables are checked against it.

* log_pairs — the (origin, later step, time bin) pairs that Analysis/overlap.c
  and Analysis/msd_pos.c visit: origins every run/num_origins steps
  (prepareSavingArray, MDcode/main.c:71-95), offsets 1 then *factor truncated
  (+1 when that does not advance) below max_interval (Analysis/overlap.c:28,
  50-100), one time bin per offset; origins that find no free snapshot slot
  among max_live are left out, as on the device.
* pair_sums — per (origin frame, later frame): the overlap count with the
  minimum image of Analysis/overlap.c:61-83, |dr|^2, sum dx^4, |dr|^4 of
  Analysis/msd_pos.c:64-76, and sum over wave vectors of cos(q.dr).
"""
from __future__ import annotations

import numpy as np


def offsets(run_length, factor, max_interval):
    out, off = [], 1
    while off < max_interval and off < run_length:
        out.append(off)
        nxt = int(off * factor)
        off = off + 1 if nxt == off else int(float(off) * factor)
    return out


def log_pairs(run_length, num_origins, factor, max_interval=0, max_live=64):
    maxint = max_interval if max_interval > 0 else run_length // 2
    offs = offsets(run_length, factor, maxint)
    lin = run_length // num_origins
    busy = [-1] * max_live
    pairs = []
    for k in range(num_origins):
        t0 = k * lin
        valid = [(m, o) for m, o in enumerate(offs) if t0 + o < run_length]
        last = t0 + valid[-1][1] if valid else t0
        slot = next((q for q in range(max_live) if busy[q] < t0), None)
        if slot is None:
            continue
        busy[slot] = last
        pairs += [(t0, t0 + o, m) for m, o in valid]
    return offs, pairs


def pair_sums(x0, x1, L, a, qvec=None):
    """Sums over particles for one (origin, later) pair of unfolded reduced
    coordinates: (overlap count, sum |dr|^2, sum d^4, sum |dr|^4, sum_q cos)."""
    d = x1 - x0
    m = d.copy()
    m = np.where(m >= 0.5, m - 1.0, np.where(m < -0.5, m + 1.0, m))
    r2q = L * L * (m * m).sum(axis=1)
    ov = float((r2q < a * a).sum())
    r2 = L * L * (d * d).sum(axis=1)
    r4 = L * L * L * L * (d ** 4).sum(axis=1)
    fs = 0.0
    if qvec is not None and len(qvec):
        fs = float(np.cos(2 * np.pi * (d @ np.asarray(qvec, dtype=np.float64).T)).sum())
    return ov, float(r2.sum()), float(r4.sum()), float((r2 * r2).sum()), fs


def analyse(frames, L, run_length, num_origins, factor, max_interval, a, qvec=None, max_live=64,
            skip_missing=False):
    """Per-bin sums (Q, Q^2, msd, msd_d4, msd_r4, Fs, count) from frames =
    {step: [N,3] unfolded reduced coordinates}, as the device accumulates them.
    skip_missing: leave out pairs whose frame is absent, as the reference's
    frame lookup does (Analysis/overlap.c:55-57)."""
    offs, pairs = log_pairs(run_length, num_origins, factor, max_interval, max_live)
    out = np.zeros((len(offs), 7))
    nq = 0 if qvec is None else len(qvec)
    for t0, t1, m in pairs:
        if skip_missing and (t0 not in frames or t1 not in frames):
            continue
        x0, x1 = frames[t0], frames[t1]
        n = x0.shape[0]
        ov, r2, r4, r2sq, fs = pair_sums(x0, x1, L, a, qvec)
        Q = ov / n
        out[m] += [Q, Q * Q, r2 / n, r4 / n, r2sq / n, fs / (n * nq) if nq else 0.0, 1.0]
    return np.asarray(offs), out
