"""The reference program's files, read and written from GPU state.

Text formats, byte for byte as the reference writes them:

* ``restart_file.dat`` (MDcode/main.c:272-289 write, :290-305 read): a header
  ``L\\titer\\tlast_saved_index`` (``%.14lf\\t%d\\t%d``) then one line per
  particle ``x_u y_u z_u px py pz type`` (``%.14lf`` x6, ``%d``), tab
  separated, reduced unfolded coordinates.
* ``ActiveFileIndex.dat`` (MDcode/active.c:4-29): the Nact active particle
  indices, ``%d`` per line, in active-slot order.
* ``ActiveDirection*.dat`` (MDcode/active.c:87-121): ``kx\\tky\\tkz`` per
  active slot.
* ``data_coor.out`` (MDcode/print.c:4-16): frames appended at the log-time
  steps, ``x_u\\ty_u\\tz_u\\ttype`` with ``%.5lf``.
* ``time_index_file.dat`` (MDcode/main.c:110-117): ``total timesteps equals
  %d`` then one step index (``%llu``) per line.

Python's ``%`` formatting rounds correctly like glibc's printf, so the files
are identical to the reference's for the same numbers (tested against the
reference's own ``write_restart_state``).

Resuming from a restart follows ``initialise_restart_state``
(MDcode/main.c:307-333): the wrapped position is the unfolded one reduced into
[0, 1) by repeated +-1 (``applypbc``, MDcode/time_evolve.c:27-37) and the
unfolded coordinate is reset to the wrapped one.
"""
from __future__ import annotations

import numpy as np

from .init import State


# ---------------------------------------------------------------------------
# restart_file.dat
def write_restart(path, L, xu, p, type_, iteration=0, last_saved_index=0):
    xu = np.asarray(xu, dtype=np.float64).reshape(-1, 3)
    p = np.asarray(p, dtype=np.float64).reshape(-1, 3)
    type_ = np.asarray(type_, dtype=np.int64)
    lines = ["%.14f\t%d\t%d\n" % (L, iteration, last_saved_index)]
    for i in range(xu.shape[0]):
        lines.append("%.14f\t%.14f\t%.14f\t%.14f\t%.14f\t%.14f\t%d\n" %
                     (xu[i, 0], xu[i, 1], xu[i, 2], p[i, 0], p[i, 1], p[i, 2], type_[i]))
    with open(path, "w") as f:
        f.write("".join(lines))


def read_restart(path, n):
    """(L, iteration, last_saved_index, x_u[n,3], p[n,3], type[n]) of the
    first n particle lines, like read_restart_state's fscanf loop."""
    with open(path) as f:
        head = f.readline().split()
        if len(head) < 3:
            raise ValueError(f"{path}: bad restart header")
        L, it, last = float(head[0]), int(head[1]), int(head[2])
        rows = []
        for _ in range(n):
            fields = f.readline().split()
            if len(fields) < 7:
                raise ValueError(f"{path}: expected {n} particle lines, found {len(rows)}")
            rows.append(fields[:7])
    a = np.array(rows)
    return L, it, last, a[:, 0:3].astype(np.float64), a[:, 3:6].astype(np.float64), a[:, 6].astype(np.int32)


def wrap_repeated(x):
    """applypbc: subtract 1 while x >= 1, then add 1 while x < 0.  The two
    loops run in that order once, so a tiny negative coordinate ends at
    exactly 1.0 as in the reference (the cell index is clamped downstream)."""
    x = np.array(x, dtype=np.float64, copy=True)
    while True:
        hi = x >= 1.0
        if not hi.any():
            break
        x[hi] -= 1.0
    while True:
        lo = x < 0.0
        if not lo.any():
            break
        x[lo] += 1.0
    return x


# ---------------------------------------------------------------------------
# active particles and directions
def write_active_index(path, index):
    with open(path, "w") as f:
        f.write("".join("%d\n" % int(i) for i in index))


def read_active_index(path, nact):
    with open(path) as f:
        v = [int(t) for t in f.read().split()[:nact]]
    if len(v) < nact:
        raise ValueError(f"{path}: expected {nact} indices, found {len(v)}")
    return np.array(v, dtype=np.int32)


def write_active_direction(path, k):
    """k is component-major, shape (3, Nact), as Engine.get_directions."""
    k = np.asarray(k).reshape(3, -1).T
    with open(path, "w") as f:
        f.write("".join("%d\t%d\t%d\n" % (int(a), int(b), int(c)) for a, b, c in k))


def read_active_direction(path, nact):
    with open(path) as f:
        v = [int(t) for t in f.read().split()[:3 * nact]]
    if len(v) < 3 * nact:
        raise ValueError(f"{path}: expected {nact} direction rows")
    return np.ascontiguousarray(np.array(v, dtype=np.int32).reshape(nact, 3).T)


def act_tag_from_index(n, index):
    """readActiveParticles: actTag = -1, then actTag[index[i]] = i."""
    tag = np.full(n, -1, dtype=np.int32)
    tag[np.asarray(index, dtype=np.int64)] = np.arange(len(index), dtype=np.int32)
    return tag


def active_index_from_tag(tag):
    tag = np.asarray(tag)
    nact = int((tag >= 0).sum())
    idx = np.empty(nact, dtype=np.int32)
    sel = np.nonzero(tag >= 0)[0]
    idx[tag[sel]] = sel
    return idx


# ---------------------------------------------------------------------------
# trajectory frames and the step index file
def append_frame(path, xu, type_):
    xu = np.asarray(xu, dtype=np.float64).reshape(-1, 3)
    with open(path, "a") as f:
        f.write("".join("%.5f\t%.5f\t%.5f\t%d\n" % (a, b, c, int(t)) for (a, b, c), t in zip(xu, type_)))


def write_time_index(path, steps):
    with open(path, "w") as f:
        f.write("total timesteps equals %d\n" % len(steps))
        f.write("".join("%d\n" % int(s) for s in steps))


def read_time_index(path):
    with open(path) as f:
        head = f.readline().split()
        count = int(head[-1])
        return np.array([int(f.readline()) for _ in range(count)], dtype=np.int64)


# ---------------------------------------------------------------------------
# engine <-> files
def save_run(engine, sys, restart_path, direction_path=None, index_path=None, iteration=0, last_saved_index=0):
    """write_restart_state + saveActiveDirection (+ the active index file)
    for system `sys` of an Engine."""
    x, xu, p, _ = engine.get_state(sys)
    st = engine.state_meta(sys)
    write_restart(restart_path, st["L"], xu, p, st["type"], iteration, last_saved_index)
    if direction_path is not None:
        write_active_direction(direction_path, engine.get_directions(sys))
    if index_path is not None:
        write_active_index(index_path, active_index_from_tag(st["act_tag"]))


def load_restart_state(restart_path, index_path, direction_path, n):
    """The State a reference restart resumes from (initialise_restart_state):
    x = applypbc(x_u), then x_u = x; active tags and directions from the two
    active files.  Returns (State, iteration, last_saved_index)."""
    L, it, last, xu, p, type_ = read_restart(restart_path, n)
    x = wrap_repeated(xu)
    with open(index_path) as f:
        idx = np.array([int(t) for t in f.read().split()], dtype=np.int32)
    if idx.size and (idx.min() < 0 or idx.max() >= n or np.unique(idx).size != idx.size):
        raise ValueError(f"{index_path}: active indices must be distinct and in [0, {n})")
    k = read_active_direction(direction_path, len(idx))
    st = State(L, x, x.copy(), p, type_.astype(np.int32), act_tag_from_index(n, idx), k)
    return st, it, last
