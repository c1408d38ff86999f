"""Launch-shape autotuner for an Engine.

Times the force stage (acg_time_stage, forces only, so the trajectory is not
changed) for each candidate launch shape of the force kernels and keeps the
fastest: threads per particle of the cell-group and whole-box kernels, and
threads per particle x block size of the per-particle kernel (boxes with fewer
than 3 cells per side that are too large for the whole-box kernels).  Each candidate is timed over `reps` launches after a
warm launch.
"""
from __future__ import annotations

from .engine import Engine
from .init import box_length

GROUP_TPP = (1, 2, 4)
SMALL_SHAPES = ((1, 64), (1, 128), (2, 128), (2, 256), (4, 128), (4, 256), (8, 256))


def autotune(e: Engine, reps: int = 20, verbose: bool = False) -> dict:
    # the per-particle kernel serves boxes with fewer than 3 cells per side
    # (Ncell = (int)((int)L / 2.85)) that are too large for the whole-box kernels
    def per_particle(r):
        nc = int(int(box_length(e.n(r))) / 2.85)
        return nc < 2 or (nc < 3 and e.n(r) > 8192)
    has_small = any(per_particle(r) for r in range(e.nsys))
    best_g, best_t = None, float("inf")
    for g in GROUP_TPP:
        e.set_group_tpp(g)
        e.time_stage(1, 1)
        t = e.time_stage(1, reps)
        if verbose:
            print(f"group tpp {g}: {t * 1e3:.1f} us")
        if t < best_t:
            best_g, best_t = g, t
    e.set_group_tpp(best_g)
    best_s = e.get_launch()
    if has_small:
        best_t2 = float("inf")
        for tpp, block in SMALL_SHAPES:
            e.set_launch(tpp, block)
            e.time_stage(1, 1)
            t = e.time_stage(1, reps)
            if verbose:
                print(f"small-box kernel tpp {tpp} block {block}: {t * 1e3:.1f} us")
            if t < best_t2:
                best_s, best_t2 = (tpp, block), t
        e.set_launch(*best_s)
        best_t = best_t2
    return {"group_tpp": best_g, "tpp": best_s[0], "block": best_s[1], "force_ms": best_t}
